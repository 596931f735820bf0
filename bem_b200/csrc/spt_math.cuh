// Device math for the tracer: complete elliptic integrals K(1-p), E(1-p)
// and the unit-charge ring field, float64 and float32.
//
// K and E are computed here from published methods (not from SciPy's or
// CUDA's code):
//   * p < 1e-3 : the logarithmic series about m = 1 of DLMF 19.12.1 (K) and
//                19.12.2 (E), in powers of p = 1 - m with L = ln(1/sqrt(p)):
//                K = sum a_n^2 p^n (L + d_n),
//                E = 1 + (p/2) sum b_n p^n (L + d_n - 1/((2n+1)(2n+2))),
//                a_n = (1/2)_n/n!, b_n = (1/2)_n (3/2)_n / ((2)_n n!),
//                d_n = psi(1+n) - psi(1/2+n) = 2 ln 2 - sum_{k<=n} 1/(k(2k-1)).
//                Ten terms keep the truncation below 1e-29 for p < 1e-3.
//   * p >= 1e-3: the arithmetic-geometric mean, DLMF 19.8.1 (K = pi/(2 M)) and
//                19.8.6 (E = K (1 - sum 2^(n-1) c_n^2)), started from
//                a0 = 1, b0 = sqrt(p), c0^2 = 1 - p.
// Checked against SciPy's ellipkm1/ellipe to 3 ulp on p in [1e-300, 1].
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace spt {

constexpr double kPi = 3.141592653589793;

// Series coefficients of the two DLMF 19.12 expansions (a_n^2, a_n^2 d_n,
// b_n, b_n (d_n - 1/((2n+1)(2n+2)))), n = 0..9, computed from the
// recurrences a_n = a_{n-1}(n-1/2)/n, b_n = b_{n-1}(n-1/2)(n+1/2)/((n+1)n),
// d_n = d_{n-1} - 1/(n(2n-1)), d_0 = 2 ln 2.
static __device__ __constant__ double kSerK[10] = {
    1.0, 0.25, 0.140625, 0.09765625, 0.07476806640625, 0.0605621337890625,
    0.050889015197753906, 0.043878793716430664, 0.03856534603983164, 0.034399336436763406};
static __device__ __constant__ double kSerKd[10] = {
    1.3862943611198906, 0.09657359027997264, 0.030885144532484612, 0.01493760036978098,
    0.008766312197176064, 0.0057548876844001106, 0.004064658549993974, 0.003022546550344074,
    0.0023351571703480825, 0.0018580702734561816};
static __device__ __constant__ double kSerE[10] = {
    1.0, 0.375, 0.234375, 0.1708984375, 0.13458251953125, 0.11103057861328125,
    0.09450817108154297, 0.0822727382183075, 0.0728456536307931, 0.06535873922985047};
static __device__ __constant__ double kSerEd[10] = {
    0.8862943611198906, 0.11361038541995896, 0.043662740887474356, 0.023089042834616717,
    0.014284000626791913, 0.00970948667432989, 0.007029375927562748, 0.005324471705985524,
    0.004172794741275812, 0.0033583368373829277};

__device__ __forceinline__ double horner10(const double* c, double p) {
    double s = c[9];
#pragma unroll
    for (int n = 8; n >= 0; --n) s = fma(s, p, c[n]);
    return s;
}

// K(1-p), E(1-p), float64.
__device__ __forceinline__ void ellip_ke(double p, double& K, double& E) {
    if (p < 1e-3) {
        const double L = -0.5 * log(p);
        K = fma(L, horner10(kSerK, p), horner10(kSerKd, p));
        E = fma(0.5 * p, fma(L, horner10(kSerE, p), horner10(kSerEd, p)), 1.0);
        return;
    }
    double a = 1.0, b = sqrt(p);
    double S = 0.5 * (1.0 - p), w = 0.5;
#pragma unroll 1
    for (int it = 0; it < 12; ++it) {
        const double c = 0.5 * (a - b);
        const double an = 0.5 * (a + b);
        b = sqrt(a * b);
        a = an;
        w += w;
        S = fma(w * c, c, S);
        if (fabs(c) <= 1e-17 * a) break;
    }
    K = kPi / (2.0 * a);
    E = K * (1.0 - S);
}

// Field (E_rho, E_z) at (rho, z) of a unit-total-charge ring of radius a at
// height 0 (G = 1/(4 pi r) convention), float64.  The formula and the
// near-axis Taylor branch follow bem/axisymmetric.py:248-265.
__device__ __forceinline__ void ring_field(double rho, double z, double a, double& er, double& ez) {
    const double z2 = z * z, a2 = a * a, rho2 = rho * rho;
    const double D = (rho + a) * (rho + a) + z2;
    const double d2 = (rho - a) * (rho - a) + z2;
    if (rho2 < 1e-10 * (a2 + z2)) {
        const double ax2 = a2 + z2;
        const double s = sqrt(ax2);
        const double ax15 = ax2 * s, ax25 = ax2 * ax15, ax35 = ax2 * ax25;
        er = rho * (2.0 * z2 - a2) / (8.0 * kPi * ax25);
        ez = z / (4.0 * kPi * ax15) + 3.0 * rho2 * z * (3.0 * a2 - 2.0 * z2) / (16.0 * kPi * ax35);
        return;
    }
    double K, E;
    ellip_ke(d2 / D, K, E);
    const double sD = sqrt(D);
    er = (K - (a2 - rho2 + z2) * E / d2) / (4.0 * kPi * kPi * rho * sD);
    ez = z * E / (2.0 * kPi * kPi * sD * d2);
}


// Same K(1-p), E(1-p) with a fixed six-step AGM (no data-dependent exit) so
// several evaluations can be interleaved by the compiler.  For p >= 1e-3 the
// sixth half-difference c_6 is below 1e-14, so a_6 has converged to the AGM
// (its error is c_7 ~ 1e-28) and the neglected E-sum terms are below 1e-26.
// The series branch (p < 1e-3: the point within ~3 % of the ring's radius
// of the ring) out of line: it is rare in a far sum, and every interleaved
// copy of the AGM below would otherwise carry its own copy of it.
static __device__ __noinline__ void ellip_ke_series(double p, double& K, double& E) {
    const double L = -0.5 * log(p);
    K = fma(L, horner10(kSerK, p), horner10(kSerKd, p));
    E = fma(0.5 * p, fma(L, horner10(kSerE, p), horner10(kSerEd, p)), 1.0);
}

__device__ __forceinline__ void ellip_ke_fixed(double p, double& K, double& E) {
    if (p < 1e-3) {
        ellip_ke_series(p, K, E);
        return;
    }
    double a = 1.0, b = sqrt(p);
    double S = 0.5 * (1.0 - p), w = 0.5;
#pragma unroll
    for (int it = 0; it < 6; ++it) {
        const double c = 0.5 * (a - b);
        const double an = 0.5 * (a + b);
        b = sqrt(a * b);
        a = an;
        w += w;
        S = fma(w * c, c, S);
    }
    K = (0.5 * kPi) / a;
    E = K * (1.0 - S);
}

// Near-axis Taylor branch of the ring field (rho^2 < 1e-10 (a^2 + z^2)), out
// of line for the same reason as ellip_ke_series.
static __device__ __noinline__ void ring_axis_taylor(double rho, double z, double a, double& er, double& ez) {
    const double z2 = z * z, a2 = a * a, rho2 = rho * rho;
    const double ax2 = a2 + z2;
    const double s = sqrt(ax2);
    const double ax15 = ax2 * s, ax25 = ax2 * ax15, ax35 = ax2 * ax25;
    er = rho * (2.0 * z2 - a2) / (8.0 * kPi * ax25);
    ez = z / (4.0 * kPi * ax15) + 3.0 * rho2 * z * (3.0 * a2 - 2.0 * z2) / (16.0 * kPi * ax35);
}

// Ring field for the far-quadrature sum: the formula of ring_field with one
// reciprocal of D*d2 in place of the divisions by D and d2, and 1/rho
// supplied by the caller (constant over a point's whole node loop).
__device__ __forceinline__ void ring_field_far(double rho, double inv_rho, double z, double a, double& er,
                                               double& ez) {
    const double z2 = z * z, a2 = a * a, rho2 = rho * rho;
    const double D = (rho + a) * (rho + a) + z2;
    const double d2 = (rho - a) * (rho - a) + z2;
    if (rho2 < 1e-10 * (a2 + z2)) {
        ring_axis_taylor(rho, z, a, er, ez);
        return;
    }
    const double inv = 1.0 / (D * d2);
    const double invD = d2 * inv, inv_d2 = D * inv;
    double K, E;
    ellip_ke_fixed(d2 * invD, K, E);
    const double rsD = sqrt(invD);
    er = (K - (a2 - rho2 + z2) * E * inv_d2) * (rsD * inv_rho * (1.0 / (4.0 * kPi * kPi)));
    ez = z * E * rsD * inv_d2 * (1.0 / (2.0 * kPi * kPi));
}

// ring_field_far out of line, for the rare float64 terms of a float32 sum.
static __device__ __noinline__ void ring_field_far_cold(double rho, double inv_rho, double z, double a, double& er,
                                                        double& ez) {
    ring_field_far(rho, inv_rho, z, a, er, ez);
}

// ---------------------------------------------------------------------------
// float32 variants (SPT_FORM_MIXED).
//
// K(1-p), E(1-p) for p >= 1e-3 from the polynomial-logarithmic
// approximations of C. Hastings Jr. (Approximations for Digital Computers,
// 1955) as tabulated in Abramowitz & Stegun, Handbook of Mathematical
// Functions, 17.3.34 (K) and 17.3.36 (E), with m1 = 1 - m = p:
//   K = sum_{i<=4} a_i p^i + ln(1/p) sum_{i<=4} b_i p^i,   |error| <= 2e-8,
//   E = 1 + sum_{1<=i<=4} c_i p^i + ln(1/p) sum_{1<=i<=4} d_i p^i,  |error| <= 2e-8
// (checked against SciPy's ellipkm1/ellipe: 1.3e-8 and 1.6e-8 at most on
// p in [1e-6, 1]), below float32 rounding: one logarithm and four degree-4
// Horner chains instead of the AGM's six square roots.
__device__ __forceinline__ void ellip_ke_hastings_f(float p, float& K, float& E) {
    const float L = -__logf(p);
    const float ka = fmaf(fmaf(fmaf(fmaf(0.01451196212f, p, 0.03742563713f), p, 0.03590092383f), p, 0.09666344259f), p,
                          1.38629436112f);
    const float kb = fmaf(fmaf(fmaf(fmaf(0.00441787012f, p, 0.03328355346f), p, 0.06880248576f), p, 0.12498593597f), p,
                          0.5f);
    const float ea = fmaf(fmaf(fmaf(fmaf(0.01736506451f, p, 0.04757383546f), p, 0.06260601220f), p, 0.44325141463f), p,
                          1.0f);
    const float eb = fmaf(fmaf(fmaf(0.00526449639f, p, 0.04069697526f), p, 0.09200180037f), p, 0.24998368310f) * p;
    K = fmaf(kb, L, ka);
    E = fmaf(eb, L, ea);
}

// The series branch (DLMF 19.12, four terms, truncation < 1e-9) below
// p = 1e-2, Hastings above.
__device__ __forceinline__ void ellip_ke_f(float p, float& K, float& E) {
    if (p >= 1e-2f) {
        ellip_ke_hastings_f(p, K, E);
        return;
    }
    const float L = -0.5f * __logf(p);
    const float A = fmaf(fmaf(fmaf(0.09765625f, p, 0.140625f), p, 0.25f), p, 1.0f);
    const float B = fmaf(fmaf(fmaf(0.01493760037f, p, 0.03088514453f), p, 0.09657359028f), p, 1.386294361f);
    const float C = fmaf(fmaf(fmaf(0.1708984375f, p, 0.234375f), p, 0.375f), p, 1.0f);
    const float D = fmaf(fmaf(fmaf(0.02308904283f, p, 0.04366274089f), p, 0.1136103854f), p, 0.8862943611f);
    K = fmaf(L, A, B);
    E = fmaf(0.5f * p, fmaf(L, C, D), 1.0f);
}

__device__ __forceinline__ void ring_field_f(float rho, float z, float a, float& er, float& ez) {
    const float z2 = z * z, a2 = a * a, rho2 = rho * rho;
    const float D = (rho + a) * (rho + a) + z2;
    const float d2 = (rho - a) * (rho - a) + z2;
    if (rho2 < 1e-10f * (a2 + z2)) {
        const float ax2 = a2 + z2;
        const float r1 = rsqrtf(ax2);
        const float i15 = r1 / ax2, i25 = i15 / ax2, i35 = i25 / ax2;
        er = rho * (2.0f * z2 - a2) * i25 * (1.0f / (8.0f * 3.14159265f));
        ez = z * i15 * (1.0f / (4.0f * 3.14159265f)) + 3.0f * rho2 * z * (3.0f * a2 - 2.0f * z2) * i35 * (1.0f / (16.0f * 3.14159265f));
        return;
    }
    float K, E;
    const float invD = __frcp_rn(D);
    ellip_ke_f(d2 * invD, K, E);
    const float rsD = rsqrtf(D);
    const float inv_d2 = __frcp_rn(d2);
    er = (K - (a2 - rho2 + z2) * E * inv_d2) * rsD * __frcp_rn(rho) * (1.0f / (4.0f * 9.8696044f));
    ez = z * E * rsD * inv_d2 * (1.0f / (2.0f * 9.8696044f));
}


// float32 unit-ring field near the axis: with r^2 = a^2 + z^2, x = rho / r and
// t = z / r, the potential of the ring expands in Legendre polynomials of t
// (the z-derivatives of the on-axis potential 1 / (4 pi r)):
//   E_rho = 1/(4 pi r^2) sum_{k>=1} (-1)^(k+1) c_k x^(2k-1) P_2k(t)
//   E_z   = 1/(4 pi r^2) sum_{k>=0} (-1)^k c_(k+1) x^(2k) P_(2k+1)(t)
// with c_k = 2k binom(2k, k) / 4^k.  Every term is O(1): no cancellation and
// no overflow for nm rings.  Terms through P_17; for x^2 < 0.09 the remainder
// is below 2e-8 of 1/(4 pi r^2).
__device__ __forceinline__ void ring_axis_f(float rho, float z, float a, float& er, float& ez) {
    constexpr float ck[10] = {0.0f, 1.0f, 1.5f, 1.875f, 2.1875f, 2.4609375f, 2.70703125f, 2.9326171875f,
                              3.14208984375f, 3.338470458984375f};
    const float r2 = fmaf(a, a, z * z);
    const float ir = rsqrtf(r2);
    const float x = rho * ir, t = z * ir, x2 = x * x;
    float pm = 1.0f, pn = t;  // P_(n-1), P_n
    float sr = 0.0f, sz = t;  // E_z term k = 0: c_1 P_1
    float xo = x, xe = x2;    // x^(2k-1) for the next E_rho term, x^(2k) for the next E_z term
#pragma unroll
    for (int n = 1; n <= 16; ++n) {
        const float pnext = ((float)(2 * n + 1) * t * pn - (float)n * pm) * (1.0f / (float)(n + 1));
        pm = pn;
        pn = pnext;
        if ((n + 1) % 2 == 0) {
            const int k = (n + 1) / 2;
            const float term = ck[k] * xo * pn;
            sr = (k % 2 == 1) ? sr + term : sr - term;
            xo *= x2;
        } else {
            const int k = n / 2;
            const float term = ck[k + 1] * xe * pn;
            sz = (k % 2 == 0) ? sz + term : sz - term;
            xe *= x2;
        }
    }
    const float s = 0.07957747154594767f * (ir * ir);  // 1/(4 pi r^2)
    er = s * sr;
    ez = s * sz;
}

// float32 ring field for the far sum of the mixed form.  dr = rho - a and
// sr = rho + a are formed in float64 by the caller (rho and a are close near
// a wall), then rounded.  Near the axis (rho^2 < 0.09 (a^2 + z^2)) the
// Legendre expansion above; elsewhere K and E from the Hastings
// approximations (p >= 1e-3) -- the radial formula's cancellation there costs
// at most ~eps_f / x of the ring's field scale.  Returns false (the caller
// evaluates the pair in float64) when p = d2 / D < 1e-3: the point is close
// to the ring itself.
__device__ __forceinline__ bool ring_far_f(float rho, float inv_rho, float dr, float sr, float z, float a, float& er,
                                           float& ez) {
    const float z2 = z * z, a2 = a * a, rho2 = rho * rho;
    if (rho2 < 0.09f * (a2 + z2)) {
        ring_axis_f(rho, z, a, er, ez);
        return true;
    }
    const float D = fmaf(sr, sr, z2);
    const float d2 = fmaf(dr, dr, z2);
    const float invD = __frcp_rn(D);
    const float p = d2 * invD;
    const bool ok = p >= 1e-3f;
    float K, E;
    ellip_ke_hastings_f(fminf(fmaxf(p, 1e-3f), 1.0f), K, E);
    const float inv_d2 = __frcp_rn(d2);
    const float rsD = rsqrtf(D);
    er = (K - (a2 - rho2 + z2) * E * inv_d2) * (rsD * inv_rho * 0.025330295910584444f);  // 1/(4 pi^2)
    ez = z * E * rsD * inv_d2 * 0.05066059182116889f;                                    // 1/(2 pi^2)
    return ok;
}

__device__ __forceinline__ void kahan_add(float& s, float& c, float v) {
    const float y = v - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
}

}  // namespace spt
