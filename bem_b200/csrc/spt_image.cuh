// Device code of the BEM image-charge force (bem/toroidal.py,
// bem/ring_modes.py, bem/image_charge.py): toroidal harmonics, the local
// mirror charge, and `group_force`, the force on one group computed by a
// whole CTA.  Used by the standalone entry point (spt_image.cu) and, for
// geometries built with an image plane z0, inside the persistent trace
// kernel's stage evaluation (spt_device.cuh).
#pragma once
#include <stdint.h>

#include "spt_b200.h"
#include "spt_math.cuh"

namespace spt_img {

constexpr double kPi = 3.14159265358979323846;
constexpr double kChiMin = 1.0000000000000002;  // the next double above 1 (bem/toroidal.py:205)

// Downward ratio recurrence: start M + pad terms above the last mode needed.
// The continued fraction's truncation error after pad terms is about
// exp(-2 eta pad); pad >= 22 / eta keeps it below 1e-19, far under a double's
// rounding (the reference pads by max(50, 40 / eta) for the same limit, so
// both give the converged ratios).
constexpr int kPadMin = 4;
constexpr double kPadConst = 22.0;

// chi = 1 + ((rho - a)^2 + (z - za)^2) / (2 rho a) (bem/ring_modes.py:81-89)
// in the reference's own rounding (no contraction: near coincidence the last
// bits of chi - 1 set K), clipped at the next double above 1.
__device__ __forceinline__ double chi_of(double rho, double z, double a, double za) {
    const double dr = __dadd_rn(rho, -a), dz = __dadd_rn(z, -za);
    const double num = __dadd_rn(__dmul_rn(dr, dr), __dmul_rn(dz, dz));
    const double den = __dmul_rn(__dmul_rn(2.0, rho), a);
    return fmax(__dadd_rn(1.0, __ddiv_rn(num, den)), kChiMin);
}

// Q_{n-1/2}(chi) for n = 0..M into q[0..M] (M = max(n_max, 1) <= MP) and
// dQ_{-1/2}/dchi (bem/toroidal.py:120-178): elliptic seeds Q_{-1/2} =
// sqrt(2/(chi+1)) K, Q_{1/2} = chi Q_{-1/2} - sqrt(2(chi+1)) E with K, E of
// the complementary parameter (chi-1)/(chi+1); upward three-term recurrence
// where M acosh(chi) <= 1, downward ratios (cumulative product from Q_{-1/2})
// elsewhere.
template <int MP>
__device__ __forceinline__ void toroidal(double chi, int M, double (&q)[MP + 1], double& dq0) {
    const double p = (chi - 1.0) / (chi + 1.0);
    double K, E;
    spt::ellip_ke(p, K, E);
    const double root = sqrt(2.0 / (chi + 1.0));
    const double q0 = root * K;
    dq0 = -root * E / (2.0 * (chi - 1.0));
    q[0] = q0;
    const double eta = acosh(chi);
    if ((double)M * eta <= 1.0) {
        double prev = q0, cur = chi * q0 - sqrt(2.0 * (chi + 1.0)) * E;
        q[1] = cur;
#pragma unroll
        for (int n = 1; n < MP; ++n) {
            if (n < M) {
                const double nxt = (2.0 * n * chi * cur - (n - 0.5) * prev) / (n + 0.5);
                q[n + 1] = nxt;
                prev = cur;
                cur = nxt;
            }
        }
    } else {
        const int pad = max(kPadMin, (int)ceil(kPadConst / eta));
        double r = 0.0;
#pragma unroll 1
        for (int n = M + pad; n > M; --n) r = (n - 0.5) / (2.0 * n * chi - (n + 0.5) * r);
#pragma unroll
        for (int n = MP; n >= 1; --n) {
            if (n <= M) {
                r = (n - 0.5) / (2.0 * n * chi - (n + 0.5) * r);
                q[n] = r;
            }
        }
#pragma unroll
        for (int n = 1; n <= MP; ++n)
            if (n <= M) q[n] *= q[n - 1];
    }
}

// dQ_{n-1/2}/dchi from the values (DLMF 14.10.5 at degree n - 1/2):
// (n - 1/2)(chi Q_n - Q_{n-1}) / ((chi - 1)(chi + 1)), n >= 1.
__device__ __forceinline__ double dq_of(int n, double chi, double qn, double qm1) {
    return (n - 0.5) * (chi * qn - qm1) / ((chi - 1.0) * (chi + 1.0));
}

__device__ __forceinline__ double smoothstep01(double t) {
    t = fmin(fmax(t, 0.0), 1.0);
    return t * t * (3.0 - 2.0 * t);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Closest point of (rho, z) on the profile (first strict minimum over the
// segments, bem/axisymmetric.py:341-389), the local mirror charge's weight
// (image_charge.py:333-342; skipped where the mirror plane is nearer,
// image_charge.py:538-585) and its position reflected through the tangent
// line (image_charge.py:364-378).  Whole warp; every lane returns the result.
__device__ inline void mirror_of(const SptImage& im, double rho, double z, int phantoms, double z0, double& r_img,
                          double& z_img, double& side, double& w) {
    const int lane = threadIdx.x & 31;
    const int ns = im.n_nodes - 1;
    double best = INFINITY;
    int arg = 0;
    double bt = 0.0;
    for (int j = lane; j < ns; j += 32) {
        const double p0r = im.seg[j], p0z = im.seg[ns + j], tr = im.seg[2 * ns + j], tz = im.seg[3 * ns + j];
        const double ab2 = tr * tr + tz * tz;
        const double t = fmin(fmax(((rho - p0r) * tr + (z - p0z) * tz) / ab2, 0.0), 1.0);
        const double dr = rho - (p0r + t * tr), dz = z - (p0z + t * tz);
        const double d2 = dr * dr + dz * dz;
        if (d2 < best) {
            best = d2;
            arg = j;
            bt = t;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oa = __shfl_xor_sync(0xffffffffu, arg, o);
        const double ot = __shfl_xor_sync(0xffffffffu, bt, o);
        if (ob < best || (ob == best && oa < arg)) {
            best = ob;
            arg = oa;
            bt = ot;
        }
    }
    const double p0r = im.seg[arg], p0z = im.seg[ns + arg], tr = im.seg[2 * ns + arg], tz = im.seg[3 * ns + arg];
    const double nr = im.seg[4 * ns + arg], nz = im.seg[5 * ns + arg];
    const double cr = p0r + bt * tr, cz = p0z + bt * tz;
    const double len = sqrt(tr * tr + tz * tz);
    const double ur = tr / len, uz = tz / len;
    const double dist = sqrt(best);
    w = im.d_hi > im.d_lo ? smoothstep01((im.d_hi - dist) / (im.d_hi - im.d_lo)) : 0.0;
    if (phantoms && !(fabs(z + z0) > dist)) w = 0.0;  // the plane z = -z0 is nearer than the profile
    const double dr = rho - cr, dz = z - cz;
    const double d_t = dr * ur + dz * uz, d_n = dr * nr + dz * nz;
    const double ri = cr + d_t * ur - d_n * nr;
    z_img = cz + d_t * uz - d_n * nz;
    side = ri < 0.0 ? -1.0 : 1.0;
    r_img = fabs(ri);
}


// Parameters of one image-force evaluation besides the tables.
struct ImgParams {
    int phantoms;         // mirror-doubled profile: a phantom source per particle (z -> -2 z0 - z, -q)
    int geometry;         // geometry level: blend with the flat plane image (bem/geometry.py:44-55, 326-344)
    int chunks;           // partial right-hand sides per profile node (source subsets summed in a fixed order)
    double z0, z_lo, z_hi;  // plane image at -z0; BEM below z_lo, plane above z_hi
    double k_coulomb, soft2, inv_eps0;
};

// The parameters of one call: geometry level when geom is given (z0, the
// blend heights z_handoff / 2 and z_handoff), phantoms for a mirror-doubled
// profile; 1 / eps0 = 4 pi k.  chunks is set by the caller.
__host__ __device__ inline ImgParams image_params(const SptImage& im, const SptGeometry* geom, double k_coulomb,
                                                  double plummer_radius) {
    ImgParams a{};
    a.phantoms = im.mirror_symmetric ? 1 : 0;
    a.geometry = geom ? 1 : 0;
    a.chunks = 1;
    a.z0 = geom ? geom->z0 : 0.0;
    a.z_lo = geom ? 0.5 * geom->z_handoff : 0.0;
    a.z_hi = geom ? geom->z_handoff : 1.0;
    a.k_coulomb = k_coulomb;
    a.soft2 = plummer_radius * plummer_radius;
    a.inv_eps0 = 4.0 * kPi * k_coulomb;
    return a;
}

// Scratch of one group of at most E particles (doubles).  Sources, S = E
// (2E with phantoms), then their S mirror charges: rho (floored), z, cos phi,
// sin phi, charge -- 5 x 2S; x, y and the blend weight of the particles --
// 3E; cos(m phi), sin(m phi) of each particle -- 2 (n_max+1) E; the
// right-hand sides rhs_c, rhs_s -- 2 (n_max+1) P; the work area of `chunks`
// partial right-hand sides, which then holds the solved sigma_c, sigma_s.
__host__ __device__ inline long long scratch_doubles(int E, int phantoms, int P, int n_max, int chunks) {
    const long long S = (long long)E * (phantoms ? 2 : 1);
    const long long MPN = (long long)(n_max + 1) * P;
    return 10 * S + 3LL * E + 2LL * (n_max + 1) * E + 2 * MPN + (long long)chunks * 2 * MPN;
}

// Image-charge force on the E particles of one group, computed by the whole
// CTA (every thread calls it; blockDim.x a multiple of 32).  load(i, x, y, z,
// q) gives particle i with q = 0 when it is inactive.  Writes fx[i], fy[i],
// fz[i] for i < E (0 for inactive particles).  `scratch` holds
// scratch_doubles(E, ...) doubles of shared memory; `flag` is one shared int.
//
//   A. sources: rho = hypot(x, y) floored, phi = atan2(y, x)
//      (image_charge.py:1003-1008); phantoms for a mirror-doubled profile
//   B. the local mirror charge of every source (warp per source)
//   C. rhs_m(p) = -sum_s q_s C_m Q_m(chi_ps) / sqrt(rho_p rho_s) x (cos | sin)
//      (m phi_s) over the sources and their mirror charges
//      (image_charge.py:1019-1035); thread per (node, source subset)
//   D. sigma_m = A_m^-1 rhs_m (image_charge.py:1037-1051): warp per row
//   E. per particle (warp per particle, lanes over the reconstruction nodes):
//      the field of the solved density (image_charge.py:1296-1347), the
//      direct field of every mirror charge (:1369-1395), times q / eps0;
//      geometry level: + the plane image for phantoms, blended with the
//      plane image by height.
// Phases B-D run only when some active particle needs the BEM force.
template <int MP, class Load>
__device__ void group_force(const SptImage& im, const ImgParams& a, int E, Load load, double* scratch, double* fx,
                            double* fy, double* fz, int* flag) {
    const int P = im.n_nodes, nm = im.n_max, M = max(nm, 1);
    const int MPN = (nm + 1) * P;
    const int nt = blockDim.x, nw = nt >> 5;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int S = a.phantoms ? 2 * E : E;
    double* srho = scratch;
    double* sz = srho + 2 * S;
    double* sc = sz + 2 * S;
    double* ss = sc + 2 * S;
    double* sq = ss + 2 * S;
    double* px = sq + 2 * S;
    double* py = px + E;
    double* wb = py + E;
    double* cs = wb + E;             // cos(m phi_i) [E][n_max+1]
    double* sn = cs + (nm + 1) * E;  // sin(m phi_i)
    double* rhs_c = sn + (nm + 1) * E;
    double* rhs_s = rhs_c + MPN;
    double* work = rhs_s + MPN;
    double* sig_c = work;
    double* sig_s = work + MPN;
    if (tid == 0) *flag = 0;
    __syncthreads();
    // A
    for (int i = tid; i < E; i += nt) {
        double x, y, z, q;
        load(i, x, y, z, q);
        double sp, cp;
        sincos(atan2(y, x), &sp, &cp);
        const double rs = fmax(hypot(x, y), im.rho_floor);
        px[i] = x;
        py[i] = y;
        srho[i] = rs;
        sz[i] = z;
        sc[i] = cp;
        ss[i] = sp;
        sq[i] = q;
        if (a.phantoms) {
            srho[E + i] = rs;
            sz[E + i] = -2.0 * a.z0 - z;
            sc[E + i] = cp;
            ss[E + i] = sp;
            sq[E + i] = -q;
        }
        double c1 = 1.0, s1 = 0.0;
        for (int m = 0; m <= nm; ++m) {
            cs[i * (nm + 1) + m] = c1;
            sn[i * (nm + 1) + m] = s1;
            const double cn = c1 * cp - s1 * sp;
            s1 = s1 * cp + c1 * sp;
            c1 = cn;
        }
        const double w = a.geometry ? smoothstep01((a.z_hi - z) / (a.z_hi - a.z_lo)) : 1.0;
        wb[i] = w;
        if (q != 0.0 && w > 0.0) atomicOr(flag, 1);
    }
    __syncthreads();
    if (*flag) {
        // B
        for (int i = warp; i < S; i += nw) {
            double ri, zi, side, w;
            mirror_of(im, srho[i], sz[i], a.phantoms, a.z0, ri, zi, side, w);
            if (lane == 0) {
                srho[S + i] = ri;
                sz[S + i] = zi;
                sc[S + i] = side > 0.0 ? sc[i] : -sc[i];  // across the axis: phi + pi
                ss[S + i] = side > 0.0 ? ss[i] : -ss[i];
                sq[S + i] = -sq[i] * w;
            }
        }
        for (int e = tid; e < a.chunks * 2 * MPN; e += nt) work[e] = 0.0;
        __syncthreads();
        // C: each (node, subset) pair is owned by one thread, so its partial sums need no atomics
        const int NC = a.chunks;
        for (int item = tid; item < P * NC; item += nt) {
            const int p = item % P, ch = item / P;
            const double rp = im.node[p], zp = im.node[P + p];
            double* pc = work + (size_t)ch * 2 * MPN + p;
            double q[MP + 1];
            for (int j = ch; j < 2 * S; j += NC) {
                const double qs = sq[j];
                if (qs == 0.0) continue;
                const double rj = srho[j];
                double dq0;
                toroidal<MP>(chi_of(rp, zp, rj, sz[j]), M, q, dq0);
                const double coef = qs / sqrt(rp * rj);
                const double c1 = sc[j], s1 = ss[j];
                double cm = 1.0, sm = 0.0;
#pragma unroll
                for (int m = 0; m <= MP; ++m) {
                    if (m <= nm) {
                        const double gm = coef * (m == 0 ? 1.0 / (4.0 * kPi * kPi) : 1.0 / (2.0 * kPi * kPi)) * q[m];
                        pc[m * P] += gm * cm;
                        pc[MPN + m * P] += gm * sm;
                        const double cn = cm * c1 - sm * s1;
                        sm = sm * c1 + cm * s1;
                        cm = cn;
                    }
                }
            }
        }
        __syncthreads();
        for (int e = tid; e < MPN; e += nt) {
            double c = 0.0, s = 0.0;
            for (int ch = 0; ch < NC; ++ch) {
                c += work[(size_t)ch * 2 * MPN + e];
                s += work[(size_t)ch * 2 * MPN + MPN + e];
            }
            rhs_c[e] = -c;
            rhs_s[e] = -s;
        }
        __syncthreads();
        // D
        for (int row = warp; row < MPN; row += nw) {
            const int m = row / P;
            const double* arow = im.a_inv + (size_t)row * P;
            double c = 0.0, s = 0.0;
            for (int k = lane; k < P; k += 32) {
                const double av = __ldg(arow + k);
                c += av * rhs_c[m * P + k];
                s += av * rhs_s[m * P + k];
            }
            c = warp_sum(c);
            s = warp_sum(s);
            if (lane == 0) {
                sig_c[row] = c;
                sig_s[row] = s;
            }
        }
        __syncthreads();
    }
    // E
    for (int i = warp; i < E; i += nw) {
        const double qi = sq[i];
        double f0 = 0.0, f1 = 0.0, f2 = 0.0;
        if (qi != 0.0) {
            const double xi = px[i], yi = py[i], zi = sz[i];
            double far0 = 0.0, far1 = 0.0, far2 = 0.0;
            if (a.geometry) {  // plane image at -z0 (forces.py:60-98) of every active particle of the group
                for (int j = lane; j < E; j += 32) {
                    const double qj = sq[j];
                    if (qj == 0.0) continue;
                    const double dx = xi - px[j], dy = yi - py[j], dz = zi - (-2.0 * a.z0 - sz[j]);
                    const double d2 = dx * dx + dy * dy + dz * dz + a.soft2;
                    const double c = a.k_coulomb * qi * (-qj) / (d2 * sqrt(d2));
                    far0 += c * dx;
                    far1 += c * dy;
                    far2 += c * dz;
                }
                far0 = warp_sum(far0);
                far1 = warp_sum(far1);
                far2 = warp_sum(far2);
            }
            const double w = wb[i];
            double n0 = 0.0, n1 = 0.0, n2 = 0.0;
            if (w > 0.0) {
                const double rq = srho[i], cq = sc[i], sqn = ss[i];
                const double* ci = cs + i * (nm + 1);
                const double* si = sn + i * (nm + 1);
                double er = 0.0, ez = 0.0, ep = 0.0;
                double q[MP + 1];
                const int NQ = im.n_quad;
                for (int k = lane; k < NQ; k += 32) {
                    const double rk = __ldg(im.quad + k), zk = __ldg(im.quad + NQ + k);
                    const double lk = __ldg(im.quad + 2 * NQ + k), tk = __ldg(im.quad + 3 * NQ + k);
                    const int jk = (int)__ldg(im.quad + 4 * NQ + k);
                    const double chi = chi_of(rq, zi, rk, zk);
                    double dq0;
                    toroidal<MP>(chi, M, q, dq0);
                    double SQ = 0.0, T = 0.0, SA = 0.0, c0 = 0.0;
#pragma unroll
                    for (int m = 0; m <= MP; ++m) {
                        if (m <= nm) {
                            const double a0 = sig_c[m * P + jk], a1 = sig_c[m * P + jk + 1];
                            const double b0 = sig_s[m * P + jk], b1 = sig_s[m * P + jk + 1];
                            const double dc = (a0 + tk * (a1 - a0)) * lk;
                            const double ds = (b0 + tk * (b1 - b0)) * lk;
                            const double cmv = dc * ci[m] + ds * si[m];
                            const double amv = dc * si[m] - ds * ci[m];
                            SQ += cmv * q[m];
                            SA += amv * (double)m * q[m];
                            if (m == 0) c0 = cmv;
                            else T += cmv * (m - 0.5) * (chi * q[m] - q[m - 1]);
                        }
                    }
                    const double SD = c0 * dq0 + T / ((chi - 1.0) * (chi + 1.0));
                    const double pref = sqrt(rk / rq) / (2.0 * kPi);
                    const double dzq = zi - zk;
                    const double dchi_drho = (rq * rq - rk * rk - dzq * dzq) / (2.0 * rk * rq * rq);
                    const double dchi_dz = dzq / (rk * rq);
                    er -= pref * (-SQ / (2.0 * rq) + SD * dchi_drho);
                    ez -= pref * SD * dchi_dz;
                    ep += pref * SA;
                }
                er = warp_sum(er);
                ez = warp_sum(ez);
                ep = warp_sum(ep) / rq;
                double e0 = er * cq - ep * sqn, e1 = er * sqn + ep * cq, e2 = ez;
                const double qx = rq * cq, qy = rq * sqn;
                double m0 = 0.0, m1 = 0.0, m2 = 0.0;
                for (int j = lane; j < S; j += 32) {
                    const double qm = sq[S + j];
                    if (qm == 0.0) continue;
                    const double rm = srho[S + j];
                    const double dx = qx - rm * sc[S + j], dy = qy - rm * ss[S + j], dz = zi - sz[S + j];
                    const double r = sqrt(dx * dx + dy * dy + dz * dz);
                    if (r > 0.0) {
                        const double c = qm / (4.0 * kPi * r * r * r);
                        m0 += c * dx;
                        m1 += c * dy;
                        m2 += c * dz;
                    }
                }
                e0 += warp_sum(m0);
                e1 += warp_sum(m1);
                e2 += warp_sum(m2);
                n0 = qi * e0 * a.inv_eps0;
                n1 = qi * e1 * a.inv_eps0;
                n2 = qi * e2 * a.inv_eps0;
                if (a.phantoms) {  // the phantoms' direct pull: the plane image (bem/geometry.py:404-415)
                    n0 += far0;
                    n1 += far1;
                    n2 += far2;
                }
            }
            if (a.geometry) {
                f0 = w * n0 + (1.0 - w) * far0;
                f1 = w * n1 + (1.0 - w) * far1;
                f2 = w * n2 + (1.0 - w) * far2;
            } else {
                f0 = n0;
                f1 = n1;
                f2 = n2;
            }
        }
        if (lane == 0) {
            fx[i] = f0;
            fy[i] = f1;
            fz[i] = f2;
        }
    }
    __syncthreads();
}

}  // namespace spt_img
