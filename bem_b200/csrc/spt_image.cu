// B200 (sm_100a) kernels of the BEM image-charge force: the induced charge
// of an axisymmetric grounded conductor, solved mode by mode in the
// azimuthal Fourier series of the free-space Green's function
// (bem/toroidal.py, bem/ring_modes.py, bem/image_charge.py).
//
//   spt_toroidal_q      Q_{m-1/2}(chi), dQ/dchi for m = 0..n_max
//   spt_image_assemble  per-mode single-layer collocation operators A[m]
//   spt_image_force     per call: local mirror charges, the joint per-group
//                       right-hand side of every mode, sigma = A^-1 rhs, the
//                       field of the solved density at each particle, the
//                       direct mirror-charge field, and (geometry level) the
//                       blend with the flat plane image above z_handoff / 2.
//
// One CTA owns one group at a time (grid-stride over groups): the group's
// sources, their mirror charges, the right-hand sides and the solved mode
// densities stay in shared memory between the phases of the call.  The
// toroidal harmonics of a (point, ring) pair are built in registers for all
// modes at once: a template bound MP on the mode count keeps the per-mode
// arrays in registers (instantiated for MP = 16, 32, 64).
#include <cuda_runtime.h>
#include <stdint.h>

#include "spt_abi.hpp"
#include "spt_b200.h"
#include "spt_image.cuh"

namespace spt_img {

constexpr int kThreads = 256;

// ---------------------------------------------------------------------------
// spt_toroidal_q

template <int MP>
__global__ void __launch_bounds__(kThreads) toroidal_kernel(const double* chi_in, long long n, int n_max, double* q_out,
                                                            double* dq_out) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double chi = fmax(chi_in[i], kChiMin);
    const int M = max(n_max, 1);
    double q[MP + 1];
    double dq0;
    toroidal<MP>(chi, M, q, dq0);
#pragma unroll
    for (int m = 0; m <= MP; ++m) {
        if (m <= n_max) {
            q_out[m * n + i] = q[m];
            dq_out[m * n + i] = m == 0 ? dq0 : dq_of(m, chi, q[m], q[m - 1]);
        }
    }
}

// ---------------------------------------------------------------------------
// spt_image_assemble: thread per (collocation node i, segment j); the hat
// halves of nodes j and j+1 are added to A[m][i][j], A[m][i][j+1] (each
// entry receives exactly two additions, from segments j-1 and j, so the sum
// is independent of their order).  Bisection as bem/image_charge.py:379-411:
// refine while the sub-segment's length exceeds refine_ratio times the
// distance from the node to its midpoint, up to max_depth levels; Gauss-4
// on each leaf with the mode kernel Phi_m = sqrt(a/rho) Q_{m-1/2} / (2 pi).

template <int MP>
__global__ void __launch_bounds__(128) assemble_modes_kernel(const double* pr, const double* pz, int n, int n_max,
                                                             double rho_floor, double refine_ratio, int max_depth,
                                                             const double* g4x, const double* g4w, double* A) {
    const long long pair = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long n_pairs = (long long)n * (n - 1);
    if (pair >= n_pairs) return;
    const int i = (int)(pair / (n - 1));
    const int j = (int)(pair - (long long)i * (n - 1));
    const double rf = fmax(pr[i], rho_floor), zf = pz[i];
    const int M = max(n_max, 1);
    double st0[48], st1[48];
    int sd[48];
    int top = 1;
    st0[0] = 0.0;
    st1[0] = 1.0;
    sd[0] = 0;
    const double ar = pr[j], az = pz[j], br = pr[j + 1], bz = pz[j + 1];
    double acc0[MP + 1], acc1[MP + 1], q[MP + 1];
#pragma unroll
    for (int m = 0; m <= MP; ++m) acc0[m] = acc1[m] = 0.0;
    while (top > 0) {
        --top;
        const double t0 = st0[top], t1 = st1[top];
        const int depth = sd[top];
        const double p0r = ar + t0 * (br - ar), p0z = az + t0 * (bz - az);
        const double p1r = ar + t1 * (br - ar), p1z = az + t1 * (bz - az);
        const double mr = 0.5 * (p0r + p1r), mz = 0.5 * (p0z + p1z);
        const double len = sqrt((p1r - p0r) * (p1r - p0r) + (p1z - p0z) * (p1z - p0z));
        const double dist = sqrt((rf - mr) * (rf - mr) + (zf - mz) * (zf - mz));
        if (depth < max_depth && len > refine_ratio * dist && top + 2 <= 48) {
            const double tm = 0.5 * (t0 + t1);
            st0[top] = tm; st1[top] = t1; sd[top] = depth + 1; ++top;
            st0[top] = t0; st1[top] = tm; sd[top] = depth + 1; ++top;
            continue;
        }
#pragma unroll 1
        for (int k = 0; k < 4; ++k) {
            const double u = 0.5 * (g4x[k] + 1.0);
            const double rs = p0r + u * (p1r - p0r), zs = p0z + u * (p1z - p0z);
            const double tt = t0 + u * (t1 - t0);
            const double w = sqrt(rs / rf) / (2.0 * kPi) * (len * 0.5 * g4w[k]);
            double dq0;
            toroidal<MP>(chi_of(rf, zf, rs, zs), M, q, dq0);
#pragma unroll
            for (int m = 0; m <= MP; ++m) {
                if (m <= n_max) {
                    acc0[m] += (1.0 - tt) * w * q[m];
                    acc1[m] += tt * w * q[m];
                }
            }
        }
    }
    const size_t nn = (size_t)n * n;
#pragma unroll
    for (int m = 0; m <= MP; ++m) {
        if (m <= n_max) {
            atomicAdd(&A[m * nn + (size_t)i * n + j], acc0[m]);
            atomicAdd(&A[m * nn + (size_t)i * n + j + 1], acc1[m]);
        }
    }
}

// ---------------------------------------------------------------------------
// spt_image_force: one CTA per group at a time (grid-stride over groups)

struct ForceArgs {
    const double* x;
    const double* y;
    const double* z;
    const double* charge;
    const uint8_t* active;
    const int64_t* group_offset;
    int n_groups;
    int max_e;
    SptImage img;
    ImgParams prm;
    double* fx;
    double* fy;
    double* fz;
};

template <int MP>
__global__ void __launch_bounds__(kThreads, 1) image_force_kernel(const __grid_constant__ ForceArgs a) {
    extern __shared__ __align__(16) double smem[];
    __shared__ int s_flag;
    for (int g = blockIdx.x; g < a.n_groups; g += gridDim.x) {
        const long long off = a.group_offset[g];
        const int E = (int)(a.group_offset[g + 1] - off);
        auto load = [&](int i, double& x, double& y, double& z, double& q) {
            x = a.x[off + i];
            y = a.y[off + i];
            z = a.z[off + i];
            q = a.active[off + i] ? a.charge[off + i] : 0.0;
        };
        group_force<MP>(a.img, a.prm, E, load, smem, a.fx + off, a.fy + off, a.fz + off, &s_flag);
    }
}

}  // namespace spt_img

// ===========================================================================
// C ABI

namespace {
using spt_abi::cuda_check;
using spt_abi::fail;

int mode_bound(int n_max) { return n_max <= 16 ? 16 : (n_max <= 32 ? 32 : 64); }

int sm_count() {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return 148;
    return n > 0 ? n : 148;
}

template <int MP>
int launch_force(const spt_img::ForceArgs& a, size_t bytes, cudaStream_t st) {
    auto k = spt_img::image_force_kernel<MP>;
    int rc = cuda_check(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes),
                        "cudaFuncSetAttribute(image_force_kernel)");
    if (rc) return rc;
    const int grid = a.n_groups < sm_count() ? a.n_groups : sm_count();
    k<<<grid, spt_img::kThreads, bytes, st>>>(a);
    return cuda_check(cudaGetLastError(), "image_force_kernel launch");
}
}  // namespace

extern "C" {

int spt_toroidal_q(const double* chi, int64_t n, int32_t n_max, double* q, double* dq, void* stream) {
    if (n < 0) return fail(SPT_ERR_ARG, "n must be >= 0");
    if (n_max < 0 || n_max > SPT_IMAGE_MAX_MODES)
        return fail(SPT_ERR_CAPACITY, "n_max %d outside [0, %d]", n_max, SPT_IMAGE_MAX_MODES);
    if (n == 0) return SPT_OK;
    if (!chi || !q || !dq) return fail(SPT_ERR_ARG, "null argument");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const unsigned blocks = (unsigned)((n + spt_img::kThreads - 1) / spt_img::kThreads);
    switch (mode_bound(n_max)) {
        case 16: spt_img::toroidal_kernel<16><<<blocks, spt_img::kThreads, 0, st>>>(chi, n, n_max, q, dq); break;
        case 32: spt_img::toroidal_kernel<32><<<blocks, spt_img::kThreads, 0, st>>>(chi, n, n_max, q, dq); break;
        default: spt_img::toroidal_kernel<64><<<blocks, spt_img::kThreads, 0, st>>>(chi, n, n_max, q, dq); break;
    }
    return cuda_check(cudaGetLastError(), "toroidal_kernel launch");
}

int spt_image_assemble(const double* profile_rho, const double* profile_z, int32_t n_nodes, int32_t n_max,
                       double rho_floor, double refine_ratio, int32_t max_depth, const double* gauss4_x,
                       const double* gauss4_w, double* A, void* stream) {
    if (n_nodes < 2) return fail(SPT_ERR_ARG, "profile needs at least 2 nodes");
    if (n_max < 0 || n_max > SPT_IMAGE_MAX_MODES)
        return fail(SPT_ERR_CAPACITY, "n_max %d outside [0, %d]", n_max, SPT_IMAGE_MAX_MODES);
    if (!profile_rho || !profile_z || !A || !gauss4_x || !gauss4_w) return fail(SPT_ERR_ARG, "null argument");
    if (max_depth < 0 || max_depth > 40) return fail(SPT_ERR_CAPACITY, "max_depth must be in [0, 40]");
    if (!(rho_floor > 0.0)) return fail(SPT_ERR_ARG, "rho_floor must be > 0");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int rc = cuda_check(cudaMemsetAsync(A, 0, sizeof(double) * (size_t)(n_max + 1) * n_nodes * n_nodes, st),
                        "cudaMemsetAsync");
    if (rc) return rc;
    const long long pairs = (long long)n_nodes * (n_nodes - 1);
    const unsigned blocks = (unsigned)((pairs + 127) / 128);
#define SPT_ASSEMBLE(MP)                                                                                         \
    spt_img::assemble_modes_kernel<MP><<<blocks, 128, 0, st>>>(profile_rho, profile_z, n_nodes, n_max, rho_floor, \
                                                               refine_ratio, max_depth, gauss4_x, gauss4_w, A)
    switch (mode_bound(n_max)) {
        case 16: SPT_ASSEMBLE(16); break;
        case 32: SPT_ASSEMBLE(32); break;
        default: SPT_ASSEMBLE(64); break;
    }
#undef SPT_ASSEMBLE
    return cuda_check(cudaGetLastError(), "assemble_modes_kernel launch");
}

int spt_image_force(const double* x, const double* y, const double* z, const double* charge, const uint8_t* active,
                    const int64_t* group_offset, int32_t n_groups, int32_t max_group_size, const SptImage* image,
                    const SptGeometry* geom, double coulomb_constant, double plummer_radius, double* fx, double* fy,
                    double* fz, void* stream) {
    if (!image) return fail(SPT_ERR_ARG, "image tables required");
    if (n_groups < 0) return fail(SPT_ERR_ARG, "n_groups must be >= 0");
    if (n_groups == 0) return SPT_OK;
    if (!x || !y || !z || !charge || !active || !group_offset || !fx || !fy || !fz)
        return fail(SPT_ERR_ARG, "null argument");
    const SptImage& im = *image;
    if (im.n_nodes < 2 || !im.node || !im.seg || !im.quad || !im.a_inv) return fail(SPT_ERR_ARG, "incomplete image tables");
    if (im.n_max < 0 || im.n_max > SPT_IMAGE_MAX_MODES)
        return fail(SPT_ERR_CAPACITY, "n_max %d outside [0, %d]", im.n_max, SPT_IMAGE_MAX_MODES);
    if (im.n_quad <= 0 || im.n_quad % 4) return fail(SPT_ERR_ARG, "n_quad must be a positive multiple of 4");
    if (!(im.rho_floor > 0.0)) return fail(SPT_ERR_ARG, "rho_floor must be > 0");
    if (geom) {
        if (geom->kind != SPT_GEOM_TIP_BEM && geom->kind != SPT_GEOM_WELL_BEM)
            return fail(SPT_ERR_ARG, "the BEM image force belongs to SPT_GEOM_TIP_BEM / SPT_GEOM_WELL_BEM");
        if (!geom->has_image) return fail(SPT_ERR_ARG, "geometry has no image force (has_image = 0)");
        if (!(geom->z_handoff > 0.0)) return fail(SPT_ERR_ARG, "z_handoff must be > 0");
    } else if (im.mirror_symmetric) {
        return fail(SPT_ERR_ARG, "a mirror-doubled profile needs the geometry (its plane z0)");
    }
    const int max_e = im.mirror_symmetric ? 256 : 512;
    if (max_group_size <= 0 || max_group_size > max_e)
        return fail(SPT_ERR_CAPACITY, "max_group_size %d outside [1, %d]", max_group_size, max_e);
    spt_img::ForceArgs a{};
    a.x = x; a.y = y; a.z = z; a.charge = charge; a.active = active; a.group_offset = group_offset;
    a.n_groups = n_groups;
    a.max_e = max_group_size;
    a.img = im;
    a.prm = spt_img::image_params(im, geom, coulomb_constant, plummer_radius);
    a.fx = fx; a.fy = fy; a.fz = fz;
    const size_t limit = 227 * 1024;
    int chunks = spt_img::kThreads / im.n_nodes;
    chunks = chunks < 1 ? 1 : (chunks > 8 ? 8 : chunks);
    size_t bytes = 0;
    for (; chunks >= 1; --chunks) {
        bytes = 8 * (size_t)spt_img::scratch_doubles(max_group_size, a.prm.phantoms, im.n_nodes, im.n_max, chunks);
        if (bytes <= limit) break;
    }
    if (chunks < 1)
        return fail(SPT_ERR_CAPACITY, "image tables too large for one CTA: %lld bytes of shared memory (limit %lld)",
                    (long long)bytes, (long long)limit);
    a.prm.chunks = chunks;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    switch (mode_bound(im.n_max)) {
        case 16: return launch_force<16>(a, bytes, st);
        case 32: return launch_force<32>(a, bytes, st);
        default: return launch_force<64>(a, bytes, st);
    }
}

}  // extern "C"
