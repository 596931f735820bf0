// B200 (sm_100a) kernels for the specific_particle_tracer hot path: the C ABI.
//
// One persistent kernel (trace_kernel, spt_device.cuh; instantiated per
// geometry kind in spt_trace_<kind>.cu) advances emission groups through the
// per-group adaptive Dormand-Prince 5(4) integrator of batched_rk45.py.  A
// CTA owns one group at a time (groups come from a device work queue); the
// group's state, its seven stage slopes and the stage positions live in
// shared memory, so a step attempt never leaves the SM.  Every stage
// evaluates, on the stage positions:
//   * the external field: analytic (fields.py) or the BEM ring-charge sum
//     blended with the flat fallback (bem/axisymmetric.py, bem/geometry.py),
//   * Plummer-softened Coulomb pair forces within the group (forces.py:16-57),
//   * the image-charge pair forces (forces.py:60-191).
//
// This file holds the argument checks and launches of every entry point of
// include/spt_b200.h, and the small kernels only they use (BEM field at
// arbitrary points, compaction, ring field, elliptic integrals, BEM
// collocation matrix).
#include <mutex>
#include <stdarg.h>

#include "spt_abi.hpp"
#include "spt_device.cuh"

namespace spt {

SPT_DECLARE_KIND(SPT_GEOM_FLAT)
SPT_DECLARE_KIND(SPT_GEOM_TIP)
SPT_DECLARE_KIND(SPT_GEOM_TIP_BEM)
SPT_DECLARE_KIND(SPT_GEOM_WELL_BEM)
SPT_DECLARE_KIND(SPT_GEOM_POST_BEM)

// BEM perturbation field at arbitrary points (spt_bem_field): kRound*8 points per CTA
constexpr int kFieldChunk = 64;
template <int FORM, int FAR>
__global__ void __launch_bounds__(kMaxThreads, 1)
bem_field_kernel(const double* x, const double* y, const double* z, long long n, const __grid_constant__ SptBem bem,
                 double* ex, double* ey, double* ez, unsigned long long* counters) {
    extern __shared__ __align__(16) double smem[];
    __shared__ int s_flag;
    __shared__ unsigned long long s_cnt[SPT_N_COUNTERS];
    __shared__ SptGeometry s_geo;
    if (threadIdx.x == 0) s_geo = SptGeometry{};
    __syncthreads();
    Ctx c(s_geo, bem);
    bind(c, smem, kFieldChunk, FAR, nullptr, s_cnt);
    init_barriers(c);
    const long long p0 = (long long)blockIdx.x * kFieldChunk;
    const int np_ = (int)min((long long)kFieldChunk, n - p0);
    for (int k = threadIdx.x; k < np_; k += c.nt) {
        c.bpt[8 * k + 0] = x[p0 + k];
        c.bpt[8 * k + 1] = y[p0 + k];
        c.bpt[8 * k + 2] = z[p0 + k];
    }
    if (threadIdx.x == 0) s_flag = 0;
    __syncthreads();
    bem_points<FORM, FAR>(c, np_, false, &s_flag);
    for (int k = threadIdx.x; k < np_; k += c.nt) {
        ex[p0 + k] = c.bpt[8 * k + 5];
        ey[p0 + k] = c.bpt[8 * k + 6];
        ez[p0 + k] = c.bpt[8 * k + 7];
    }
    __syncthreads();
    flush_counters(c, counters);
}

// learned-form field at arbitrary points (spt_surrogate_field): 128 points
// (one MLP tile) per CTA, through the stage kernel's surrogate_points
constexpr int kSurChunk = 128;
template <int FAR>
__global__ void __launch_bounds__(kMaxThreads, 1)
surrogate_field_kernel(const double* x, const double* y, const double* z, long long n,
                       const __grid_constant__ SptBem bem, const __grid_constant__ SptTraceParams prm, double* ex,
                       double* ey, double* ez, unsigned long long* counters) {
    extern __shared__ __align__(16) double smem[];
    __shared__ int s_flag;
    __shared__ uint32_t s_tmem;
    __shared__ unsigned long long s_cnt[SPT_N_COUNTERS];
    __shared__ SptGeometry s_geo;
    if (threadIdx.x == 0) s_geo = SptGeometry{};
    __syncthreads();
    Ctx c(s_geo, bem);
    bind(c, smem, kSurChunk, FAR, nullptr, s_cnt, true);
    bind_surrogate(c, prm, &s_tmem);
    init_barriers(c);
    c.key = 0x2545F491u;
    const long long p0 = (long long)blockIdx.x * kSurChunk;
    const int np_ = (int)min((long long)kSurChunk, n - p0);
    for (int k = threadIdx.x; k < np_; k += c.nt) {
        c.bpt[8 * k + 0] = x[p0 + k];
        c.bpt[8 * k + 1] = y[p0 + k];
        c.bpt[8 * k + 2] = z[p0 + k];
        c.list[k] = (int)(p0 + k);
    }
    if (threadIdx.x == 0) s_flag = 0;
    __syncthreads();
    surrogate_points<FAR>(c, np_, &s_flag);
    // records were reordered (exact ones first): c.list holds each one's point index
    for (int k = threadIdx.x; k < np_; k += c.nt) {
        const long long i = c.list[k];
        ex[i] = c.bpt[8 * k + 5];
        ey[i] = c.bpt[8 * k + 6];
        ez[i] = c.bpt[8 * k + 7];
    }
    __syncthreads();
    flush_counters(c, counters);
    release_surrogate(c);
}

// order-preserving compaction of the running groups (spt_compact_groups):
// one CTA of kCompactThreads walks the list in chunks; each chunk is read,
// scanned (warp ballots + per-warp counts) and written after a barrier, so
// out may alias order (a chunk's writes land at or before its reads).
constexpr int kCompactThreads = 1024;
__global__ void __launch_bounds__(kCompactThreads, 1)
compact_kernel(const int* order, int n, const int* status, int* out, int* n_active) {
    __shared__ int s_w[kCompactThreads / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    int run = 0;
    for (int base = 0; base < n; base += kCompactThreads) {
        const int j = base + tid;
        int g = 0;
        bool keep = false;
        if (j < n) {
            g = order ? order[j] : j;
            keep = status[g] < SPT_GROUP_DONE;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, keep);
        if (lane == 0) s_w[warp] = __popc(bal);
        __syncthreads();
        int pre = 0, tot = 0;
        for (int w = 0; w < kCompactThreads / 32; ++w) {
            if (w < warp) pre += s_w[w];
            tot += s_w[w];
        }
        if (keep) out[run + pre + __popc(bal & ((1u << lane) - 1u))] = g;
        run += tot;
        __syncthreads();
    }
    if (tid == 0) *n_active = run;
}

__global__ void ring_kernel(const double* rho, const double* z, const double* a, long long n, int form, double* er,
                            double* ez) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        if (form == SPT_FORM_FP64) {
            ring_field(rho[i], z[i], a[i], er[i], ez[i]);
        } else {
            float r, zz;
            ring_field_f((float)rho[i], (float)z[i], (float)a[i], r, zz);
            er[i] = r;
            ez[i] = zz;
        }
    }
}

__global__ void ellip_kernel(const double* p, long long n, int form, double* K, double* E) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        if (form == SPT_FORM_FP64) {
            ellip_ke(p[i], K[i], E[i]);
        } else {
            float k, e;
            ellip_ke_f((float)p[i], k, e);
            K[i] = k;
            E[i] = e;
        }
    }
}


// ---------------------------------------------------------------------------
// BEM collocation matrix (AxisymmetricBEMSolution.solve, bem/axisymmetric.py:411-443
// with the adaptive segment rule of :275-302): A[i][j] is the potential at
// profile node i of the P1 hat density of node j.  One thread per (node i,
// segment j) pair walks the bisection tree depth first with an explicit
// stack (refine while length > refine_ratio * distance to the sub-segment
// midpoint, up to max_depth), Gauss-4 on each leaf, and adds the two hat
// halves into A[i][j] and A[i][j+1] with atomics (the two segments adjacent
// to node j both contribute to column j).
__device__ __forceinline__ double ring_potential(double rho, double z, double a) {
    const double D = (rho + a) * (rho + a) + z * z;
    const double p = ((rho - a) * (rho - a) + z * z) / D;
    double K, E;
    ellip_ke(p, K, E);
    return K / (2.0 * kPi * kPi * sqrt(D));
}

__global__ void assemble_kernel(const double* pr, const double* pz, int n, double refine_ratio, int max_depth,
                                const double* g4x, const double* g4w, double* A) {
    const long long pair = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long n_pairs = (long long)n * (n - 1);
    if (pair >= n_pairs) return;
    const int i = (int)(pair / (n - 1));
    const int j = (int)(pair - (long long)i * (n - 1));
    const double rf = pr[i], zf = pz[i];
    // stack entries: t0, t1 (parameters along segment j), depth
    double st0[48], st1[48];
    int sd[48];
    int top = 0;
    st0[0] = 0.0; st1[0] = 1.0; sd[0] = 0; top = 1;
    const double ar = pr[j], az = pz[j], br = pr[j + 1], bz = pz[j + 1];
    double acc0 = 0.0, acc1 = 0.0;  // hat of node j (1 -> 0) and of node j+1 (0 -> 1)
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
            st0[top] = tm; st1[top] = t1; sd[top] = depth + 1; ++top;   // right half, processed second
            st0[top] = t0; st1[top] = tm; sd[top] = depth + 1; ++top;   // left half first
            continue;
        }
        for (int k = 0; k < 4; ++k) {
            const double u = 0.5 * (g4x[k] + 1.0);
            const double rs = p0r + u * (p1r - p0r), zs = p0z + u * (p1z - p0z);
            const double tt = t0 + u * (t1 - t0);          // position along the full segment
            const double base = 2.0 * kPi * rs * ring_potential(rf, zf - zs, rs) * (len * 0.5 * g4w[k]);
            acc0 += (1.0 - tt) * base;
            acc1 += tt * base;
        }
    }
    atomicAdd(&A[(size_t)i * n + j], acc0);
    atomicAdd(&A[(size_t)i * n + j + 1], acc1);
}

}  // namespace spt

// ===========================================================================
// C ABI

namespace spt_abi {
thread_local char g_err[512];

int fail(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

int cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) return fail(SPT_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    return SPT_OK;
}
}  // namespace spt_abi

namespace {
using spt_abi::cuda_check;
using spt_abi::fail;
using spt_abi::g_err;

int check_bem(const SptBem* b) {
    if (!b || !b->seg || !b->node) return fail(SPT_ERR_ARG, "BEM tables required for this geometry");
    if (b->n_seg <= 0 || b->nodes_per_seg <= 0 || b->nodes_per_seg % 4 || b->nodes_per_seg > 256)
        return fail(SPT_ERR_ARG, "nodes_per_seg must be a positive multiple of 4, at most 256");
    if ((reinterpret_cast<uintptr_t>(b->node) & 15) || (b->node_stride & 1))
        return fail(SPT_ERR_ARG, "node table must be 16-byte aligned with an even row stride");
    if (b->node_stride < (int64_t)b->n_seg * b->nodes_per_seg || b->seg_stride < b->n_seg)
        return fail(SPT_ERR_ARG, "table strides too small");
    if (b->far_rule == SPT_FAR_ADAPTIVE) {
        if (!b->coarse || b->coarse_stride < 6 * (int64_t)b->n_seg)
            return fail(SPT_ERR_ARG, "adaptive far rule: coarse node table missing or too small");
        if (!(b->ratio4 >= 1.0) || !(b->ratio2 >= b->ratio4))
            return fail(SPT_ERR_ARG, "adaptive far rule: need 1 <= ratio4 <= ratio2");
        const int64_t n_run = (b->n_seg + SPT_BLOCK_SEGS - 1) / SPT_BLOCK_SEGS;
        if (b->blk && b->blk_stride < n_run) return fail(SPT_ERR_ARG, "run bounds table too small");
        if (b->blk && b->run_nodes && b->ratio_run > 0.0) {
            // a run at least one arclength away holds no near segment
            if (!(b->ratio_run >= 1.0)) return fail(SPT_ERR_ARG, "adaptive far rule: ratio_run must be >= 1 (or <= 0: off)");
            if (b->run_stride < SPT_RUN_NODES * n_run) return fail(SPT_ERR_ARG, "run-node table too small");
        }
    } else if (b->far_rule != SPT_FAR_REFERENCE) {
        return fail(SPT_ERR_ARG, "unknown far rule %d", b->far_rule);
    }
    if (b->blk && b->blk_stride < (b->n_seg + SPT_BLOCK_SEGS - 1) / SPT_BLOCK_SEGS)
        return fail(SPT_ERR_ARG, "run bounds table too small");
    if (b->far_rule == SPT_FAR_ADAPTIVE && b->clusters && b->cluster_kappa > 0.0) {
        const int n_run = (b->n_seg + SPT_BLOCK_SEGS - 1) / SPT_BLOCK_SEGS;
        int levels = 1;
        for (int size = 1; (n_run + size - 1) / size > 1; size *= 2) ++levels;
        if (!b->blk) return fail(SPT_ERR_ARG, "cluster expansions need the run bounds table");
        if (n_run > SPT_MAX_CLUSTER_RUNS)
            return fail(SPT_ERR_CAPACITY, "cluster expansions: %d runs exceed %d", n_run, SPT_MAX_CLUSTER_RUNS);
        if (b->cluster_levels != levels)
            return fail(SPT_ERR_ARG, "cluster table has %d levels, %d runs need %d", b->cluster_levels, n_run, levels);
        if (b->cluster_terms < 1 || b->cluster_terms > 64) return fail(SPT_ERR_ARG, "cluster_terms must be in [1, 64]");
        if (!(b->cluster_kappa > 1.0)) return fail(SPT_ERR_ARG, "cluster_kappa must exceed 1 (or be <= 0: off)");
    }
    return SPT_OK;
}

bool is_bem(int kind) { return kind == SPT_GEOM_TIP_BEM || kind == SPT_GEOM_WELL_BEM || kind == SPT_GEOM_POST_BEM; }

// The BEM image-charge force of a tip or well geometry built with z0
// (has_image): its tables must be given, with at most SPT_TRACE_IMAGE_MODES
// modes (the per-mode arrays of the stage evaluation live in registers).
int check_image(const SptGeometry* g, const SptBem* b, int max_group_size) {
    if (!(g->kind == SPT_GEOM_TIP_BEM || g->kind == SPT_GEOM_WELL_BEM) || !g->has_image) return SPT_OK;
    const SptImage& im = b->image;
    if (im.n_nodes < 2 || !im.node || !im.seg || !im.quad || !im.a_inv)
        return fail(SPT_ERR_ARG, "a BEM tip or well with an image plane (has_image) needs the image-charge tables");
    if (im.n_max < 0 || im.n_max > SPT_TRACE_IMAGE_MODES)
        return fail(SPT_ERR_CAPACITY, "image-charge n_max %d outside [0, %d] in the trace", im.n_max,
                    SPT_TRACE_IMAGE_MODES);
    if (im.n_quad <= 0 || im.n_quad % 4 || !(im.rho_floor > 0.0)) return fail(SPT_ERR_ARG, "bad image-charge tables");
    if (!(g->z_handoff > 0.0)) return fail(SPT_ERR_ARG, "z_handoff must be > 0");
    const int lim = im.mirror_symmetric ? 256 : 512;
    if (max_group_size > lim)
        return fail(SPT_ERR_CAPACITY, "groups with the BEM image force hold at most %d particles", lim);
    return SPT_OK;
}

int check_surrogate_params(const SptTraceParams* p) {
    if (!p->sur_w || !p->sur_w16 || !p->sur_s_start || !p->sur_log_scale)
        return fail(SPT_ERR_ARG, "learned form: surrogate parameters missing");
    if (reinterpret_cast<uintptr_t>(p->sur_w16) & 15) return fail(SPT_ERR_ARG, "sur_w16 must be 16-byte aligned");
    if (!(p->sur_d_min > 0.0) || !(p->sur_d_max > p->sur_d_min) || !(p->sur_s_end > 0.0))
        return fail(SPT_ERR_ARG, "learned form: bad feature ranges");
    return SPT_OK;
}

// (groups are at most 1024 particles in every form: surrogate_points
// reorders a stage's points through the 64 KiB MLP operand tiles, 8 doubles each)
int check_surrogate(const SptTraceParams* p, const SptGeometry* g) {
    if (!is_bem(g->kind)) return fail(SPT_ERR_ARG, "the learned form needs a BEM geometry");
    return check_surrogate_params(p);
}

template <typename K>
int set_smem(K kernel, size_t bytes) {
    return cuda_check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes),
                      "cudaFuncSetAttribute");
}

int far_rule_of(const SptGeometry* g, const SptBem* b) { return is_bem(g->kind) && b ? b->far_rule : SPT_FAR_REFERENCE; }

// CTA width of a trace launch: SptTraceParams.cta_threads when it is 32, 64,
// 128 or 256, else by group size (narrow CTAs for small groups: more groups
// per SM, fewer warps behind each barrier).  The reference far rule streams
// 96 KiB node tiles per CTA, so it keeps 256 threads; the learned form needs
// at least 4 warps (one per 32 TMEM lanes of its 128-row accumulator).
int trace_threads(const SptState* s, const SptTraceParams* p, int far) {
    const int want = p->cta_threads;
    int t;
    if (want == 32 || want == 64 || want == 128 || want == 256)
        t = want;
    else if (far == SPT_FAR_REFERENCE || s->max_group_size > 64)
        t = 256;
    else
        t = s->max_group_size > 16 ? 128 : 64;
    if (p->form == SPT_FORM_SURROGATE && t < 128) t = 128;
    return t;
}

// The warp team (one group per warp) serves BEM geometries without the BEM
// image-charge force, the float64 form with the adaptive far rule, and
// groups of at most 32 particles; SptTraceParams.team may ask for it or
// keep the CTA team.
bool warp_team_offered(const SptState* s, const SptTraceParams* p, const SptGeometry* g, const SptBem* b, int far) {
    return is_bem(g->kind) && b && far == SPT_FAR_ADAPTIVE && p->form == SPT_FORM_FP64 && s->max_group_size <= 32 &&
           spt::image_scratch(*g, *b, s->max_group_size, spt::kMaxThreads) == 0;
}

// CTA width of a warp-team launch: SptTraceParams.cta_threads when it is 32,
// 64, 128 or 256, else 256 (every width keeps the same warps per SM; wider
// CTAs take fewer CTA slots).
int warp_team_threads(const SptTraceParams* p) {
    const int want = p->cta_threads;
    return (want == 32 || want == 64 || want == 128 || want == 256) ? want : 256;
}

constexpr int kNotLaunched = -2;  // run_warp_team: the CTA team takes the launch

int64_t warp_team_slot_bytes(int threads) { return (int64_t)(threads / 32) * spt::kWarpSlotDoubles * 8; }

int dispatch_kind(int kind, const spt::TraceLaunch& t, int form, int far, bool launch, int* grid, size_t* smem,
                  int* per_sm) {
    switch (kind) {
        case SPT_GEOM_FLAT: return spt::trace_dispatch<SPT_GEOM_FLAT>(t, form, far, launch, grid, smem, per_sm);
        case SPT_GEOM_TIP: return spt::trace_dispatch<SPT_GEOM_TIP>(t, form, far, launch, grid, smem, per_sm);
        case SPT_GEOM_TIP_BEM: return spt::trace_dispatch<SPT_GEOM_TIP_BEM>(t, form, far, launch, grid, smem, per_sm);
        case SPT_GEOM_WELL_BEM: return spt::trace_dispatch<SPT_GEOM_WELL_BEM>(t, form, far, launch, grid, smem, per_sm);
        case SPT_GEOM_POST_BEM: return spt::trace_dispatch<SPT_GEOM_POST_BEM>(t, form, far, launch, grid, smem, per_sm);
        default: return -1;
    }
}

// One trace launch with scratch at `scratch`: the work-queue counter in its
// first 256 bytes, then (groups above 256 particles) per-CTA slope buffers,
// scratch_bytes in all; the persistent grid is capped by the buffers it holds
// and by SptTraceParams.max_ctas.
// Grid of a warp-team launch on this device (the whole GPU, or the groups,
// or SptTraceParams.max_ctas); without a device, SMs x two CTAs.
int warp_team_grid(const SptState* s, const SptTraceParams* p, const SptGeometry* g, const SptBem* b, int far) {
    spt::TraceLaunch t{};
    t.s = s;
    t.p = p;
    t.g = g;
    t.bem = *b;
    t.threads = warp_team_threads(p);
    t.warp_team = true;
    t.max_slots = p->max_ctas > 0 ? p->max_ctas : 0;
    int grid = 0, per_sm = 0;
    size_t smem = 0;
    if (dispatch_kind(g->kind, t, p->form, far, false, &grid, &smem, &per_sm) == 0 && grid > 0) return grid;
    cudaGetLastError();  // no device: clear the error of the query
    const int nw = t.threads / 32;
    long long cap = 148LL * (65536 / (128 * t.threads));
    if (p->max_ctas > 0 && cap > p->max_ctas) cap = p->max_ctas;
    const long long need = ((long long)s->n_groups + nw - 1) / nw;
    return (int)(need < cap ? need : cap);
}

// One warp-team launch: slope slots after the work-queue counter, grid
// capped by the slots the scratch holds.  Returns kNotLaunched when the team
// was not asked for (SPT_TEAM_AUTO) and either the groups do not fill every
// resident warp of the launch at least once (fewer groups are spread wider by
// one group per CTA) or the scratch holds fewer slots than a full grid.
int run_warp_team(const SptState* s, const SptTraceParams* p, const SptGeometry* g, const SptBem* b, int far,
                  unsigned char* scratch, int64_t scratch_bytes, cudaStream_t stream, const char* who) {
    spt::TraceLaunch t{};
    t.s = s;
    t.p = p;
    t.g = g;
    t.bem = *b;
    t.threads = warp_team_threads(p);
    t.work = reinterpret_cast<int*>(scratch);
    t.stream = stream;
    t.warp_team = true;
    t.slots = reinterpret_cast<double*>(scratch + 256);
    const long long avail = scratch_bytes > 256 ? (scratch_bytes - 256) / warp_team_slot_bytes(t.threads) : 0;
    const int full = warp_team_grid(s, p, g, b, far);
    if (p->team != SPT_TEAM_WARP) {
        // the launch's resident CTAs, were there groups for all of them
        SptState many = *s;
        many.n_groups = 1 << 30;
        const long long resident = warp_team_grid(&many, p, g, b, far);
        if ((long long)s->n_groups < resident * (t.threads / 32) || avail < full) return kNotLaunched;
    }
    if (avail < 1)
        return fail(SPT_ERR_ARG, "%s: scratch of %lld bytes holds no warp-team slot of %lld bytes", who,
                    (long long)scratch_bytes, (long long)warp_team_slot_bytes(t.threads));
    t.max_slots = avail;
    if (p->max_ctas > 0 && t.max_slots > p->max_ctas) t.max_slots = p->max_ctas;
    int grid = 0, per_sm = 0;
    size_t smem = 0;
    int rc = dispatch_kind(g->kind, t, p->form, far, false, &grid, &smem, &per_sm);
    if (rc) return fail(SPT_ERR_CUDA, "%s: warp-team launch setup: %s", who, cudaGetErrorString((cudaError_t)rc));
    if (per_sm < 1) return fail(SPT_ERR_CAPACITY, "%s: warp team of %d threads does not fit an SM", who, t.threads);
    rc = cuda_check(cudaMemsetAsync(t.work, 0, sizeof(int), stream), "cudaMemsetAsync");
    if (rc) return rc;
    rc = dispatch_kind(g->kind, t, p->form, far, true, &grid, &smem, &per_sm);
    if (rc) return fail(SPT_ERR_CUDA, "%s: trace_warp_kernel launch: %s", who, cudaGetErrorString((cudaError_t)rc));
    return SPT_OK;
}

int run_trace(const SptState* s, const SptTraceParams* p, const SptGeometry* g, const SptBem* b,
              unsigned char* scratch, int64_t scratch_bytes, cudaStream_t stream, const char* who) {
    const int far = far_rule_of(g, b);
    if (p->team != SPT_TEAM_AUTO && p->team != SPT_TEAM_CTA && p->team != SPT_TEAM_WARP)
        return fail(SPT_ERR_ARG, "%s: unknown team %d", who, p->team);
    const bool warp_ok = warp_team_offered(s, p, g, b, far);
    if (p->team == SPT_TEAM_WARP && !warp_ok)
        return fail(SPT_ERR_ARG,
                    "%s: the warp team needs a BEM geometry without the image-charge force, the float64 form, the "
                    "adaptive far rule and groups of at most 32 particles", who);
    if (warp_ok && p->team != SPT_TEAM_CTA) {
        const int rc = run_warp_team(s, p, g, b, far, scratch, scratch_bytes, stream, who);
        if (rc != kNotLaunched) return rc;
    }
    const spt::Layout L = spt::make_layout(s->max_group_size, far, p->form == SPT_FORM_SURROGATE);
    spt::TraceLaunch t{};
    t.s = s;
    t.p = p;
    t.g = g;
    t.bem = b ? *b : SptBem{};
    t.threads = trace_threads(s, p, far);
    t.work = reinterpret_cast<int*>(scratch);
    t.stream = stream;
    if (L.big) {
        const int64_t slot_bytes = (int64_t)spt::big_slot_doubles(s->max_group_size) * 8;
        t.max_slots = (scratch_bytes - 256) / slot_bytes;
        if (t.max_slots < 1)
            return fail(SPT_ERR_ARG, "%s: scratch of %lld bytes holds no slope buffer of %lld bytes", who,
                        (long long)scratch_bytes, (long long)slot_bytes);
        t.slots = reinterpret_cast<double*>(scratch + 256);
    }
    if (p->max_ctas > 0 && (t.max_slots == 0 || t.max_slots > p->max_ctas)) t.max_slots = p->max_ctas;
    int grid = 0, per_sm = 0;
    size_t smem = 0;
    int rc = dispatch_kind(g->kind, t, p->form, far, false, &grid, &smem, &per_sm);
    if (rc == -1) return fail(SPT_ERR_ARG, "%s: form %d with far rule %d is not offered for geometry kind %d", who, p->form,
                              far, g->kind);
    if (rc) return fail(SPT_ERR_CUDA, "%s: launch setup: %s", who, cudaGetErrorString((cudaError_t)rc));
    if (per_sm < 1) return fail(SPT_ERR_CAPACITY, "%s: group size %d does not fit one CTA", who, s->max_group_size);
    // the counter must start at zero; the slot buffers are written before they are read
    rc = cuda_check(cudaMemsetAsync(t.work, 0, sizeof(int), stream), "cudaMemsetAsync");
    if (rc) return rc;
    rc = dispatch_kind(g->kind, t, p->form, far, true, &grid, &smem, &per_sm);
    if (rc) return fail(SPT_ERR_CUDA, "%s: trace_kernel launch: %s", who, cudaGetErrorString((cudaError_t)rc));
    return SPT_OK;
}

}  // namespace

extern "C" {

int spt_abi_version(void) { return SPT_ABI_VERSION; }

int spt_last_error(char* buf, int32_t len) {
    const int n = (int)strlen(g_err);
    if (buf && len > 0) {
        strncpy(buf, g_err, len - 1);
        buf[len - 1] = 0;
    }
    return n;
}

int spt_trace_workspace_bytes(const SptState* s, const SptTraceParams* p, const SptGeometry* g, const SptBem* b,
                              int64_t* bytes) {
    if (!s || !p || !g || !bytes) return fail(SPT_ERR_ARG, "null argument");
    const spt::Layout L = spt::make_layout(s->max_group_size, far_rule_of(g, b), p->form == SPT_FORM_SURROGATE);
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int64_t n = 256;
    // groups above 256 particles: one slope buffer per CTA, two 256-thread CTAs per SM
    if (L.big) n += (int64_t)sms * 2 * (int64_t)spt::big_slot_doubles(s->max_group_size) * 8;
    // the warp team: one slot per warp of its whole grid
    const int far = far_rule_of(g, b);
    if (p->team != SPT_TEAM_CTA && warp_team_offered(s, p, g, b, far)) {
        const int64_t w = 256 + (int64_t)warp_team_grid(s, p, g, b, far) * warp_team_slot_bytes(warp_team_threads(p));
        if (w > n) n = w;
    }
    *bytes = n;
    return SPT_OK;
}

int spt_trace(const SptState* s, const SptTraceParams* p, const SptGeometry* g, const SptBem* b, void* ws,
              int64_t ws_bytes, void* stream) {
    if (!s || !p || !g || !ws) return fail(SPT_ERR_ARG, "null argument");
    if (s->n_groups <= 0) return SPT_OK;
    if (s->max_group_size <= 0 || s->max_group_size > 1024)
        return fail(SPT_ERR_CAPACITY, "max_group_size %d outside [1, 1024]", s->max_group_size);
    if (s->n_active && !s->group_order) return fail(SPT_ERR_ARG, "n_active needs group_order");
    if (reinterpret_cast<uintptr_t>(ws) & 255) return fail(SPT_ERR_ARG, "workspace must be 256-byte aligned");
    if (p->form != SPT_FORM_FP64 && p->form != SPT_FORM_MIXED && p->form != SPT_FORM_SURROGATE)
        return fail(SPT_ERR_ARG, "unknown form %d", p->form);
    if (is_bem(g->kind)) {
        int rc = check_bem(b);
        if (!rc) rc = check_image(g, b, s->max_group_size);
        if (rc) return rc;
    }
    if (p->form == SPT_FORM_SURROGATE) {
        const int rc = check_surrogate(p, g);
        if (rc) return rc;
    }
    return run_trace(s, p, g, b, static_cast<unsigned char*>(ws), ws_bytes, static_cast<cudaStream_t>(stream),
                     "spt_trace");
}

int spt_accel(const SptAccelArgs* a, const SptGeometry* g, const SptBem* b, void* stream) {
    if (!a || !g) return fail(SPT_ERR_ARG, "null argument");
    if (a->n_groups <= 0) return SPT_OK;
    if (a->max_group_size <= 0 || a->max_group_size > spt::kSmallGroup)
        return fail(SPT_ERR_CAPACITY, "spt_accel: group size must be in [1, %d]", spt::kSmallGroup);
    if (a->form != SPT_FORM_FP64 && a->form != SPT_FORM_MIXED) return fail(SPT_ERR_ARG, "spt_accel: form %d", a->form);
    if (is_bem(g->kind)) {
        int rc = check_bem(b);
        if (!rc) rc = check_image(g, b, a->max_group_size);
        if (rc) return rc;
    }
    SptBem bem = b ? *b : SptBem{};
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int rc = -1;
    switch (g->kind) {
        case SPT_GEOM_FLAT: rc = spt::accel_dispatch<SPT_GEOM_FLAT>(a, g, bem, st); break;
        case SPT_GEOM_TIP: rc = spt::accel_dispatch<SPT_GEOM_TIP>(a, g, bem, st); break;
        case SPT_GEOM_TIP_BEM: rc = spt::accel_dispatch<SPT_GEOM_TIP_BEM>(a, g, bem, st); break;
        case SPT_GEOM_WELL_BEM: rc = spt::accel_dispatch<SPT_GEOM_WELL_BEM>(a, g, bem, st); break;
        case SPT_GEOM_POST_BEM: rc = spt::accel_dispatch<SPT_GEOM_POST_BEM>(a, g, bem, st); break;
        default: return fail(SPT_ERR_ARG, "unknown geometry kind %d", g->kind);
    }
    if (rc == -1) return fail(SPT_ERR_ARG, "spt_accel: form %d is not offered here", a->form);
    if (rc) return fail(SPT_ERR_CUDA, "accel_kernel launch: %s", cudaGetErrorString((cudaError_t)rc));
    return SPT_OK;
}

int spt_bem_field(const double* x, const double* y, const double* z, int64_t n, const SptBem* b, int32_t form,
                  double* ex, double* ey, double* ez, void* stream) {
    if (n <= 0) return SPT_OK;
    if (!x || !y || !z || !ex || !ey || !ez) return fail(SPT_ERR_ARG, "null argument");
    int rc = check_bem(b);
    if (rc) return rc;
    if (form != SPT_FORM_FP64 && form != SPT_FORM_MIXED) return fail(SPT_ERR_ARG, "unknown form %d", form);
    const long long blocks = (n + spt::kFieldChunk - 1) / spt::kFieldChunk;
    if (blocks > 0x7fffffffLL) return fail(SPT_ERR_CAPACITY, "too many points");
    const int far = b->far_rule;
    const spt::Layout L = spt::make_layout(spt::kFieldChunk, far);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
#define SPT_FIELD(F, R)                                                                                           \
    {                                                                                                             \
        rc = set_smem(spt::bem_field_kernel<F, R>, L.bytes);                                                       \
        if (rc) return rc;                                                                                        \
        spt::bem_field_kernel<F, R><<<(unsigned)blocks, spt::kMaxThreads, L.bytes, st>>>(x, y, z, n, *b, ex, ey, ez, \
                                                                                       nullptr);                  \
        return cuda_check(cudaGetLastError(), "bem_field_kernel launch");                                         \
    }
    if (form == SPT_FORM_FP64 && far == SPT_FAR_REFERENCE) SPT_FIELD(SPT_FORM_FP64, SPT_FAR_REFERENCE)
    if (form == SPT_FORM_FP64) SPT_FIELD(SPT_FORM_FP64, SPT_FAR_ADAPTIVE)
    if (far == SPT_FAR_REFERENCE) SPT_FIELD(SPT_FORM_MIXED, SPT_FAR_REFERENCE)
    SPT_FIELD(SPT_FORM_MIXED, SPT_FAR_ADAPTIVE)
#undef SPT_FIELD
}

int spt_surrogate_field(const double* x, const double* y, const double* z, int64_t n, const SptBem* b,
                        const SptTraceParams* sur, double* ex, double* ey, double* ez, void* stream) {
    if (n <= 0) return SPT_OK;
    if (!x || !y || !z || !ex || !ey || !ez || !sur) return fail(SPT_ERR_ARG, "null argument");
    int rc = check_bem(b);
    if (rc) return rc;
    rc = check_surrogate_params(sur);
    if (rc) return rc;
    const long long blocks = (n + spt::kSurChunk - 1) / spt::kSurChunk;
    if (blocks > 0x7fffffffLL) return fail(SPT_ERR_CAPACITY, "too many points");
    const spt::Layout L = spt::make_layout(spt::kSurChunk, b->far_rule, true);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (b->far_rule == SPT_FAR_REFERENCE) {
        rc = set_smem(spt::surrogate_field_kernel<SPT_FAR_REFERENCE>, L.bytes);
        if (rc) return rc;
        spt::surrogate_field_kernel<SPT_FAR_REFERENCE><<<(unsigned)blocks, spt::kMaxThreads, L.bytes, st>>>(
            x, y, z, n, *b, *sur, ex, ey, ez, nullptr);
    } else {
        rc = set_smem(spt::surrogate_field_kernel<SPT_FAR_ADAPTIVE>, L.bytes);
        if (rc) return rc;
        spt::surrogate_field_kernel<SPT_FAR_ADAPTIVE><<<(unsigned)blocks, spt::kMaxThreads, L.bytes, st>>>(
            x, y, z, n, *b, *sur, ex, ey, ez, nullptr);
    }
    return cuda_check(cudaGetLastError(), "surrogate_field_kernel launch");
}

int spt_compact_groups(const int32_t* order, int32_t n, const int32_t* status, int32_t* out, int32_t* n_active,
                       void* stream) {
    if (!status || !out || !n_active || n < 0) return fail(SPT_ERR_ARG, "null argument");
    spt::compact_kernel<<<1, spt::kCompactThreads, 0, static_cast<cudaStream_t>(stream)>>>(order, n, status, out, n_active);
    return cuda_check(cudaGetLastError(), "compact_kernel launch");
}

int spt_ring_field(const double* rho, const double* z, const double* a, int64_t n, int32_t form, double* er,
                   double* ez, void* stream) {
    if (n <= 0) return SPT_OK;
    if (!rho || !z || !a || !er || !ez) return fail(SPT_ERR_ARG, "null argument");
    const long long blocks = (n + 255) / 256 < 148 * 8 ? (n + 255) / 256 : 148 * 8;
    spt::ring_kernel<<<(unsigned)blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(rho, z, a, n, form, er, ez);
    return cuda_check(cudaGetLastError(), "ring_kernel launch");
}

int spt_ellip_ke(const double* p, int64_t n, int32_t form, double* K, double* E, void* stream) {
    if (n <= 0) return SPT_OK;
    if (!p || !K || !E) return fail(SPT_ERR_ARG, "null argument");
    const long long blocks = (n + 255) / 256 < 148 * 8 ? (n + 255) / 256 : 148 * 8;
    spt::ellip_kernel<<<(unsigned)blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(p, n, form, K, E);
    return cuda_check(cudaGetLastError(), "ellip_kernel launch");
}

int spt_bem_assemble(const double* profile_rho, const double* profile_z, int32_t n_nodes, double refine_ratio,
                     int32_t max_depth, const double* gauss4_x, const double* gauss4_w, double* A, void* stream) {
    if (n_nodes < 2) return fail(SPT_ERR_ARG, "profile needs at least 2 nodes");
    if (!profile_rho || !profile_z || !A || !gauss4_x || !gauss4_w) return fail(SPT_ERR_ARG, "null argument");
    if (max_depth < 0 || max_depth > 40) return fail(SPT_ERR_CAPACITY, "max_depth must be in [0, 40]");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int rc = cuda_check(cudaMemsetAsync(A, 0, sizeof(double) * (size_t)n_nodes * n_nodes, st), "cudaMemsetAsync");
    if (rc) return rc;
    const long long pairs = (long long)n_nodes * (n_nodes - 1);
    const long long blocks = (pairs + 127) / 128;
    spt::assemble_kernel<<<(unsigned)blocks, 128, 0, st>>>(profile_rho, profile_z, n_nodes, refine_ratio, max_depth,
                                                         gauss4_x, gauss4_w, A);
    return cuda_check(cudaGetLastError(), "assemble_kernel launch");
}

}  // extern "C"

// ===========================================================================
// spt_trace_noalloc: spt_trace for callers that cannot allocate device memory.
//
// Its scratch (the work-queue counter and, for groups above 256 particles,
// the per-CTA slope buffers) is this file-scope device array, so the call
// needs no workspace and allocates nothing.  The array is part of the
// library image: every GPU that loads the library holds its 4 MiB until the
// process exits.  Host code cannot use `g_noalloc_scratch` as an address --
// on the host that name is only a stand-in -- so its device address is
// looked up with cudaGetSymbolAddress, with the device current, on the first
// call in each CUDA context, and cached under that context's unique id: a
// context created after a device reset (or a caller's own driver-API
// context) loads the module again, possibly at another address, and gets a
// fresh lookup.
namespace {
constexpr size_t kNoAllocScratchBytes = size_t(4) << 20;
}
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {
struct NoAllocCache {
    std::mutex mu;
    unsigned long long ctx_id = 0;
    void* ptr = nullptr;
};
NoAllocCache g_noalloc_cache[64];

// Driver entry points for the context checks, looked up through the runtime
// (the library does not link the driver library directly, so it loads on
// machines without a GPU driver).
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

int driver_fn(const char* name, void** fn) {
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    const cudaError_t e = cudaGetDriverEntryPoint(name, fn, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !*fn)
        return fail(SPT_ERR_CUDA, "driver entry point %s unavailable", name);
    return SPT_OK;
}

int noalloc_scratch(void** out) {
    int dev = 0;
    int rc = cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    if (rc) return rc;
    if (dev < 0 || dev >= 64) return fail(SPT_ERR_CAPACITY, "device index %d above 63", dev);
    void* f_cur = nullptr;
    void* f_id = nullptr;
    if ((rc = driver_fn("cuCtxGetCurrent", &f_cur)) || (rc = driver_fn("cuCtxGetId", &f_id))) return rc;
    CUcontext ctx = nullptr;
    if (reinterpret_cast<CtxGetCurrentFn>(f_cur)(&ctx) != CUDA_SUCCESS) return fail(SPT_ERR_CUDA, "cuCtxGetCurrent failed");
    if (!ctx) {
        // no context current yet: bind the device's primary context (what the runtime would use)
        rc = cuda_check(cudaSetDevice(dev), "cudaSetDevice");
        if (rc) return rc;
        if (reinterpret_cast<CtxGetCurrentFn>(f_cur)(&ctx) != CUDA_SUCCESS || !ctx)
            return fail(SPT_ERR_CUDA, "no current CUDA context");
    }
    unsigned long long id = 0;
    if (reinterpret_cast<CtxGetIdFn>(f_id)(ctx, &id) != CUDA_SUCCESS) return fail(SPT_ERR_CUDA, "cuCtxGetId failed");
    NoAllocCache& c = g_noalloc_cache[dev];
    std::lock_guard<std::mutex> lock(c.mu);
    if (!c.ptr || c.ctx_id != id) {
        void* p = nullptr;
        rc = cuda_check(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress(g_noalloc_scratch)");
        if (rc) return rc;
        c.ptr = p;
        c.ctx_id = id;
    }
    *out = c.ptr;
    return SPT_OK;
}

}  // namespace

extern "C" int spt_trace_noalloc(const SptState* s, const SptTraceParams* p, const SptGeometry* g, const SptBem* b,
                                 void* stream) {
    if (!s || !p || !g) return fail(SPT_ERR_ARG, "null argument");
    if (s->n_groups <= 0) return SPT_OK;
    if (s->max_group_size <= 0 || s->max_group_size > 1024)
        return fail(SPT_ERR_CAPACITY, "spt_trace_noalloc: max_group_size %d outside [1, 1024]", s->max_group_size);
    if (s->n_active && !s->group_order) return fail(SPT_ERR_ARG, "n_active needs group_order");
    if (p->form == SPT_FORM_SURROGATE) return fail(SPT_ERR_ARG, "spt_trace_noalloc: the learned form is not offered");
    if (p->form != SPT_FORM_FP64 && p->form != SPT_FORM_MIXED) return fail(SPT_ERR_ARG, "unknown form %d", p->form);
    if (is_bem(g->kind)) {
        int rc = check_bem(b);
        if (!rc) rc = check_image(g, b, s->max_group_size);
        if (rc) return rc;
    }
    void* scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    return run_trace(s, p, g, b, static_cast<unsigned char*>(scratch), (int64_t)kNoAllocScratchBytes,
                     static_cast<cudaStream_t>(stream), "spt_trace_noalloc");
}
