// Device code of the B200 (sm_100a) tracer, shared by the translation units
// that instantiate the trace kernel per geometry kind (spt_trace_<kind>.cu)
// and by the C ABI (spt_kernels.cu).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <math.h>
#include <type_traits>

#include "../../include/spt_b200.h"
#include "spt_image.cuh"
#include "spt_math.cuh"
#include "spt_umma.cuh"

namespace spt {

// A CTA is one team of nt = blockDim.x threads (32, 64, 128 or 256) working on
// one group at a time; its width is a launch parameter (smaller CTAs for
// smaller groups: more CTAs per SM, fewer warps per barrier).  Static shared
// arrays are sized for the widest CTA.
constexpr int kMaxThreads = 256;
constexpr int kMaxWarps = kMaxThreads / 32;
constexpr int kRound = 4;           // points per far-sum round (largest; the register tile of the far sums)
constexpr double kKappa = 16.0;     // default conditioning bound of the mixed form's float32 sums
constexpr int kTileNodes = 2048;    // nodes per TMA tile row (largest; halved while shared memory is short)
constexpr size_t kMaxSmem = 226 * 1024;  // dynamic part; the static __shared__ scalars take the rest of 227 KB
constexpr int kSmallGroup = 256;    // groups above this keep slopes in global memory

// Dormand-Prince 5(4) tableau (batched_rk45.py:30-50).
static __device__ __constant__ double kA[6][5] = {
    {0, 0, 0, 0, 0},
    {1.0 / 5, 0, 0, 0, 0},
    {3.0 / 40, 9.0 / 40, 0, 0, 0},
    {44.0 / 45, -56.0 / 15, 32.0 / 9, 0, 0},
    {19372.0 / 6561, -25360.0 / 2187, 64448.0 / 6561, -212.0 / 729, 0},
    {9017.0 / 3168, -355.0 / 33, 46732.0 / 5247, 49.0 / 176, -5103.0 / 18656}};
static __device__ __constant__ double kB[6] = {35.0 / 384, 0.0, 500.0 / 1113, 125.0 / 192, -2187.0 / 6784, 11.0 / 84};
static __device__ __constant__ double kE[7] = {71.0 / 57600, 0.0, -71.0 / 16695, 71.0 / 1920, -17253.0 / 339200, 22.0 / 525, -1.0 / 40};

constexpr double kSpeedOfLight = 299792458.0;
constexpr double kTiny = 2.2250738585072014e-308;  // np.finfo(float).tiny

// ---------------------------------------------------------------------------
// small helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tma_load_1d(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// Bounded wait on an mbarrier phase.  Returns false when the iteration limit
// ran out (the caller flags the group instead of spinning forever).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase) {
    uint32_t done = 0;
    for (int it = 0; it < (1 << 22); ++it) {
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// ---------------------------------------------------------------------------
// geometry helpers (fields.py, geometry.py, bem/fields.py, bem/geometry.py)

__device__ __forceinline__ bool well_contains(double rho, double z, const SptGeometry& g) {
    const double R = g.R, H = g.H;
    const double eps = 1e-6 * R;
    bool solid = (rho >= R * (1.0 - 1e-6)) ? (z <= 0.0) : (z <= -H * (1.0 + 1e-6));
    if (g.rim_fillet > 0.0) {
        const double rf = g.rim_fillet, cr = R + rf, cz = -rf;
        if (rho >= R - eps && rho <= R + rf + eps && z >= -rf - eps && z <= eps) solid = hypot(rho - cr, z - cz) <= rf;
    }
    if (g.bottom_fillet > 0.0) {
        const double bf = g.bottom_fillet, cr = R - bf, cz = -H + bf;
        if (rho <= R + eps && rho >= R - bf - eps && z <= -H + bf + eps && z >= -H - eps)
            solid = hypot(rho - cr, z - cz) >= bf;
    }
    return solid;
}

__device__ __forceinline__ bool post_inside(double x, double y, double z, const SptGeometry& g) {
    const double rk = g.R * (1.0 - 1e-6);
    const double r2 = x * x + y * y;
    const double zc = z - g.L;
    return (r2 <= rk * rk && z <= g.L) || (r2 + zc * zc <= rk * rk);
}

template <int KIND>
__device__ __forceinline__ bool kill_test(double x, double y, double z, const SptGeometry& g) {
    bool k = false;
    if (KIND == SPT_GEOM_FLAT) {
        k = g.has_kill_below && z <= g.kill_z_below;
    } else if (KIND == SPT_GEOM_TIP || KIND == SPT_GEOM_TIP_BEM) {
        const double rk = g.R * (1.0 - 1e-6);
        k = (x * x + y * y + z * z) <= rk * rk;
        if (g.has_kill_below) k = k || (z <= g.kill_z_below);
    } else if (KIND == SPT_GEOM_WELL_BEM) {
        k = well_contains(sqrt(x * x + y * y), z, g);
    } else {
        k = post_inside(x, y, z, g);
        if (g.has_kill_below) k = k || (z <= g.kill_z_below);
    }
    if (g.has_z_max) k = k || (z >= g.z_max);
    return k;
}

// analytic tip field (fields.py:119-160)
__device__ __forceinline__ void tip_field(double x, double y, double z, double Ez, double R, double& ex, double& ey,
                                          double& ez) {
    const double r = sqrt(x * x + y * y + z * z);
    const bool ok = (r >= R * (1.0 - 1e-6)) && (z >= 0.0);
    if (!ok) {
        ex = ey = ez = 0.0;
        return;
    }
    const double r3 = r * r * r;
    const double r5 = r3 * r * r;
    const double R3 = R * R * R;
    ex = 3.0 * Ez * R3 * x * z / r5;
    ey = 3.0 * Ez * R3 * y * z / r5;
    ez = Ez * (1.0 - R3 / r3 + 3.0 * R3 * z * z / r5);
}

// BEM geometries: is the point in the field's valid (vacuum) region
template <int KIND>
__device__ __forceinline__ bool bem_valid(double x, double y, double z, const SptGeometry& g) {
    if (KIND == SPT_GEOM_TIP_BEM) return (sqrt(x * x + y * y + z * z) >= g.R * (1.0 - 1e-6)) && (z >= 0.0);
    if (KIND == SPT_GEOM_WELL_BEM) return !well_contains(sqrt(x * x + y * y), z, g);
    return !post_inside(x, y, z, g) && (z >= 0.0);
}

__device__ __forceinline__ double blend_weight(double z, double zh) {
    const double zlo = 0.5 * zh;
    double s = (zh - z) / (zh - zlo);
    s = fmin(fmax(s, 0.0), 1.0);
    return s * s * (3.0 - 2.0 * s);
}

// ---------------------------------------------------------------------------
// shared-memory layout of one CTA

struct Layout {
    // offsets in doubles from the start of dynamic shared memory
    int y0, nw, sp, kp, kv;   // y0: 6E, nw: 6E, sp: 3E, kp/kv: 21E each
    int tb, td, q, m, cps;    // E each
    int fld;                  // 3E field
    int img;                  // 4E sphere images
    int bpt;                  // 8E per BEM list entry: x y z rho_e z_e near_r near_z (+1 pad)
    int imgs;                 // scratch of the BEM image-charge force (geometries with z0), or 0 doubles
    int sur;                  // surrogate region: act (4096), wt (4096), sout 2E, sseg E, st E, sd E, feat 128; -1 if none
    int tiles;                // reference far rule: 2 * 3 * tile_cap node tiles; adaptive: per-warp scratch
    int tile_cap;             // nodes per TMA tile row (reference far rule)
    int red;                  // kMaxWarps * 3 * kRound (far-round reduction: E_rho, E_z, sum of |terms|)
    int ints;                 // int region start (in doubles)
    int total_doubles;
    int live_off, list_off, flags_off;  // in ints from ints start
    size_t bytes;
    bool big;                 // slopes/y0/nw in global memory
};

// Segments per chunk of the adaptive far rule (8 runs of SPT_BLOCK_SEGS).
// Each warp classifies and sums its own rounds in a private scratch of
// kWarpScratchInts ints: three segment lists of kWarpChunk entries, the
// near masks of the first (kWarpChunk bytes) and four run lists.
constexpr int kWarpChunk = 256;
constexpr int kWarpScratchInts = 3 * kWarpChunk + kWarpChunk / 4 + 4 * (kWarpChunk / SPT_BLOCK_SEGS) +
                                  SPT_MAX_CLUSTER_RUNS / 32;
static_assert(kWarpScratchInts % 2 == 0, "per-warp scratch keeps 8-byte alignment");

// Shared-memory layout of one CTA for groups of up to E particles.  The far
// rule decides the big region: node tiles for the reference rule (the TMA
// bulk engine streams the node table through them), segment lists for the
// adaptive rule (which reads its few nodes through L1/L2), one scratch per
// warp of a CTA of `warps` warps.  want_tiles false: neither (paths that
// evaluate no far sum).
__host__ __device__ inline Layout make_layout(int E, int far_rule, bool want_sur = false, bool want_tiles = true,
                                              int warps = kMaxWarps, int img_doubles = 0) {
    Layout L;
    const bool big = E > kSmallGroup;
    int o = 0;
    L.big = big;
    if (!big) {
        L.y0 = o; o += 6 * E;
        L.nw = o; o += 6 * E;
        L.kp = o; o += 21 * E;
        L.kv = o; o += 21 * E;
    } else {
        L.y0 = L.nw = L.kp = L.kv = -1;
    }
    L.sp = o; o += 3 * E;
    L.tb = o; o += E;
    L.td = o; o += E;
    L.q = o; o += E;
    L.m = o; o += E;
    L.cps = o; o += E;
    L.fld = o; o += 3 * E;
    L.img = o; o += 4 * E;
    L.bpt = o; o += 8 * E;
    L.imgs = o; o += img_doubles;
    if (want_sur) {
        o = (o + 127) & ~127;  // 1 KiB alignment for the tensor-core operand tiles
        L.sur = o; o += 8192 + 5 * E + 128;
    } else {
        L.sur = -1;
    }
    o = (o + 1) & ~1;  // 16-byte alignment for the TMA tiles
    const int base = o;
    const int n_ints = 2 * E + kRound * 256 / 4 + 4;  // live, list, near flags (bytes) packed in ints
    const bool tiles = want_tiles && far_rule == SPT_FAR_REFERENCE;
    const bool lists = want_tiles && far_rule != SPT_FAR_REFERENCE;
    for (int cap = kTileNodes; cap >= 256; cap >>= 1) {
        o = base;
        L.tile_cap = tiles ? cap : 0;
        L.tiles = o; o += tiles ? 2 * 3 * cap : (lists ? warps * kWarpScratchInts / 2 : 0);
        L.red = o; o += kMaxWarps * 3 * kRound;
        L.ints = o;
        L.total_doubles = o + (n_ints + 1) / 2;
        L.bytes = (size_t)L.total_doubles * 8 + 64;  // + mbarriers
        if (L.bytes <= kMaxSmem || !tiles) break;
    }
    L.live_off = 0;
    L.list_off = E;
    L.flags_off = 2 * E;
    return L;
}

// Partial right-hand sides of the image-charge solve per profile node: as
// many source subsets as the CTA has threads per node, 1 to 4.
__host__ __device__ inline int image_chunks(int P, int threads) {
    const int c = threads / (P > 0 ? P : 1);
    return c < 1 ? 1 : (c > 4 ? 4 : c);
}

// Shared doubles the BEM image-charge force needs for groups of up to E
// particles on a CTA of `threads` threads: 0 unless the geometry is a BEM
// tip or well built with z0 and the image tables are given.
__host__ __device__ inline int image_scratch(const SptGeometry& g, const SptBem& b, int E, int threads) {
    if (!(g.kind == SPT_GEOM_TIP_BEM || g.kind == SPT_GEOM_WELL_BEM) || !g.has_image || b.image.n_nodes < 2) return 0;
    return (int)spt_img::scratch_doubles(E, b.image.mirror_symmetric, b.image.n_nodes, b.image.n_max,
                                         image_chunks(b.image.n_nodes, threads));
}

// global per-CTA slot for big groups: y0 6E, nw 6E, kp 21E, kv 21E
__host__ __device__ inline size_t big_slot_doubles(int E) { return (size_t)54 * E; }

struct Ctx {
    // the kernel's parameter blocks (__grid_constant__: referenced in place, never copied)
    const SptGeometry& g;
    const SptBem& bem;
    __device__ Ctx(const SptGeometry& g_, const SptBem& b_) : g(g_), bem(b_) {}
    int nt, nw;      // threads and warps of this CTA (blockDim.x, a multiple of 32)
    double cm;       // charge_to_mass
    double kc;       // Coulomb constant 1/(4 pi eps0)
    double soft2;    // plummer^2
    int round_pts;           // points per far-sum round, 1..kRound
    double kappa;            // mixed form: float32 sums whose sum of |terms| exceeds kappa x |result| are redone in float64
    int* redo;               // shared flag of that test
    int E;
    double* base;    // dynamic smem
    Layout L;
    double *y0, *nw_, *sp, *kp, *kv, *tb, *td, *q, *m, *cps, *fld, *img, *bpt, *tiles, *red, *imgs;
    int* live;
    int* list;
    unsigned char* nflag;
    uint64_t* bars;
    uint32_t phase[3];          // parity of the next phase to wait for on bars[0..2] (identical in every thread)
    unsigned long long* cnt;    // shared-memory counter partials of the CTA (flushed by flush_counters)
    // learned form
    uint8_t *act, *wt;          // BF16 operand tiles (activations, weights), canonical K-major, 32 KiB each
    double *sout, *st, *sd;     // surrogate E (rho, z) per record; closest-point parameter and distance
    int* sseg;                  // closest segment per record
    float* feat;                // features of the current 128-row chunk
    const float* sw;            // FP32 (BF16-rounded) parameters
    const __nv_bfloat16* sw16;  // BF16 parameters
    const double *s_start, *log_scale;
    double s_end, sig_floor, band, spot, dmin, dmax;
    unsigned long long* sstats;
    uint32_t tmem;
    uint32_t key;               // hash key of the current stage evaluation (spot checks)
};

// add v (a per-thread partial) to the CTA's counter k: warp sum, one shared atomic per warp
__device__ __forceinline__ void count_add(Ctx& c, int k, unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(c.cnt + k, v);
}

__device__ inline void bind(Ctx& c, double* smem, int E, int far_rule, double* slot, unsigned long long* s_cnt,
                            bool sur = false) {
    c.base = smem;
    c.E = E;
    c.nt = blockDim.x;
    c.nw = blockDim.x >> 5;
    c.L = make_layout(E, far_rule, sur, true, blockDim.x >> 5, image_scratch(c.g, c.bem, E, blockDim.x));
    c.round_pts = kRound;
    c.kappa = kKappa;
    c.cnt = s_cnt;
    const Layout& L = c.L;
    if (!L.big) {
        c.y0 = smem + L.y0;
        c.nw_ = smem + L.nw;
        c.kp = smem + L.kp;
        c.kv = smem + L.kv;
    } else {
        c.y0 = slot;
        c.nw_ = slot + 6 * E;
        c.kp = slot + 12 * E;
        c.kv = slot + 33 * E;
    }
    c.sp = smem + L.sp;
    c.tb = smem + L.tb;
    c.td = smem + L.td;
    c.q = smem + L.q;
    c.m = smem + L.m;
    c.cps = smem + L.cps;
    c.fld = smem + L.fld;
    c.img = smem + L.img;
    c.bpt = smem + L.bpt;
    c.imgs = smem + L.imgs;
    c.tiles = smem + L.tiles;
    c.red = smem + L.red;
    int* ib = reinterpret_cast<int*>(smem + L.ints);
    c.live = ib + L.live_off;
    c.list = ib + L.list_off;
    c.nflag = reinterpret_cast<unsigned char*>(ib + L.flags_off);
    c.redo = ib + L.flags_off + kRound * 256 / 4;  // first spare int after the near-flag bytes
    c.bars = reinterpret_cast<uint64_t*>(smem + L.total_doubles + 1);
    for (int k = threadIdx.x; k < SPT_N_COUNTERS; k += blockDim.x) s_cnt[k] = 0;
    if (L.sur >= 0) {
        double* r = smem + L.sur;
        c.act = reinterpret_cast<uint8_t*>(r);
        c.wt = reinterpret_cast<uint8_t*>(r + 4096);
        c.sout = r + 8192;
        c.st = c.sout + 2 * E;
        c.sd = c.st + E;
        c.sseg = reinterpret_cast<int*>(c.sd + E);
        c.feat = reinterpret_cast<float*>(c.sd + 2 * E);
    }
}

// ---------------------------------------------------------------------------
// BEM: segment table access

struct Seg {
    double p0r, p0z, tr, tz, len, ur, uz, nr, nz, s0, s1;
};

__device__ __forceinline__ double segf(const SptBem& b, int f, int s) { return __ldg(b.seg + (size_t)f * b.seg_stride + s); }

// closest-point distance^2 of (rq, zq) to segment s (bem/axisymmetric.py:117-133,
// 374-381), with no FMA contraction: the on-surface offset below is a
// threshold test on this value, so it is rounded like the reference's.
__device__ __forceinline__ double seg_dist2(const SptBem& b, int s, double rq, double zq) {
    const double p0x = segf(b, 0, s), p0y = segf(b, 1, s), ax = segf(b, 2, s), ay = segf(b, 3, s);
    const double ab = __dadd_rn(__dmul_rn(ax, ax), __dmul_rn(ay, ay));
    double t = __ddiv_rn(__dadd_rn(__dmul_rn(__dadd_rn(rq, -p0x), ax), __dmul_rn(__dadd_rn(zq, -p0y), ay)), ab);
    t = fmin(fmax(t, 0.0), 1.0);
    const double cr = __dadd_rn(p0x, __dmul_rn(t, ax)), cz = __dadd_rn(p0y, __dmul_rn(t, ay));
    const double dr = __dadd_rn(rq, -cr), dz = __dadd_rn(zq, -cz);
    return __dadd_rn(__dmul_rn(dr, dr), __dmul_rn(dz, dz));
}

// near test of bem/axisymmetric.py:566-570 -> (near, projection, distance)
__device__ __forceinline__ bool seg_near(const SptBem& b, int s, double re, double ze, double& proj, double& dist) {
    const double p0r = segf(b, 0, s), p0z = segf(b, 1, s), L = segf(b, 4, s), ur = segf(b, 5, s), uz = segf(b, 6, s);
    const double dr = re - p0r, dz = ze - p0z;
    const double along = dr * ur + dz * uz;
    proj = fmin(fmax(along, 0.0), L);
    const double ar = dr - proj * ur, az = dz - proj * uz;
    dist = sqrt(ar * ar + az * az);
    return dist < L;
}

// Runs of SPT_BLOCK_SEGS consecutive segments (SptBem.blk): a lower bound of
// the distance from (r, z) to every segment of run q, less a relative margin
// that covers the rounding of this bound and of the table, and the run's
// largest segment length.
__device__ __forceinline__ double blk_lower(const SptBem& b, int q, double r, double z) {
    const double cr = __ldg(b.blk + q), cz = __ldg(b.blk + b.blk_stride + q), rad = __ldg(b.blk + 2 * b.blk_stride + q);
    const double dc = sqrt((r - cr) * (r - cr) + (z - cz) * (z - cz));
    return dc - rad - 1e-9 * (dc + rad);
}
__device__ __forceinline__ double blk_lmax(const SptBem& b, int q) { return __ldg(b.blk + 3 * b.blk_stride + q); }


// Fixed-order block reduction of a far round's accumulators into record
// slots 5, 6 (far + near sums).  Mixed form: the Kahan sums are folded in,
// and when the sum of |float32 terms| at a point exceeds kappa times the
// whole field there (uniform + perturbation), *c.redo is set -- the float32
// result is then ill-conditioned (shielded regions, where the perturbation
// cancels the uniform field) and the caller recomputes the round in float64.
template <int NP, bool MIX>
__device__ __forceinline__ void round_reduce(Ctx& c, int r0, int np_, double* ar, double* az, const float* fr,
                                             const float* fz, const float* kr, const float* kz, const float* sa) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double* P = c.bpt;
#pragma unroll
    for (int p = 0; p < NP; ++p) {
        if (MIX) {
            ar[p] += (double)fr[p] - (double)kr[p];
            az[p] += (double)fz[p] - (double)kz[p];
        }
        const double vr = warp_sum(ar[p]);
        const double vz = warp_sum(az[p]);
        const double va = MIX ? warp_sum((double)sa[p]) : 0.0;
        if (lane == 0) {
            c.red[warp * 3 * kRound + p] = vr;
            c.red[warp * 3 * kRound + kRound + p] = vz;
            c.red[warp * 3 * kRound + 2 * kRound + p] = va;
        }
    }
    __syncthreads();
    if (tid < np_) {
        double sr = 0.0, sz = 0.0, sabs = 0.0;
        for (int w = 0; w < c.nw; ++w) {
            sr += c.red[w * 3 * kRound + tid];
            sz += c.red[w * 3 * kRound + kRound + tid];
            sabs += c.red[w * 3 * kRound + 2 * kRound + tid];
        }
        const int k = r0 + tid;
        const double er = sr + P[8 * k + 7], ez = sz + c.fld[3 * k + 2];
        P[8 * k + 5] = er;
        P[8 * k + 6] = ez;
        if (MIX) {
            const double tz = ez + c.g.E_gun;
            if (!(sabs <= c.kappa * sqrt(er * er + tz * tz))) atomicOr(c.redo, 1);
        }
    }
    __syncthreads();
}

// One far-sum round for points r0..r0+np_-1 of the list (np_ <= NP): the
// node table streams through shared memory in TMA tiles (double buffered);
// each thread takes NQ nodes at a time, strided by the CTA width, against
// all NP points (NP * NQ independent ring evaluations per iteration).
template <int NP, int NQ, bool MIX>
__device__ void far_round(Ctx& c, int r0, int np_, int n_tiles, int segs_per_tile, bool& ok,
                          unsigned long long& far_evals) {
    const SptBem& b = c.bem;
    const int tid = threadIdx.x;
    const int nseg = b.n_seg, nps = b.nodes_per_seg;
    const int tile_cap = c.L.tile_cap;
    double* P = c.bpt;
    double* tile[2] = {c.tiles, c.tiles + 3 * tile_cap};
    uint64_t* bars = c.bars;
    double pr[NP], pinv[NP], pz[NP], ar[NP], az[NP];
    float fr[NP], fz[NP], kr[NP], kz[NP], prf[NP], pinvf[NP];  // mixed form: Kahan sums and float copies
    float sa[NP];                                               // mixed form: sum of |float32 terms|
#pragma unroll
    for (int p = 0; p < NP; ++p) {
        const int k = r0 + (p < np_ ? p : 0);
        pr[p] = P[8 * k + 3];
        pinv[p] = pr[p] > 0.0 ? 1.0 / pr[p] : 0.0;
        pz[p] = P[8 * k + 4];
        ar[p] = 0.0;
        az[p] = 0.0;
        fr[p] = fz[p] = kr[p] = kz[p] = sa[p] = 0.0f;
        prf[p] = (float)pr[p];
        pinvf[p] = (float)pinv[p];
    }
    if (MIX && tid == 0) *c.redo = 0;  // ordered before the reduction's writes by the barriers between
    auto issue = [&](int t, int buf) {
        const int s_first = t * segs_per_tile;
        const int nn = min(segs_per_tile, nseg - s_first) * nps;
        const uint32_t bytes = (uint32_t)nn * 8u;
        mbar_expect_tx(&bars[buf], 3u * bytes);
        for (int row = 0; row < 3; ++row)
            tma_load_1d(tile[buf] + row * tile_cap, b.node + (size_t)row * b.node_stride + (size_t)s_first * nps, bytes,
                        &bars[buf]);
    };
    if (tid == 0) {
        issue(0, 0);
        if (n_tiles > 1) issue(1, 1);
    }
    for (int t = 0; t < n_tiles; ++t) {
        const int buf = t & 1;
        const int s_first = t * segs_per_tile;
        const int ns = min(segs_per_tile, nseg - s_first);
        for (int idx = tid; idx < np_ * ns; idx += c.nt) {
            const int p = idx / ns, sl = idx - p * ns;
            double proj, dist;
            c.nflag[p * 256 + sl] = seg_near(b, s_first + sl, P[8 * (r0 + p) + 3], P[8 * (r0 + p) + 4], proj, dist);
        }
        if (!mbar_wait(&bars[buf], c.phase[buf])) ok = false;
        c.phase[buf] ^= 1u;
        __syncthreads();
        if (ok) {
            const double* tr = tile[buf];
            const double* tz = tr + tile_cap;
            const double* tw = tz + tile_cap;
            const int nn = ns * nps;
            for (int q0 = tid; q0 < nn; q0 += c.nt * NQ) {
                double rq[NQ], zq[NQ], wq[NQ];
                int sl[NQ];
                bool in[NQ];
#pragma unroll
                for (int j = 0; j < NQ; ++j) {
                    const int q = q0 + j * c.nt;
                    in[j] = q < nn;
                    const int qq = in[j] ? q : 0;
                    rq[j] = tr[qq];
                    zq[j] = tz[qq];
                    wq[j] = tw[qq];
                    sl[j] = qq / nps;
                }
                if (MIX) {
                    // float32 Kahan sums; pairs the float path declines (p < 1e-3 or
                    // near the axis) are evaluated in float64
#pragma unroll
                    for (int p = 0; p < NP; ++p) {
#pragma unroll
                        for (int j = 0; j < NQ; ++j) {
                            if (p < np_ && in[j] && !c.nflag[p * 256 + sl[j]]) {
                                const double dz = pz[p] - zq[j];
                                float er, ez;
                                if (ring_far_f(prf[p], pinvf[p], (float)(pr[p] - rq[j]), (float)(pr[p] + rq[j]),
                                               (float)dz, (float)rq[j], er, ez)) {
                                    const float w = (float)wq[j];
                                    kahan_add(fr[p], kr[p], w * er);
                                    kahan_add(fz[p], kz[p], w * ez);
                                    sa[p] += fabsf(w * er) + fabsf(w * ez);
                                } else {
                                    // close to the ring: the term in float64, summed like the others
                                    double e64r, e64z;
                                    ring_field_far_cold(pr[p], 1.0 / pr[p], dz, rq[j], e64r, e64z);
                                    const float ter = (float)(wq[j] * e64r), tez = (float)(wq[j] * e64z);
                                    kahan_add(fr[p], kr[p], ter);
                                    kahan_add(fz[p], kz[p], tez);
                                    sa[p] += fabsf(ter) + fabsf(tez);
                                }
                                ++far_evals;
                            }
                        }
                    }
                } else {
#pragma unroll
                for (int p = 0; p < NP; ++p) {
#pragma unroll
                    for (int j = 0; j < NQ; ++j) {
                        if (p < np_ && in[j] && !c.nflag[p * 256 + sl[j]]) {
                            const double dz = pz[p] - zq[j];
                            double er, ez;
                            ring_field_far(pr[p], pinv[p], dz, rq[j], er, ez);
                            ar[p] = fma(wq[j], er, ar[p]);
                            az[p] = fma(wq[j], ez, az[p]);
                            ++far_evals;
                        }
                    }
                }
                }
            }
        }
        __syncthreads();
        if (tid == 0 && t + 2 < n_tiles) issue(t + 2, buf);
    }
    // fixed-order block reduction of the round's accumulators
    round_reduce<NP, MIX>(c, r0, np_, ar, az, fr, fz, kr, kz, sa);
}

// Adaptive far sum (SPT_FAR_ADAPTIVE) for points r0..r0+np_-1 of the list,
// computed by ONE warp (each warp of the CTA takes its own rounds; nothing
// here waits on another warp).  Segments are taken kWarpChunk at a time
// (kWarpRuns runs of SPT_BLOCK_SEGS).  The warp classifies the chunk's runs by
// the smallest lower-bound distance over the round's points: flagged runs at
// least ratio_run arclengths away take the 8-point rule over the whole run
// (list R3), runs whose every segment is at least ratio2 lengths away take
// Gauss-2 on each segment (R2), the rest (M) are classified segment by
// segment -- below ratio4 lengths the reference nodes, with an 8-bit mask of
// the points for which the segment is near (they skip it), below ratio2
// Gauss-4, else Gauss-2 (lists L0, L1, L2 in the warp's own shared scratch).
// The flattened node list L0 | L1 | L2 | R2 | R3 is then evaluated by the
// warp's lanes, NQ nodes in flight per lane, nodes read through L1/L2.
// Without run bounds every run is in M.  Lane 0 ends with the round's
// fields in record slots 5, 6 (near parts included); returns, in every lane,
// whether a float32 sum (MIX) was ill-conditioned (kappa test).
// Recurrence constants of the Legendre polynomials, P_(n+1) = a_n u P_n - b_n P_(n-1).
static __device__ __constant__ double kLegA[64] = {
#define SPT_LA(n) (2.0 * (n) + 1.0) / ((n) + 1.0)
    SPT_LA(0), SPT_LA(1), SPT_LA(2), SPT_LA(3), SPT_LA(4), SPT_LA(5), SPT_LA(6), SPT_LA(7), SPT_LA(8), SPT_LA(9),
    SPT_LA(10), SPT_LA(11), SPT_LA(12), SPT_LA(13), SPT_LA(14), SPT_LA(15), SPT_LA(16), SPT_LA(17), SPT_LA(18),
    SPT_LA(19), SPT_LA(20), SPT_LA(21), SPT_LA(22), SPT_LA(23), SPT_LA(24), SPT_LA(25), SPT_LA(26), SPT_LA(27),
    SPT_LA(28), SPT_LA(29), SPT_LA(30), SPT_LA(31), SPT_LA(32), SPT_LA(33), SPT_LA(34), SPT_LA(35), SPT_LA(36),
    SPT_LA(37), SPT_LA(38), SPT_LA(39), SPT_LA(40), SPT_LA(41), SPT_LA(42), SPT_LA(43), SPT_LA(44), SPT_LA(45),
    SPT_LA(46), SPT_LA(47), SPT_LA(48), SPT_LA(49), SPT_LA(50), SPT_LA(51), SPT_LA(52), SPT_LA(53), SPT_LA(54),
    SPT_LA(55), SPT_LA(56), SPT_LA(57), SPT_LA(58), SPT_LA(59), SPT_LA(60), SPT_LA(61), SPT_LA(62), SPT_LA(63)};
#undef SPT_LA
static __device__ __constant__ double kLegB[64] = {
#define SPT_LB(n) (n) / ((n) + 1.0)
    SPT_LB(0), SPT_LB(1), SPT_LB(2), SPT_LB(3), SPT_LB(4), SPT_LB(5), SPT_LB(6), SPT_LB(7), SPT_LB(8), SPT_LB(9),
    SPT_LB(10), SPT_LB(11), SPT_LB(12), SPT_LB(13), SPT_LB(14), SPT_LB(15), SPT_LB(16), SPT_LB(17), SPT_LB(18),
    SPT_LB(19), SPT_LB(20), SPT_LB(21), SPT_LB(22), SPT_LB(23), SPT_LB(24), SPT_LB(25), SPT_LB(26), SPT_LB(27),
    SPT_LB(28), SPT_LB(29), SPT_LB(30), SPT_LB(31), SPT_LB(32), SPT_LB(33), SPT_LB(34), SPT_LB(35), SPT_LB(36),
    SPT_LB(37), SPT_LB(38), SPT_LB(39), SPT_LB(40), SPT_LB(41), SPT_LB(42), SPT_LB(43), SPT_LB(44), SPT_LB(45),
    SPT_LB(46), SPT_LB(47), SPT_LB(48), SPT_LB(49), SPT_LB(50), SPT_LB(51), SPT_LB(52), SPT_LB(53), SPT_LB(54),
    SPT_LB(55), SPT_LB(56), SPT_LB(57), SPT_LB(58), SPT_LB(59), SPT_LB(60), SPT_LB(61), SPT_LB(62), SPT_LB(63)};
#undef SPT_LB

// Field (E_rho, E_z) at (rho, z) of a cluster from its record (z_c, r_max,
// M_0 .. M_(nt-1)): with r, u = cos(theta), s = sin(theta) about (0, z_c) and
// x = r_max / r, the potential (1/4 pi) sum_n M_n x^n P_n(u) / r gives
// E_r = (1/4 pi r^2) sum (n+1) M_n x^n P_n(u), E_theta = (s/4 pi r^2) sum
// M_n x^n P_n'(u), turned into (rho, z) components.  P_n' by
// P'_(n+1) = P'_(n-1) + (2n+1) P_n.
__device__ __forceinline__ void cluster_field(const double* rec, int nt, double rho, double z, double& er,
                                              double& ez) {
    const double dz = z - __ldg(rec);
    const double r2 = rho * rho + dz * dz;
    const double ir = rsqrt(r2);
    const double u = dz * ir, s = rho * ir, x = __ldg(rec + 1) * ir;
    double p0 = 1.0, p1 = u, d0 = 0.0, d1 = 1.0;
    double A = __ldg(rec + 2), B = 0.0;
    double xn = x;
    auto term = [&](int n, double moment) {
        const double m = moment * xn;
        A = fma((double)(n + 1) * m, p1, A);
        B = fma(m, d1, B);
        const double p2 = fma(kLegA[n] * u, p1, -kLegB[n] * p0);
        const double d2 = fma((double)(2 * n + 1), p1, d0);
        p0 = p1;
        p1 = p2;
        d0 = d1;
        d1 = d2;
        xn *= x;
    };
    // moments loaded four terms ahead of the recurrence that consumes them
    int n = 1;
    for (; n + 3 < nt; n += 4) {
        const double m0 = __ldg(rec + 2 + n), m1 = __ldg(rec + 3 + n), m2 = __ldg(rec + 4 + n),
                     m3 = __ldg(rec + 5 + n);
        term(n, m0);
        term(n + 1, m1);
        term(n + 2, m2);
        term(n + 3, m3);
    }
    for (; n < nt; ++n) term(n, __ldg(rec + 2 + n));
    const double sc = ir * ir * 0.07957747154594767;  // 1 / (4 pi r^2)
    const double e_r = A * sc, e_t = s * B * sc;
    er = e_r * s + e_t * u;
    ez = e_r * u - e_t * s;
}

constexpr int kWarpRuns = kWarpChunk / SPT_BLOCK_SEGS;
static_assert(kWarpRuns <= 32, "one lane classifies each run of a chunk");

template <int NP, int NQ, bool MIX>
__device__ bool far_adaptive_warp(Ctx& c, int r0, int np_, unsigned long long& far_evals,
                                  unsigned long long& cl_evals) {
    const SptBem& b = c.bem;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nseg = b.n_seg, nps = b.nodes_per_seg;
    double* P = c.bpt;
    int* scratch = reinterpret_cast<int*>(c.tiles) + warp * kWarpScratchInts;
    int* lists = scratch;                                                    // L0 | L1 | L2, kWarpChunk each
    unsigned char* mask = reinterpret_cast<unsigned char*>(scratch + 3 * kWarpChunk);  // near masks of L0
    int* R2 = scratch + 3 * kWarpChunk + kWarpChunk / 4;
    int* R3 = R2 + kWarpRuns;
    int* M = R3 + kWarpRuns;
    int* Mcls = M + kWarpRuns;
    unsigned* covered = reinterpret_cast<unsigned*>(Mcls + kWarpRuns);  // runs summed by cluster expansions
    double pr[NP], pinv[NP], pz[NP], ar[NP], az[NP];
    float fr[NP], fz[NP], kr[NP], kz[NP], prf[NP], pinvf[NP];
    float sa[NP];
#pragma unroll
    for (int p = 0; p < NP; ++p) {
        const int k = r0 + (p < np_ ? p : 0);
        pr[p] = P[8 * k + 3];
        pinv[p] = pr[p] > 0.0 ? 1.0 / pr[p] : 0.0;
        pz[p] = P[8 * k + 4];
        ar[p] = 0.0;
        az[p] = 0.0;
        fr[p] = fz[p] = kr[p] = kz[p] = sa[p] = 0.0f;
        prf[p] = (float)pr[p];
        pinvf[p] = (float)pinv[p];
    }
    const double r4 = b.ratio4, r2 = b.ratio2;
    const double* cr = b.coarse;
    const double* cz = b.coarse + b.coarse_stride;
    const double* cw = b.coarse + 2 * b.coarse_stride;
    const bool run_rule = b.blk && b.run_nodes && b.ratio_run > 0.0;
    const unsigned lt = (1u << lane) - 1u;
    // Cluster expansions (one point per task): lane = run; the run is covered
    // by its highest ancestor cluster that is at least kappa radii away, and
    // the lane of the cluster's first run adds that cluster's expansion.
    const int n_run = (nseg + SPT_BLOCK_SEGS - 1) / SPT_BLOCK_SEGS;
    const bool use_cl = NP == 1 && b.blk && b.clusters && b.cluster_kappa > 0.0 && n_run <= SPT_MAX_CLUSTER_RUNS;
    if (use_cl) {
        const int nt = b.cluster_terms, rec_len = nt + 2;
        // the covering clusters' heads, listed first (the segment lists are free
        // until the chunk loop) and then expanded in one lane-parallel pass
        int* const heads = lists;
        int n_heads = 0;
        for (int qb = 0; qb < n_run; qb += 32) {
            const int q = qb + lane;
            int lv = -1, idx = 0;
            if (q < n_run) {
                int off = 0;
                for (int l = 0; l < b.cluster_levels; ++l) {
                    const int i = off + (q >> l);
                    const double* rec = b.clusters + (size_t)i * rec_len;
                    const double dz = pz[0] - __ldg(rec);
                    if (pr[0] * pr[0] + dz * dz >= b.cluster_kappa * b.cluster_kappa * __ldg(rec + 1) * __ldg(rec + 1)) {
                        lv = l;
                        idx = i;
                    }
                    off += (n_run + (1 << l) - 1) >> l;
                }
            }
            const unsigned cov = __ballot_sync(0xffffffffu, lv >= 0);
            if (lane == 0) covered[qb >> 5] = cov;
            const bool head = lv >= 0 && (q & ((1 << lv) - 1)) == 0;
            const unsigned hm = __ballot_sync(0xffffffffu, head);
            if (head) heads[n_heads + __popc(hm & lt)] = idx;
            n_heads += __popc(hm);
        }
        __syncwarp();
        for (int hh = lane; hh < n_heads; hh += 32) {
            double er, ez;
            cluster_field(b.clusters + (size_t)heads[hh] * rec_len, nt, pr[0], pz[0], er, ez);
            ar[0] += er;
            az[0] += ez;
            ++cl_evals;
        }
        __syncwarp();
    }
    for (int c0 = 0; c0 < nseg; c0 += kWarpChunk) {
        const int q0 = c0 / SPT_BLOCK_SEGS;
        const int nr = min(kWarpRuns, (nseg - c0 + SPT_BLOCK_SEGS - 1) / SPT_BLOCK_SEGS);
        const int q = q0 + lane;
        int cls = -1;  // 3 run rule, 2 Gauss-2 on every segment, 1 no near segment, 0 full test
        if (lane < nr && !(use_cl && ((covered[q >> 5] >> (q & 31)) & 1u))) {
            cls = 0;
            if (b.blk) {
                double lb = INFINITY;
                for (int p = 0; p < np_; ++p) lb = fmin(lb, blk_lower(b, q, P[8 * (r0 + p) + 3], P[8 * (r0 + p) + 4]));
                const double lm = blk_lmax(b, q);
                if (run_rule && __ldg(b.blk + 5 * b.blk_stride + q) != 0.0 &&
                    lb >= b.ratio_run * __ldg(b.blk + 4 * b.blk_stride + q))
                    cls = 3;
                else if (lb >= r2 * lm) cls = 2;
                else if (lb >= r4 * lm) cls = 1;
            }
        }
        const unsigned b3 = __ballot_sync(0xffffffffu, cls == 3);
        const unsigned b2 = __ballot_sync(0xffffffffu, cls == 2);
        const unsigned bm = __ballot_sync(0xffffffffu, cls == 0 || cls == 1);
        if (cls == 3) R3[__popc(b3 & lt)] = q;
        if (cls == 2) R2[__popc(b2 & lt)] = q;
        if (cls == 0 || cls == 1) { M[__popc(bm & lt)] = q; Mcls[__popc(bm & lt)] = cls; }
        const int nR2 = __popc(b2), nR3 = __popc(b3), nm = __popc(bm);
        __syncwarp();
        // segment classification of the M runs, one run at a time (lane = segment)
        int n0 = 0, n1 = 0, n2 = 0;
        for (int mi = 0; mi < nm; ++mi) {
            const int sg = M[mi] * SPT_BLOCK_SEGS + lane;
            int lvl = 3;
            unsigned m = 0;
            if (sg < nseg) {
                const int mc = Mcls[mi];
                const double L = segf(b, 4, sg);
                double dmin = INFINITY;
                for (int p = 0; p < np_; ++p) {
                    double proj, dist;
                    if (seg_near(b, sg, P[8 * (r0 + p) + 3], P[8 * (r0 + p) + 4], proj, dist)) m |= 1u << p;
                    dmin = fmin(dmin, dist);
                }
                if (mc == 1) m = 0, lvl = dmin < r2 * L ? 1 : 2;
                else lvl = dmin < r4 * L ? 0 : (dmin < r2 * L ? 1 : 2);
            }
            const unsigned v0 = __ballot_sync(0xffffffffu, lvl == 0);
            const unsigned v1 = __ballot_sync(0xffffffffu, lvl == 1);
            const unsigned v2 = __ballot_sync(0xffffffffu, lvl == 2);
            if (lvl == 0) {
                const int pos = n0 + __popc(v0 & lt);
                lists[pos] = sg;
                mask[pos] = (unsigned char)m;
            } else if (lvl == 1) {
                lists[kWarpChunk + n1 + __popc(v1 & lt)] = sg;
            } else if (lvl == 2) {
                lists[2 * kWarpChunk + n2 + __popc(v2 & lt)] = sg;
            }
            n0 += __popc(v0);
            n1 += __popc(v1);
            n2 += __popc(v2);
        }
        __syncwarp();
        const int e0 = n0 * nps, e1 = e0 + 4 * n1, e2 = e1 + 2 * n2;
        const int e3 = e2 + 2 * SPT_BLOCK_SEGS * nR2, e4 = e3 + SPT_RUN_NODES * nR3;
        for (int q0i = lane; q0i < e4; q0i += 32 * NQ) {
            double rq[NQ], zq[NQ], wq[NQ];
            unsigned mk[NQ];
            bool in[NQ];
#pragma unroll
            for (int j = 0; j < NQ; ++j) {
                const int qq = q0i + j * 32;
                in[j] = qq < e4;
                size_t src = 0;
                const double *tr = cr, *tz = cz, *tw = cw;
                mk[j] = 0;
                if (!in[j]) {
                    // padding lane: any valid node, not accumulated
                } else if (qq < e0) {
                    const int li = qq / nps;
                    src = (size_t)lists[li] * nps + (qq - li * nps);
                    tr = b.node;
                    tz = b.node + b.node_stride;
                    tw = b.node + 2 * b.node_stride;
                    mk[j] = mask[li];
                } else if (qq < e1) {
                    const int i = qq - e0;
                    src = (size_t)lists[kWarpChunk + (i >> 2)] * 6 + (i & 3);
                } else if (qq < e2) {
                    const int i = qq - e1;
                    src = (size_t)lists[2 * kWarpChunk + (i >> 1)] * 6 + 4 + (i & 1);
                } else if (qq < e3) {
                    const int i = qq - e2;
                    const int sgi = R2[i / (2 * SPT_BLOCK_SEGS)] * SPT_BLOCK_SEGS + ((i & (2 * SPT_BLOCK_SEGS - 1)) >> 1);
                    if (sgi < nseg) src = (size_t)sgi * 6 + 4 + (i & 1);
                    else in[j] = false;  // past the last segment of a short final run
                } else {
                    const int i = qq - e3;
                    src = (size_t)R3[i / SPT_RUN_NODES] * SPT_RUN_NODES + (i % SPT_RUN_NODES);
                    tr = b.run_nodes;
                    tz = b.run_nodes + b.run_stride;
                    tw = b.run_nodes + 2 * b.run_stride;
                }
                rq[j] = __ldg(tr + src);
                zq[j] = __ldg(tz + src);
                wq[j] = __ldg(tw + src);
            }
#pragma unroll
            for (int p = 0; p < NP; ++p) {
#pragma unroll
                for (int j = 0; j < NQ; ++j) {
                    if (p < np_ && in[j] && !((mk[j] >> p) & 1u)) {
                        const double dz = pz[p] - zq[j];
                        if (MIX) {
                            float er, ez;
                            if (ring_far_f(prf[p], pinvf[p], (float)(pr[p] - rq[j]), (float)(pr[p] + rq[j]), (float)dz,
                                           (float)rq[j], er, ez)) {
                                const float w = (float)wq[j];
                                kahan_add(fr[p], kr[p], w * er);
                                kahan_add(fz[p], kz[p], w * ez);
                                sa[p] += fabsf(w * er) + fabsf(w * ez);
                            } else {
                                // close to the ring: the term in float64, summed like the others
                                double e64r, e64z;
                                ring_field_far_cold(pr[p], 1.0 / pr[p], dz, rq[j], e64r, e64z);
                                const float ter = (float)(wq[j] * e64r), tez = (float)(wq[j] * e64z);
                                kahan_add(fr[p], kr[p], ter);
                                kahan_add(fz[p], kz[p], tez);
                                sa[p] += fabsf(ter) + fabsf(tez);
                            }
                        } else {
                            double er, ez;
                            ring_field_far(pr[p], pinv[p], dz, rq[j], er, ez);
                            ar[p] = fma(wq[j], er, ar[p]);
                            az[p] = fma(wq[j], ez, az[p]);
                        }
                        ++far_evals;
                    }
                }
            }
        }
        __syncwarp();  // the lists are rewritten by the next chunk
    }
    // fixed-order warp reduction; lane 0 writes the round's fields
    bool redo = false;
#pragma unroll
    for (int p = 0; p < NP; ++p) {
        if (MIX) {
            ar[p] += (double)fr[p] - (double)kr[p];
            az[p] += (double)fz[p] - (double)kz[p];
        }
        const double vr = warp_sum(ar[p]);
        const double vz = warp_sum(az[p]);
        const double va = MIX ? warp_sum((double)sa[p]) : 0.0;
        if (lane == 0 && p < np_) {
            const int k = r0 + p;
            const double er = vr + P[8 * k + 7], ez = vz + c.fld[3 * k + 2];
            P[8 * k + 5] = er;
            P[8 * k + 6] = ez;
            if (MIX) {
                const double tz = ez + c.g.E_gun;
                if (!(va <= c.kappa * sqrt(er * er + tz * tz))) redo = true;
            }
        }
    }
    return __shfl_sync(0xffffffffu, redo, 0);
}

// ---------------------------------------------------------------------------
// BEM field of a list of points, in phases.  Records live in c.bpt (8 doubles
// each: x, y, z, rho_e, z_e, then results); every phase is called by all
// threads of the CTA.

// A: closest segment and on-surface offset of records [0, n).  With `frame`,
// also the closest segment, its parameter t and the distance, for the
// surrogate's inputs.
// One warp, record k.
__device__ __forceinline__ void closest_point(Ctx& c, int k, bool frame) {
    const SptBem& b = c.bem;
    const int lane = threadIdx.x & 31;
    double* P = c.bpt;  // record k: [0]x [1]y [2]z [3]rho_e [4]z_e [5]ax [6]ay [7]near_r ; near_z in fld tmp
    const int nseg = b.n_seg;
    {
        const double x = P[8 * k + 0], y = P[8 * k + 1], z = P[8 * k + 2];
        const double rho = hypot(x, y);
        double best = INFINITY;
        int bs = 0x7fffffff;
        if (b.blk) {
            // the run with the smallest lower bound gives an upper bound of the
            // minimum; only runs whose lower bound does not exceed it are scanned
            // (each lane still takes its segments in increasing order)
            const int nblk = (nseg + SPT_BLOCK_SEGS - 1) / SPT_BLOCK_SEGS;
            double lbm = INFINITY, lmx = 0.0;
            int qm = 0;
            for (int q = lane; q < nblk; q += 32) {
                const double lb = blk_lower(b, q, rho, z);
                if (lb < lbm) { lbm = lb; qm = q; }
                lmx = fmax(lmx, blk_lmax(b, q));
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double ol = __shfl_xor_sync(0xffffffffu, lbm, o);
                const int oq = __shfl_xor_sync(0xffffffffu, qm, o);
                if (ol < lbm || (ol == lbm && oq < qm)) { lbm = ol; qm = oq; }
                lmx = fmax(lmx, __shfl_xor_sync(0xffffffffu, lmx, o));
            }
            // Every segment at least 2e-9 x the longest segment away (the run
            // bounds are rigorous lower bounds): the on-surface offset below
            // (distance^2 < (1e-9 L)^2) cannot apply, the closest segment
            // plays no further part, and the evaluation point is the point
            // itself -- the offset path's rho + 0 and z + 0 bit for bit (z = 0
            // excepted: there the sign of the zero would follow the normal).
            if (!frame && z != 0.0 && lbm > 2e-9 * lmx) {
                if (lane == 0) {
                    P[8 * k + 3] = rho;
                    P[8 * k + 4] = z;
                }
                return;
            }
            double ub = INFINITY;
            if (qm * SPT_BLOCK_SEGS + lane < nseg) ub = seg_dist2(b, qm * SPT_BLOCK_SEGS + lane, rho, z);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) ub = fmin(ub, __shfl_xor_sync(0xffffffffu, ub, o));
            const double ubd = sqrt(ub);
            for (int q0 = 0; q0 < nblk; q0 += 32) {
                const bool cand = q0 + lane < nblk && !(blk_lower(b, q0 + lane, rho, z) > ubd);
                unsigned cm = __ballot_sync(0xffffffffu, cand);
                while (cm) {
                    const int j = __ffs(cm) - 1;
                    cm &= cm - 1;
                    const int s = (q0 + j) * SPT_BLOCK_SEGS + lane;
                    if (s < nseg) {
                        const double d2 = seg_dist2(b, s, rho, z);
                        if (d2 < best) { best = d2; bs = s; }
                    }
                }
            }
        } else {
            for (int s = lane; s < nseg; s += 32) {
                const double d2 = seg_dist2(b, s, rho, z);
                if (d2 < best) { best = d2; bs = s; }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ob = __shfl_xor_sync(0xffffffffu, best, o);
            const int os = __shfl_xor_sync(0xffffffffu, bs, o);
            if (ob < best || (ob == best && os < bs)) { best = ob; bs = os; }
        }
        if (lane == 0) {
            if (bs >= nseg) bs = 0;  // every distance was NaN: the reference keeps index 0
            const double Ls = segf(b, 4, bs);
            const double thr = __dmul_rn(1e-9, Ls);
            const double off = (best < __dmul_rn(thr, thr)) ? __dmul_rn(1e-4, Ls) : 0.0;
            double re = __dadd_rn(rho, __dmul_rn(off, segf(b, 7, bs)));
            if (rho == 0.0) re = 0.0;
            P[8 * k + 3] = re;
            P[8 * k + 4] = __dadd_rn(z, __dmul_rn(off, segf(b, 8, bs)));
            if (frame) {
                const double p0x = segf(b, 0, bs), p0y = segf(b, 1, bs), ax = segf(b, 2, bs), ay = segf(b, 3, bs);
                double tt = ((rho - p0x) * ax + (z - p0y) * ay) / (ax * ax + ay * ay);
                c.sseg[k] = bs;
                c.st[k] = fmin(fmax(tt, 0.0), 1.0);
                c.sd[k] = sqrt(best);
            }
        }
    }
}

static __device__ void bem_closest(Ctx& c, int n, bool frame) {
    // one warp per point
    for (int k = threadIdx.x >> 5; k < n; k += c.nw) closest_point(c, k, frame);
    __syncthreads();
}


// B for one record k, by one warp: the near-segment sinh quadrature
// (bem/axisymmetric.py:566-600); lane 0 ends with near_r in record slot 7 and
// near_z in fld[3k + 2].
__device__ __forceinline__ void near_point(Ctx& c, int k, unsigned long long& n_near, unsigned long long& n_ring_near) {
    const SptBem& b = c.bem;
    const int lane = threadIdx.x & 31;
    double* P = c.bpt;
    const int nseg = b.n_seg;
    {
        const double re = P[8 * k + 3], ze = P[8 * k + 4];
        double acc_r = 0.0, acc_z = 0.0;
        const int nblk = (nseg + SPT_BLOCK_SEGS - 1) / SPT_BLOCK_SEGS;
        for (int q0 = 0; q0 < nblk; q0 += 32) {
          // runs that may hold a near segment (every run without the bounds table)
          const bool cand = q0 + lane < nblk && !(b.blk && blk_lower(b, q0 + lane, re, ze) >= blk_lmax(b, q0 + lane));
          unsigned cm = __ballot_sync(0xffffffffu, cand);
          while (cm) {
            const int jq = __ffs(cm) - 1;
            cm &= cm - 1;
            const int s0 = (q0 + jq) * SPT_BLOCK_SEGS;
            const int s = s0 + lane;
            double proj = 0.0, dist = 0.0;
            const bool nr = (s < nseg) && seg_near(b, s, re, ze, proj, dist);
            unsigned mask = __ballot_sync(0xffffffffu, nr);
            while (mask) {
                const int j = __ffs(mask) - 1;
                mask &= mask - 1;
                const int sg = s0 + j;
                const double sp = __shfl_sync(0xffffffffu, proj, j);
                const double Ls = segf(b, 4, sg);
                const double d = fmax(__shfl_sync(0xffffffffu, dist, j), 1e-15 * Ls);
                const double lo = asinh(-sp / d), hi = asinh((Ls - sp) / d);
                const int cnt = max(1, (int)ceil((hi - lo) / 0.5));
                const double width = (hi - lo) / cnt;
                const double half = 0.5 * (hi - lo) / cnt;
                const double p0r = segf(b, 0, sg), p0z = segf(b, 1, sg), ur = segf(b, 5, sg), uz = segf(b, 6, sg);
                const double sg0 = segf(b, 9, sg), sg1 = segf(b, 10, sg);
                for (int qn = lane; qn < cnt * 8; qn += 32) {
                    const int iv = qn >> 3, gi = qn & 7;
                    const double v = lo + (iv + 0.5 * (b.gauss8_x[gi] + 1.0)) * width;
                    const double sl = sp + d * sinh(v);
                    const double sr = p0r + sl * ur, sz = p0z + sl * uz;
                    const double dens = sg0 + (sl / Ls) * (sg1 - sg0);
                    const double w = dens * (2.0 * kPi * sr) * d * cosh(v) * half * b.gauss8_w[gi];
                    double er, ez;
                    ring_field(re, ze - sz, sr, er, ez);
                    acc_r += w * er;
                    acc_z += w * ez;
                }
                if (lane == 0) { n_near += 1; n_ring_near += (unsigned long long)cnt * 8; }
            }
          }
        }
        acc_r = warp_sum(acc_r);
        acc_z = warp_sum(acc_z);
        if (lane == 0) {
            P[8 * k + 7] = acc_r;
            c.fld[3 * k + 2] = acc_z;  // temporary near_z (fld is rewritten after the far sum)
        }
    }
}

// Adaptive far rule for record k, by this warp: float32 first in the mixed
// form, float64 again when its sum is ill-conditioned.  The float64 tile is
// the float64 form's, so with every sum redone the mixed form reproduces it.
// Ring evaluations each lane keeps in flight in the float64 adaptive far sum.
// One: every in-flight evaluation is an inlined copy of the ring kernel, and
// the trace kernel is bound by instruction fetch, not by the latency the
// copies would hide (whole C1 traces, 1184 groups: 8 in flight 8.9 M, 4 in
// flight 12.1 M, 2 in flight 15.4 M, 1 in flight 18.3 M particle-steps/s).
#ifndef SPT_FAR_NQ_FP64
#define SPT_FAR_NQ_FP64 1
#endif

template <int FORM>
__device__ __forceinline__ void far_point(Ctx& c, int k, unsigned long long& fe, unsigned long long& ce) {
    if constexpr (FORM == SPT_FORM_FP64) {
        far_adaptive_warp<1, SPT_FAR_NQ_FP64, false>(c, k, 1, fe, ce);
    } else {
        // float32 tiles keep 4 ring evaluations in flight per lane (8 spill at
        // 128 registers; more resident warps supply the parallelism instead)
        if (far_adaptive_warp<1, 4, true>(c, k, 1, fe, ce)) {
            if ((threadIdx.x & 31) == 0) atomicAdd(c.cnt + SPT_CNT_FP64_ROUNDS, 1ull);
            far_adaptive_warp<1, 8, false>(c, k, 1, fe, ce);
        }
    }
}

// Next record for this warp from the CTA's task counter (dynamic assignment:
// points near the surface cost many times more than distant ones).
__device__ __forceinline__ int next_task(int* counter) {
    int k = 0;
    if ((threadIdx.x & 31) == 0) k = atomicAdd(counter, 1);
    return __shfl_sync(0xffffffffu, k, 0);
}

// B + C: exact BEM field (E_rho, E_z into record slots 5, 6) of records [0, n)
// whose slots 3, 4 hold the evaluation point.  FORM: SPT_FORM_FP64 sums in
// float64; the other forms sum in float32 first and redo an ill-conditioned
// sum in float64.
template <int FORM, int FAR>
__device__ __forceinline__ void bem_sums(Ctx& c, int n, int* status_flag) {
    const SptBem& b = c.bem;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double* P = c.bpt;
    const int nseg = b.n_seg;
    const int nps = b.nodes_per_seg;
    if (n <= 0) return;
    // B: near-segment sinh quadrature (one warp per point)
    unsigned long long n_near = 0, n_ring_near = 0;
    for (int k = warp; k < n; k += c.nw) near_point(c, k, n_near, n_ring_near);
    count_add(c, SPT_CNT_NEAR_PAIRS, n_near);
    count_add(c, SPT_CNT_RING_NEAR, n_ring_near);
    __syncthreads();

    // C: far sum.  Adaptive rule: rounds of up to c.round_pts points, each
    // owned by one warp (as many rounds as warps where the points allow, so
    // no warp waits for another until the end).  Reference rule: rounds over
    // TMA-staged node tiles shared by the whole CTA; the round's point count
    // selects how many nodes each thread keeps in flight.
    unsigned long long far_evals = 0;
    bool ok = true;
    if constexpr (FAR == SPT_FAR_ADAPTIVE) {
        // one point per warp task, taken dynamically
        __shared__ int s_far_task;
        if (tid == 0) s_far_task = c.nw;
        __syncthreads();
        unsigned long long cl_evals = 0;
        for (int k = warp; k < n; k = next_task(&s_far_task)) far_point<FORM>(c, k, far_evals, cl_evals);
        count_add(c, SPT_CNT_CLUSTER_EVALS, cl_evals);
        __syncthreads();
    } else {
        const int tile_cap = c.L.tile_cap;
        const int segs_per_tile = min(tile_cap / nps, 256);
        const int n_tiles = (nseg + segs_per_tile - 1) / segs_per_tile;
        for (int r0 = 0; r0 < n; r0 += c.round_pts) {
            const int np_ = min(c.round_pts, n - r0);
            if constexpr (FORM == SPT_FORM_FP64) {
                if (np_ == 1) far_round<1, 8, false>(c, r0, np_, n_tiles, segs_per_tile, ok, far_evals);
                else if (np_ == 2) far_round<2, 4, false>(c, r0, np_, n_tiles, segs_per_tile, ok, far_evals);
                else far_round<4, 2, false>(c, r0, np_, n_tiles, segs_per_tile, ok, far_evals);
            } else {
                // mixed form (and the exact sums of the learned form): float32 first,
                // float64 again for a round whose float32 sums are ill-conditioned
                if (np_ == 1) far_round<1, 4, true>(c, r0, np_, n_tiles, segs_per_tile, ok, far_evals);
                else if (np_ == 2) far_round<2, 2, true>(c, r0, np_, n_tiles, segs_per_tile, ok, far_evals);
                else far_round<4, 1, true>(c, r0, np_, n_tiles, segs_per_tile, ok, far_evals);
                const bool redo = *c.redo != 0;
                // every thread has read the flag before the next round's float32 pass resets it
                __syncthreads();
                if (redo) {
                    if (tid == 0) atomicAdd(c.cnt + SPT_CNT_FP64_ROUNDS, 1ull);
                    // the tile shape the float64 form takes for this round size (same sums, bit for bit)
                    if (np_ == 1) far_round<1, 8, false>(c, r0, np_, n_tiles, segs_per_tile, ok, far_evals);
                    else if (np_ == 2) far_round<2, 4, false>(c, r0, np_, n_tiles, segs_per_tile, ok, far_evals);
                    else far_round<4, 2, false>(c, r0, np_, n_tiles, segs_per_tile, ok, far_evals);
                }
            }
        }
    }
    if (!ok && tid == 0) *status_flag = SPT_GROUP_TIMEOUT;
    count_add(c, SPT_CNT_RING_FAR, far_evals);
}

// D: rotate E_rho of records [0, n) into (x, y) (record slots 5, 6, 7 = ex, ey, ez)
static __device__ void bem_rotate(Ctx& c, int n, bool scatter) {
    const int tid = threadIdx.x;
    double* P = c.bpt;
    for (int k = tid; k < n; k += c.nt) {
        const double x = P[8 * k + 0], y = P[8 * k + 1];
        const double rho = hypot(x, y);
        const double e_rho = P[8 * k + 5], e_z = P[8 * k + 6];
        double ex = 0.0, ey = 0.0;
        if (rho != 0.0) {
            ex = e_rho * (x / rho);
            ey = e_rho * (y / rho);
        }
        if (scatter) {
            const int i = c.list[k];
            c.fld[3 * i + 0] = ex;
            c.fld[3 * i + 1] = ey;
            c.fld[3 * i + 2] = e_z;
        } else {
            P[8 * k + 5] = ex;
            P[8 * k + 6] = ey;
            P[8 * k + 7] = e_z;
        }
    }
    __syncthreads();
}


// ---------------------------------------------------------------------------
// learned form: the MLP surrogate evaluated on the tensor cores inside the
// stage (parameter offsets in the flat parameter array)
constexpr int kOW1 = 0, kOB1 = 256, kOW2 = 384, kOB2 = 16768, kOW3 = 16896, kOB3 = 33280, kOW4 = 33408, kOB4 = 49792,
              kOW5 = 49920, kOB5 = 50176;

// Surrogate field (E_rho, E_z) of records [0, n) into c.sout, from the
// closest-point frame bem_closest(c, n, true) left in sseg/st/sd.  Rows are
// processed 128 at a time: features and the first layer on the CUDA cores
// into a BF16 activation tile, three 128 x 128 layers as tcgen05.mma (K = 16
// steps) into the CTA's TMEM accumulator with the weights streamed into a
// BF16 tile, bias + SiLU applied while reading TMEM back, the last layer on
// the CUDA cores, then rescaling and rotation from the (normal, tangent)
// frame of the closest segment.
static __device__ void mlp_points(Ctx& c, int n, int* status_flag) {
    const SptBem& b = c.bem;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const float* W = c.sw;
    const double lmin = log(c.dmin), lspan = log(c.dmax) - lmin;
    for (int cs = 0; cs < n; cs += 128) {
        const int m = min(128, n - cs);
        if (tid < 128) {
            float u1 = 0.f, u2 = 0.f;
            if (tid < m) {
                const int k = cs + tid;
                const int sg = c.sseg[k];
                const double sarc = (c.s_start[sg] + c.st[k] * segf(b, 4, sg)) / c.s_end;
                const double ld = log(fmin(fmax(c.sd[k], c.dmin), c.dmax));
                u1 = (float)(2.0 * (ld - lmin) / lspan - 1.0);
                u2 = (float)(2.0 * sarc - 1.0);
            }
            c.feat[2 * tid] = u1;
            c.feat[2 * tid + 1] = u2;
        }
        __syncthreads();
        for (int idx = tid; idx < 128 * 128; idx += c.nt) {
            const int r = idx >> 7, j = idx & 127;
            float h = 0.f;
            if (r < m) {
                const float v = fmaf(W[kOW1 + 2 * j], c.feat[2 * r], fmaf(W[kOW1 + 2 * j + 1], c.feat[2 * r + 1], W[kOB1 + j]));
                h = spt_umma::silu(v);
            }
            *reinterpret_cast<__nv_bfloat16*>(c.act + spt_umma::kmajor128(r, j)) = __float2bfloat16_rn(h);
        }
        for (int l = 0; l < 3; ++l) {
            const int ow = l == 0 ? kOW2 : (l == 1 ? kOW3 : kOW4);
            const int ob = l == 0 ? kOB2 : (l == 1 ? kOB3 : kOB4);
            // weights as the B operand: element (n = out, k = in) at W16[ow + n*128 + k], K-major
            for (int v = tid; v < 2048; v += c.nt) {
                const int nrow = v >> 4, kg = v & 15;
                const uint4 val = *reinterpret_cast<const uint4*>(c.sw16 + ow + nrow * 128 + kg * 8);
                *reinterpret_cast<uint4*>(c.wt + ((nrow >> 3) * 16 + kg) * 128 + (nrow & 7) * 16) = val;
            }
            spt_umma::fence_proxy();
            __syncthreads();
            if (tid == 0) {
                spt_umma::fence_after();
                const uint32_t idesc = spt_umma::idesc_bf16_128(0, 0);
#pragma unroll
                for (int kk = 0; kk < 8; ++kk)
                    spt_umma::mma(c.tmem, spt_umma::desc(c.act + kk * 256, 128, 2048),
                                  spt_umma::desc(c.wt + kk * 256, 128, 2048), idesc, kk > 0 ? 1u : 0u);
                spt_umma::commit(&c.bars[2]);
            }
            const bool ok = mbar_wait(&c.bars[2], c.phase[2]);
            c.phase[2] ^= 1u;
            if (!ok && tid == 0) *status_flag = SPT_GROUP_TIMEOUT;
            spt_umma::fence_after();
            // epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31 (rows); with 8 warps
            // columns 64 (w / 4) .. +63, with 4 warps all 128 columns
            const int row = 32 * (warp & 3) + lane;
            for (int cb = 64 * (warp >> 2); cb < 128; cb += 64 * (c.nw >> 2))
#pragma unroll
            for (int c0 = 0; c0 < 64; c0 += 16) {
                float v[16];
                spt_umma::ld16(c.tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(cb + c0), v);
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const int col = cb + c0 + i;
                    const float h = spt_umma::silu(v[i] + W[ob + col]);
                    *reinterpret_cast<__nv_bfloat16*>(c.act + spt_umma::kmajor128(row, col)) = __float2bfloat16_rn(h);
                }
            }
            spt_umma::fence_before();
            spt_umma::fence_proxy();
            __syncthreads();
        }
        // last layer, rescaling and rotation: one warp per row
        for (int r = warp; r < m; r += c.nw) {
            float a0 = 0.f, a1 = 0.f;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int j = lane + 32 * q;
                const float h = __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(c.act + spt_umma::kmajor128(r, j)));
                a0 = fmaf(W[kOW5 + j], h, a0);
                a1 = fmaf(W[kOW5 + 128 + j], h, a1);
            }
            a0 = warp_sum(a0);
            a1 = warp_sum(a1);
            if (lane == 0) {
                const int k = cs + r;
                const int sg = c.sseg[k];
                const double t = c.st[k];
                const double sig = fabs(segf(b, 9, sg) + t * (segf(b, 10, sg) - segf(b, 9, sg))) + c.sig_floor;
                const double pos = (log(fmin(fmax(c.sd[k], c.dmin), c.dmax)) - lmin) / lspan * 63.0;
                const int i0 = min(62, max(0, (int)floor(pos)));
                const double fr = fmin(fmax(pos - i0, 0.0), 1.0);
                const double g = exp(c.log_scale[i0] + fr * (c.log_scale[i0 + 1] - c.log_scale[i0]));
                const double en = ((double)a0 + (double)W[kOB5]) * sig * g;
                const double et = ((double)a1 + (double)W[kOB5 + 1]) * sig * g;
                c.sout[2 * k] = en * segf(b, 7, sg) + et * segf(b, 5, sg);
                c.sout[2 * k + 1] = en * segf(b, 8, sg) + et * segf(b, 6, sg);
            }
        }
        __syncthreads();
    }
}

__device__ __forceinline__ bool spot_pick(uint32_t key, int particle, double frac) {
    uint32_t h = key * 0x9E3779B1u ^ (uint32_t)particle * 0x85EBCA77u;
    h ^= h >> 15;
    h *= 0x2C1B3C6Du;
    h ^= h >> 12;
    return (double)(h & 0xFFFFu) < frac * 65536.0;
}

// BEM field of the listed points in the learned form: the surrogate for
// every point, the exact sum for points within the band and for the spot
// checks (stable partition: exact records first), surrogate error of the
// spot checks recorded, then the rotation of phase D.
template <int FAR>
__device__ void surrogate_points(Ctx& c, int n, int* status_flag) {
    const int tid = threadIdx.x;
    double* P = c.bpt;
    __shared__ int s_cnt[kMaxWarps + 1];
    __shared__ int s_tot[2];
    bem_closest(c, n, true);
    mlp_points(c, n, status_flag);
    // stable partition of records [0, n): exact (band or spot) first.  The
    // destination of every record is found first (kept in sseg, which the
    // MLP no longer needs), then the records move through the act/wt scratch
    // (8 doubles each: slots 0-4 of the record, the surrogate E_rho, E_z, and
    // the list entry, negated minus one when the point lies in the band).
    if (tid == 0) s_tot[0] = 0;
    __syncthreads();
    for (int base = 0; base < n; base += c.nt) {
        const int k = base + tid;
        const bool ex = k < n && (c.sd[k] < c.band || spot_pick(c.key, c.list[k], c.spot));
        const unsigned bal = __ballot_sync(0xffffffffu, ex);
        if ((tid & 31) == 0 && bal) atomicAdd(&s_tot[0], __popc(bal));
    }
    __syncthreads();
    const int ne = s_tot[0];
    int run_ex = 0, run_su = 0;
    for (int base = 0; base < n; base += c.nt) {
        const int k = base + tid;
        const bool valid = k < n;
        const bool band = valid && c.sd[k] < c.band;
        const bool ex = valid && (band || spot_pick(c.key, c.list[k], c.spot));
        const unsigned be = __ballot_sync(0xffffffffu, ex);
        if ((tid & 31) == 0) s_cnt[tid >> 5] = __popc(be);
        __syncthreads();
        int pre_e = 0, tot_e = 0;
        for (int w = 0; w < c.nw; ++w) {
            if (w < (tid >> 5)) pre_e += s_cnt[w];
            tot_e += s_cnt[w];
        }
        const int chunk = min(c.nt, n - base);
        const int before = min((tid >> 5) * 32, chunk);  // records of this chunk before this warp
        const unsigned lt = (1u << (tid & 31)) - 1u;
        if (valid) {
            const int lane_e = __popc(be & lt);
            const int dst = ex ? run_ex + pre_e + lane_e : ne + run_su + (before - pre_e) + ((tid & 31) - lane_e);
            c.sseg[k] = 2 * dst + (band ? 1 : 0);
        }
        run_ex += tot_e;
        run_su += chunk - tot_e;
        __syncthreads();
    }
    double* tmp = reinterpret_cast<double*>(c.act);  // act + wt: 8192 doubles >= 8 n
    for (int k = tid; k < n; k += c.nt) {
        const int code = c.sseg[k];
        const int d = code >> 1;
        for (int f = 0; f < 5; ++f) tmp[8 * d + f] = P[8 * k + f];
        tmp[8 * d + 5] = c.sout[2 * k];
        tmp[8 * d + 6] = c.sout[2 * k + 1];
        tmp[8 * d + 7] = (code & 1) ? -(double)c.list[k] - 1.0 : (double)c.list[k];
    }
    __syncthreads();
    for (int k = tid; k < n; k += c.nt) {
        for (int f = 0; f < 5; ++f) P[8 * k + f] = tmp[8 * k + f];
        c.sout[2 * k] = tmp[8 * k + 5];
        c.sout[2 * k + 1] = tmp[8 * k + 6];
        const double v = tmp[8 * k + 7];
        c.list[k] = v < 0.0 ? (int)(-v - 1.0) : (int)v;
        c.fld[3 * k] = v < 0.0 ? 1.0 : 0.0;  // band flag, kept where the sums do not write
    }
    __syncthreads();
    bem_sums<SPT_FORM_SURROGATE, FAR>(c, ne, status_flag);
    unsigned long long n_spot = 0, n_band = 0;
    for (int k = tid; k < n; k += c.nt) {
        if (k >= ne) {
            P[8 * k + 5] = c.sout[2 * k];
            P[8 * k + 6] = c.sout[2 * k + 1];
        } else if (c.fld[3 * k] == 0.0) {  // a spot check: exact and surrogate both known
            // error relative to the whole external field there (uniform + perturbation)
            const double er = P[8 * k + 5], ez = P[8 * k + 6];
            const double dr = c.sout[2 * k] - er, dz = c.sout[2 * k + 1] - ez;
            const double tz = ez + c.g.E_gun;
            const float rel = (float)(sqrt(dr * dr + dz * dz) / fmax(sqrt(er * er + tz * tz), 1e-300));
            if (c.sstats) atomicMax(reinterpret_cast<unsigned int*>(c.sstats) + 6, __float_as_uint(rel));
            ++n_spot;
        } else {
            ++n_band;
        }
    }
    if (c.sstats) {
        const unsigned long long nsur = (unsigned long long)(n - ne);
        if (tid == 0 && nsur) atomicAdd(c.sstats + 0, nsur);
        n_band = warp_sum(n_band);
        n_spot = warp_sum(n_spot);
        if ((tid & 31) == 0) {
            if (n_band) atomicAdd(c.sstats + 1, n_band);
            if (n_spot) atomicAdd(c.sstats + 2, n_spot);
        }
    }
    __syncthreads();
    bem_rotate(c, n, false);
}

// BEM field of the n points listed in c.bpt (x, y, z at slots 0..2 of each
// 8-double record): the reference's evaluation, phases A-D.
// BEM field of the records [0, n) with the adaptive far rule, each point one
// warp task from start to end -- closest segment and on-surface offset, near
// quadrature, far sum, rotation -- taken dynamically from a CTA counter, so
// the only barrier is the one at the end.  Same arithmetic as the phased
// path (bem_closest, bem_sums, bem_rotate).
template <int FORM>
__device__ void bem_points_fused(Ctx& c, int n) {
    const int lane = threadIdx.x & 31;
    double* P = c.bpt;
    __shared__ int s_task;
    if (threadIdx.x == 0) s_task = c.nw;
    __syncthreads();
    unsigned long long n_near = 0, n_ring_near = 0, far_evals = 0, cl_evals = 0;
    for (int k = threadIdx.x >> 5; k < n; k = next_task(&s_task)) {
        closest_point(c, k, false);
        __syncwarp();
        near_point(c, k, n_near, n_ring_near);
        __syncwarp();
        far_point<FORM>(c, k, far_evals, cl_evals);
        if (lane == 0) {
            const double x = P[8 * k + 0], y = P[8 * k + 1];
            const double rho = hypot(x, y);
            const double e_rho = P[8 * k + 5], e_z = P[8 * k + 6];
            double ex = 0.0, ey = 0.0;
            if (rho != 0.0) {
                ex = e_rho * (x / rho);
                ey = e_rho * (y / rho);
            }
            P[8 * k + 5] = ex;
            P[8 * k + 6] = ey;
            P[8 * k + 7] = e_z;
        }
        __syncwarp();
    }
    count_add(c, SPT_CNT_NEAR_PAIRS, n_near);
    count_add(c, SPT_CNT_RING_NEAR, n_ring_near);
    count_add(c, SPT_CNT_RING_FAR, far_evals);
    count_add(c, SPT_CNT_CLUSTER_EVALS, cl_evals);
    __syncthreads();
}

template <int FORM, int FAR>
__device__ void bem_points(Ctx& c, int n, bool scatter, int* status_flag) {
    if constexpr (FAR == SPT_FAR_ADAPTIVE) {
        if (!scatter) {
            bem_points_fused<FORM>(c, n);
            return;
        }
    }
    bem_closest(c, n, false);
    bem_sums<FORM, FAR>(c, n, status_flag);
    bem_rotate(c, n, scatter);
}

// Softened pair sum over the live sources of the group (forces.py:16-29):
// sum_j k q_i q_j (r_i - r_j) / (|r_i - r_j|^2 + a^2)^1.5, sources given by
// src(j, x, y, z, q).  float64: the reference's operation order.  Mixed
// form: separations are taken in float64 (nearby particles far from the
// origin), then the rest in float32 with Kahan-compensated sums.
template <bool MIX, typename SRC>
__device__ __forceinline__ void pair_sum(const Ctx& c, int E, int j0, int jstep, double xi, double yi, double zi,
                                         double qk, SRC src, double& fx, double& fy, double& fz,
                                         double* sabs = nullptr) {
    // sources j0, j0 + jstep, ... (the callers split one target's sources over
    // the lanes of a warp and add the partial sums)
    if (!MIX) {
        double ax = 0.0, ay = 0.0, az = 0.0;
        for (int j = j0; j < E; j += jstep) {
            if (!c.live[j]) continue;
            double x, y, z, q;
            src(j, x, y, z, q);
            const double dx = xi - x, dy = yi - y, dz = zi - z;
            const double r2 = (dx * dx + dy * dy) + dz * dz + c.soft2;
            const double r3 = r2 * sqrt(r2);
            const double cf = qk * q / r3;
            ax = fma(cf, dx, ax);
            ay = fma(cf, dy, ay);
            az = fma(cf, dz, az);
        }
        fx = ax; fy = ay; fz = az;
    } else {
        float ax = 0.f, ay = 0.f, az = 0.f, cx = 0.f, cy = 0.f, cz = 0.f, sa = 0.f;
        const float soft2 = (float)c.soft2;
        for (int j = j0; j < E; j += jstep) {
            if (!c.live[j]) continue;
            double x, y, z, q;
            src(j, x, y, z, q);
            const float dx = (float)(xi - x), dy = (float)(yi - y), dz = (float)(zi - z);
            const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, soft2)));
            const float rs = rsqrtf(r2);
            const float cf = (float)(qk * q) * (rs * rs * rs);
            kahan_add(ax, cx, cf * dx);
            kahan_add(ay, cy, cf * dy);
            kahan_add(az, cz, cf * dz);
            sa += fabsf(cf * dx) + fabsf(cf * dy) + fabsf(cf * dz);
        }
        if (sabs) *sabs += sa;
        fx = (double)ax - (double)cx;
        fy = (double)ay - (double)cy;
        fz = (double)az - (double)cz;
    }
}

// sum of v over the T consecutive lanes of a lane group (T a power of two <= 32)
__device__ __forceinline__ double group_sum(double v, int T) {
    for (int o = T >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ---------------------------------------------------------------------------
// one stage evaluation for the CTA's group: acc = cm*E + Fc/m + Fimg/m on
// live particles (geometry.py:289-299).  Positions in c.sp (3E), result in
// out (3 arrays of stride E... stored as out[0*E+i], out[E+i], out[2E+i]).

// BEM image-charge force on the stage positions c.sp of the group, into
// c.img (fx, fy, fz: 3E), from the image tables in c.bem.image.  Out of line:
// its per-mode register arrays stay out of the stage code's allocation.
static __device__ __noinline__ void stage_image_force(Ctx& c) {
    __shared__ int s_imgflag;
    const int E = c.E;
    const double* sx = c.sp;
    spt_img::ImgParams ip = spt_img::image_params(c.bem.image, &c.g, c.kc, 0.0);
    ip.soft2 = c.soft2;
    ip.chunks = image_chunks(c.bem.image.n_nodes, c.nt);
    auto load = [&](int i, double& x, double& y, double& z, double& q) {
        x = sx[i];
        y = sx[E + i];
        z = sx[2 * E + i];
        q = c.live[i] ? c.q[i] : 0.0;
    };
    spt_img::group_force<SPT_TRACE_IMAGE_MODES>(c.bem.image, ip, E, load, c.imgs, c.img, c.img + E, c.img + 2 * E,
                                                 &s_imgflag);
}

template <int KIND, int FORM, int FAR>
__device__ void stage_accel(Ctx& c, double* out, int* status_flag) {
    const int E = c.E, tid = threadIdx.x;
    const double* sx = c.sp;
    const double* sy = c.sp + E;
    const double* sz = c.sp + 2 * E;
    const SptGeometry& g = c.g;

    // 1. external field
    if (KIND == SPT_GEOM_TIP_BEM || KIND == SPT_GEOM_WELL_BEM || KIND == SPT_GEOM_POST_BEM) {
        // compact the particles that need the BEM sum into c.list (stable order)
        __shared__ int s_wcount[kMaxWarps + 1];
        int n_list = 0;
        for (int base = 0; base < E; base += c.nt) {
            const int i = base + tid;
            bool need = false;
            if (i < E && c.live[i]) {
                const double x = sx[i], y = sy[i], z = sz[i];
                need = bem_valid<KIND>(x, y, z, g) && blend_weight(z, g.z_handoff) > 0.0;
            }
            const unsigned bal = __ballot_sync(0xffffffffu, need);
            if ((tid & 31) == 0) s_wcount[tid >> 5] = __popc(bal);
            __syncthreads();
            if (tid == 0) {
                int acc = 0;
                for (int w = 0; w < c.nw; ++w) { const int t = s_wcount[w]; s_wcount[w] = acc; acc += t; }
                s_wcount[c.nw] = acc;
            }
            __syncthreads();
            if (need) {
                const int pos = n_list + s_wcount[tid >> 5] + __popc(bal & ((1u << (tid & 31)) - 1u));
                c.list[pos] = i;
                c.bpt[8 * pos + 0] = sx[i];
                c.bpt[8 * pos + 1] = sy[i];
                c.bpt[8 * pos + 2] = sz[i];
            }
            n_list += s_wcount[c.nw];
            __syncthreads();
        }
        if (n_list > 0) {
            if constexpr (FORM == SPT_FORM_SURROGATE)
                surrogate_points<FAR>(c, n_list, status_flag);
            else
                bem_points<FORM, FAR>(c, n_list, false, status_flag);
        }
        // scatter: fld[i] = blended field
        for (int i = tid; i < E; i += c.nt) { c.fld[3 * i + 0] = 0.0; c.fld[3 * i + 1] = 0.0; c.fld[3 * i + 2] = 0.0; }
        __syncthreads();
        for (int k = tid; k < n_list; k += c.nt) {
            const int i = c.list[k];
            c.fld[3 * i + 0] = c.bpt[8 * k + 5];
            c.fld[3 * i + 1] = c.bpt[8 * k + 6];
            c.fld[3 * i + 2] = c.bpt[8 * k + 7];
        }
        __syncthreads();
    }

    // 1b. BEM image-charge force of a tip or well built with z0
    // (bem/geometry.py:326-344, 780-797; bem/image_charge.py:816-1056):
    // the group's joint mode solve, into c.img (fx, fy, fz: 3E)
    bool bem_img = false;
    if constexpr (KIND == SPT_GEOM_TIP_BEM || KIND == SPT_GEOM_WELL_BEM) {
        bem_img = g.has_image && c.bem.image.n_nodes >= 2;
        if (bem_img) stage_image_force(c);
    }

    // 2. image sources for the sphere-on-plane construction (forces.py:170-183)
    const bool three_img = (KIND == SPT_GEOM_TIP || KIND == SPT_GEOM_POST_BEM) && g.has_image;
    if (three_img) {
        const double a = g.R - g.z0;
        const double zc = (KIND == SPT_GEOM_POST_BEM) ? g.L : 0.0;
        for (int j = tid; j < E; j += c.nt) {
            const double x = sx[j], y = sy[j], z = sz[j] - zc;
            const double d = sqrt(x * x + y * y + z * z);
            const double ds = d > 0.0 ? d : a;
            const double sh = (a * a) / (ds * ds);
            c.img[j] = x * sh;
            c.img[E + j] = y * sh;
            c.img[2 * E + j] = z * sh;
            c.img[3 * E + j] = -c.q[j] * (a / ds);
        }
        __syncthreads();
    }

    // 3. per particle: field + pair sums.  Each target's sources are split
    // over T lanes of a warp (T = 256 / E rounded down to a power of two, at
    // most 32), whose partial sums are added with shuffles.  Mixed form: the
    // sums run in float32 first; a target whose sum of |float32 terms| / m
    // exceeds kappa times its whole acceleration is summed again in float64.
    int T = 1;
    while (T < 32 && T * 2 * E <= c.nt) T *= 2;
    const int per_pass = c.nt / T;
    const int sub = tid & (T - 1);
    const int lead = (tid & 31) & ~(T - 1);  // lane of the target's first sub-lane
    unsigned long long pairs = 0, redone = 0;
    for (int base = 0; base < E; base += per_pass) {
        const int i = base + tid / T;
        const bool act = i < E && c.live[i];
        constexpr bool mix = FORM != SPT_FORM_FP64;
        const int ii = i < E ? i : 0;
        const double xi = sx[ii], yi = sy[ii], zi = sz[ii];
        const double qk = c.kc * c.q[ii];
        // this lane's share of the target's Coulomb (fc) and image (fi) sums
        auto pass = [&](auto f32_tag, bool on, double& fcx, double& fcy, double& fcz, double& fix, double& fiy,
                        double& fiz, double& sabs) {
            constexpr bool f32 = decltype(f32_tag)::value;
            fcx = fcy = fcz = fix = fiy = fiz = sabs = 0.0;
            if (!on) return;
            double* sa = f32 ? &sabs : nullptr;
            if (E > 1) {
                auto real = [&](int j, double& x, double& y, double& z, double& q) {
                    x = sx[j]; y = sy[j]; z = sz[j]; q = c.q[j];
                };
                if constexpr (f32) pair_sum<true>(c, E, sub, T, xi, yi, zi, qk, real, fcx, fcy, fcz, sa);
                else pair_sum<false>(c, E, sub, T, xi, yi, zi, qk, real, fcx, fcy, fcz);
            }
            if (KIND == SPT_GEOM_FLAT && g.has_image) {
                const double zimg = -2.0 * g.z0;
                auto mirror = [&](int j, double& x, double& y, double& z, double& q) {
                    x = sx[j]; y = sy[j]; z = zimg - sz[j]; q = -c.q[j];
                };
                if constexpr (f32) pair_sum<true>(c, E, sub, T, xi, yi, zi, qk, mirror, fix, fiy, fiz, sa);
                else pair_sum<false>(c, E, sub, T, xi, yi, zi, qk, mirror, fix, fiy, fiz);
            } else if (three_img) {
                const double zc = (KIND == SPT_GEOM_POST_BEM) ? g.L : 0.0;
                const double pz0 = (KIND == SPT_GEOM_POST_BEM) ? g.L + g.z0 : g.z0;
                const double zl = zi - zc;
                double s1x, s1y, s1z, s2x, s2y, s2z, s3x, s3y, s3z;
                auto sphere = [&](int j, double& x, double& y, double& z, double& q) {
                    x = c.img[j]; y = c.img[E + j]; z = c.img[2 * E + j]; q = c.img[3 * E + j];
                };
                auto plane = [&](int j, double& x, double& y, double& z, double& q) {
                    x = sx[j]; y = sy[j]; z = -2.0 * pz0 - (sz[j] - zc); q = -c.q[j];
                };
                auto plane_sphere = [&](int j, double& x, double& y, double& z, double& q) {
                    x = c.img[j]; y = c.img[E + j]; z = -2.0 * pz0 - c.img[2 * E + j]; q = -c.img[3 * E + j];
                };
                if constexpr (f32) {
                    pair_sum<true>(c, E, sub, T, xi, yi, zl, qk, sphere, s1x, s1y, s1z, sa);
                    pair_sum<true>(c, E, sub, T, xi, yi, zl, qk, plane, s2x, s2y, s2z, sa);
                    pair_sum<true>(c, E, sub, T, xi, yi, zl, qk, plane_sphere, s3x, s3y, s3z, sa);
                } else {
                    pair_sum<false>(c, E, sub, T, xi, yi, zl, qk, sphere, s1x, s1y, s1z);
                    pair_sum<false>(c, E, sub, T, xi, yi, zl, qk, plane, s2x, s2y, s2z);
                    pair_sum<false>(c, E, sub, T, xi, yi, zl, qk, plane_sphere, s3x, s3y, s3z);
                }
                fix = (s1x + s2x) + s3x;
                fiy = (s1y + s2y) + s3y;
                fiz = (s1z + s2z) + s3z;
            }
            // every lane takes part in the shuffles (lanes without work add zeros)
        };
        auto reduce = [&](double& fcx, double& fcy, double& fcz, double& fix, double& fiy, double& fiz,
                          double& sabs) {
            fcx = group_sum(fcx, T); fcy = group_sum(fcy, T); fcz = group_sum(fcz, T);
            fix = group_sum(fix, T); fiy = group_sum(fiy, T); fiz = group_sum(fiz, T);
            sabs = group_sum(sabs, T);
        };
        if (act && sub == 0) {
            pairs += (E > 1 ? E : 0) + ((KIND == SPT_GEOM_FLAT && g.has_image) ? E : 0) + (three_img ? 3 * E : 0);
        }
        double fcx, fcy, fcz, fix, fiy, fiz, sabs;
        pass(std::integral_constant<bool, mix>{}, act, fcx, fcy, fcz, fix, fiy, fiz, sabs);
        reduce(fcx, fcy, fcz, fix, fiy, fiz, sabs);
        auto bem_image = [&]() {  // the BEM image force of 1b takes the place of a pair-sum image
            if (bem_img && act && sub == 0) {
                fix = c.img[i];
                fiy = c.img[E + i];
                fiz = c.img[2 * E + i];
            }
        };
        bem_image();
        double ex = 0.0, ey = 0.0, ez = 0.0;
        if (act && sub == 0) {
            if (KIND == SPT_GEOM_FLAT) {
                ex = 0.0; ey = 0.0; ez = (zi >= 0.0) ? g.E_gun : 0.0;
            } else if (KIND == SPT_GEOM_TIP) {
                tip_field(xi, yi, zi, g.E_gun, g.R, ex, ey, ez);
            } else {
                // blend(near, far) with near = where(valid, uniform + pert, 0) (bem/geometry.py:44-55, bem/fields.py:186-211)
                const double w = blend_weight(zi, g.z_handoff);
                const bool valid = bem_valid<KIND>(xi, yi, zi, g);
                const double fz = (zi >= 0.0) ? g.E_gun : 0.0;
                double nx = 0.0, ny = 0.0, nz = 0.0;
                if (valid && w > 0.0) {
                    nx = 0.0 + c.fld[3 * i + 0];
                    ny = 0.0 + c.fld[3 * i + 1];
                    nz = g.E_gun + c.fld[3 * i + 2];
                } else if (valid) {
                    nx = 0.0; ny = 0.0; nz = g.E_gun;  // pert finite; times w = 0
                }
                ex = w * nx + (1.0 - w) * 0.0;
                ey = w * ny + (1.0 - w) * 0.0;
                ez = w * nz + (1.0 - w) * fz;
            }
        }
        const double mi = act ? c.m[i] : 1.0;
        auto accel_of = [&](double& ax, double& ay, double& az) {
            ax = (c.cm * ex + fcx / mi) + fix / mi;
            ay = (c.cm * ey + fcy / mi) + fiy / mi;
            az = (c.cm * ez + fcz / mi) + fiz / mi;
        };
        double ax = 0.0, ay = 0.0, az = 0.0;
        bool redo = false;
        if (act && sub == 0) {
            accel_of(ax, ay, az);
            redo = mix && !(sabs / mi <= c.kappa * sqrt(ax * ax + ay * ay + az * az));
        }
        redo = __shfl_sync(0xffffffffu, redo, lead);
        if (mix && __any_sync(0xffffffffu, redo)) {
            pass(std::integral_constant<bool, false>{}, act && redo, fcx, fcy, fcz, fix, fiy, fiz, sabs);
            reduce(fcx, fcy, fcz, fix, fiy, fiz, sabs);
            bem_image();
            if (act && redo && sub == 0) {
                accel_of(ax, ay, az);
                ++redone;
            }
        }
        if (i < E && sub == 0) {
            out[i] = ax;
            out[E + i] = ay;
            out[2 * E + i] = az;
        }
    }
    count_add(c, SPT_CNT_FP64_TARGETS, redone);
    count_add(c, SPT_CNT_PAIR_EVALS, pairs);
    __syncthreads();
}

// ---------------------------------------------------------------------------
// add the CTA's shared-memory counters to the global ones and clear them;
// all threads call, after a barrier that orders every count_add before it
__device__ inline void flush_counters(Ctx& c, unsigned long long* counters) {
    for (int k = threadIdx.x; k < SPT_N_COUNTERS; k += blockDim.x) {
        const unsigned long long v = c.cnt[k];
        if (counters && v) atomicAdd(counters + k, v);
        c.cnt[k] = 0;
    }
}

__device__ inline void init_barriers(Ctx& c) {
    c.phase[0] = 0u;
    c.phase[1] = 0u;
    c.phase[2] = 0u;
    if (threadIdx.x == 0) {
        mbar_init(&c.bars[0], 1);
        mbar_init(&c.bars[1], 1);
        mbar_init(&c.bars[2], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// the persistent integrator

struct GroupScalars {
    double t, h, hr, next_cp, err, h_next, next_out;
    int status, exhausted, accepted, out_ptr, out_exh, fire_out;
    long long n_acc, n_rej;
};

// number of entries of the ascending array v[0..n) that are <= x
__device__ __forceinline__ int count_le(const double* v, int n, double x) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (v[mid] <= x) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// Cubic Hermite pieces (screens.py:118-152), evaluated in the reference's order.
__device__ __forceinline__ double hermite_z(double p0, double v0, double p1, double v1, double dt, double s) {
    const double s2 = s * s, s3 = s2 * s;
    const double h00 = 2 * s3 - 3 * s2 + 1, h10 = s3 - 2 * s2 + s, h01 = -2 * s3 + 3 * s2, h11 = s3 - s2;
    return h00 * p0 + h10 * dt * v0 + h01 * p1 + h11 * dt * v1;
}

__device__ __forceinline__ double sgn(double x) { return x > 0.0 ? 1.0 : (x < 0.0 ? -1.0 : 0.0); }

// Screen crossings of one particle over one accepted step (screens.py:43-115,
// 155-168): the Hermite z(s) is split at its extrema so each bracket is
// monotone; a sign change over a bracket is located by 60 bisections and the
// crossing state (Hermite position and derivative) is appended to the record
// buffer.  Half-open (t_old, t_new]: a start exactly on the screen is not a crossing.
static __device__ __noinline__ void screen_crossings(const SptTraceParams& prm, const double* o, const double* n, double t_old,
                                 double dt, long long particle) {
    const double z0 = o[2], z1 = n[2];
    bool moving = false;
    for (int k = 0; k < 6; ++k) moving |= (o[k] != n[k]);
    if (!moving || !(dt > 0.0)) return;
    const double u0 = dt * o[5], u1 = dt * n[5];
    double A = 3 * (2 * (z0 - z1) + u0 + u1);
    double B = 2 * (3 * (z1 - z0) - 2 * u0 - u1);
    double C = u0;
    double sc = fmax(fmax(fabs(A), fabs(B)), fabs(C));
    sc = sc > 0.0 ? sc : 1.0;
    A /= sc; B /= sc; C /= sc;
    const double disc = B * B - 4 * A * C;
    const double q = -0.5 * (B + (B >= 0.0 ? 1.0 : -1.0) * sqrt(fmax(disc, 0.0)));
    double r0 = q / (A != 0.0 ? A : 1.0);
    const double r1 = C / (q != 0.0 ? q : 1.0);
    const double lin = -C / (B != 0.0 ? B : 1.0);
    if (A == 0.0) r0 = lin;
    const bool v0 = (disc >= 0.0) && (A != 0.0 || B != 0.0) && (r0 > 0.0) && (r0 < 1.0);
    const bool v1 = (disc >= 0.0) && (A != 0.0) && (q != 0.0) && (r1 > 0.0) && (r1 < 1.0);
    double cut[4] = {0.0, v0 ? r0 : 1.0, v1 ? r1 : 1.0, 1.0};
    if (cut[1] > cut[2]) { const double tmp = cut[1]; cut[1] = cut[2]; cut[2] = tmp; }
    for (int sidx = 0; sidx < prm.n_screens; ++sidx) {
        const double zs = prm.screens[sidx];
        for (int iv = 0; iv < 3; ++iv) {
            const double left = cut[iv], right = cut[iv + 1];
            const double f0 = hermite_z(z0, o[5], z1, n[5], dt, left) - zs;
            const double f1 = hermite_z(z0, o[5], z1, n[5], dt, right) - zs;
            if (!(right > left) || f0 == 0.0 || sgn(f0) == sgn(f1)) continue;
            double lo = left, hi = right, flo = f0;
            for (int it = 0; it < 60; ++it) {
                const double mid = 0.5 * (lo + hi);
                const double fm = hermite_z(z0, o[5], z1, n[5], dt, mid) - zs;
                const bool same = sgn(fm) == sgn(flo);
                if (same) { lo = mid; flo = fm; } else { hi = mid; }
            }
            const double sv = 0.5 * (lo + hi);
            const double s2 = sv * sv, s3 = s2 * sv;
            const double h00 = 2 * s3 - 3 * s2 + 1, h10 = s3 - 2 * s2 + sv, h01 = -2 * s3 + 3 * s2, h11 = s3 - s2;
            const double d00 = 6 * s2 - 6 * sv, d10 = 3 * s2 - 4 * sv + 1, d01 = -6 * s2 + 6 * sv, d11 = 3 * s2 - 2 * sv;
            const unsigned long long slot = atomicAdd(prm.screen_count, 1ull);
            if ((long long)slot >= prm.screen_capacity) continue;
            const long long cap = prm.screen_capacity;
            double* r = prm.screen_rec;
            r[0 * cap + slot] = t_old + sv * dt;
            for (int k = 0; k < 3; ++k) {
                r[(1 + k) * cap + slot] = h00 * o[k] + (h10 * dt) * o[3 + k] + h01 * n[k] + (h11 * dt) * n[3 + k];
                r[(4 + k) * cap + slot] = (d00 / dt) * o[k] + d10 * o[3 + k] + (d01 / dt) * n[k] + d11 * n[3 + k];
            }
            r[7 * cap + slot] = (double)sidx;
            r[8 * cap + slot] = (double)particle;
        }
    }
}

static __device__ __noinline__ void write_output(const SptTraceParams& prm, long long n_particles, int k, long long pidx,
                                             double t, const double* s) {
    double* r = prm.output_rec + (size_t)k * 7 * n_particles;
    r[pidx] = t;
    for (int c = 0; c < 6; ++c) r[(size_t)(1 + c) * n_particles + pidx] = s[c];
    prm.output_flag[(size_t)k * n_particles + pidx] = 1;
}

// learned-form parameters into the context, and the CTA's 128 TMEM columns
// (the 128 x 128 FP32 accumulator) for its whole lifetime; all threads call
static __device__ void bind_surrogate(Ctx& c, const SptTraceParams& prm, uint32_t* s_tmem) {
    c.sw = prm.sur_w;
    c.sw16 = static_cast<const __nv_bfloat16*>(prm.sur_w16);
    c.s_start = prm.sur_s_start;
    c.log_scale = prm.sur_log_scale;
    c.s_end = prm.sur_s_end;
    c.sig_floor = prm.sur_sig_floor;
    c.band = prm.sur_band;
    c.spot = prm.sur_spot;
    c.dmin = prm.sur_d_min;
    c.dmax = prm.sur_d_max;
    c.sstats = prm.sur_stats;
    if ((threadIdx.x >> 5) == 0) spt_umma::alloc(s_tmem, 128);
    spt_umma::fence_before();
    __syncthreads();
    spt_umma::fence_after();
    c.tmem = *s_tmem;
}

static __device__ void release_surrogate(Ctx& c) {
    spt_umma::fence_before();
    __syncthreads();
    if ((threadIdx.x >> 5) == 0) spt_umma::dealloc(c.tmem, 128);
}

// Persistent trace kernel for geometry kind KIND, arithmetic form FORM and far
// rule FAR.  Launched with blockDim.x in {32, 64, 128, 256} (at most 128
// registers a thread, so two 256-thread CTAs, four of 128 or eight of 64 fit
// an SM's register file); every CTA takes groups from the work queue until it
// is empty.
template <int KIND, int FORM, int FAR>
__global__ void __launch_bounds__(kMaxThreads, 2)
trace_kernel(const __grid_constant__ SptState st, const __grid_constant__ SptTraceParams prm,
             const __grid_constant__ SptGeometry geo, const __grid_constant__ SptBem bem, int* work,
             double* big_slots) {
    extern __shared__ __align__(16) double smem[];
    __shared__ GroupScalars gs;
    __shared__ int s_g;
    __shared__ double s_red[kMaxWarps];
    __shared__ int s_flag;
    __shared__ unsigned long long s_cnt[SPT_N_COUNTERS];
    const int tid = threadIdx.x;
    Ctx c(geo, bem);
    c.cm = prm.charge_to_mass;
    c.kc = prm.coulomb_constant;
    c.soft2 = prm.plummer_radius * prm.plummer_radius;
    const int Emax = st.max_group_size;
    constexpr bool sur = FORM == SPT_FORM_SURROGATE;
    bind(c, smem, Emax, FAR, big_slots ? big_slots + (size_t)blockIdx.x * big_slot_doubles(Emax) : nullptr, s_cnt, sur);
    // launch-configuration parameters (bind sets the defaults)
    c.round_pts = (prm.round_points >= 1 && prm.round_points <= kRound) ? prm.round_points : kRound;
    if (prm.kappa_max > 0.0) c.kappa = prm.kappa_max;
    __shared__ uint32_t s_tmem;
    if constexpr (sur) bind_surrogate(c, prm, &s_tmem);
    init_barriers(c);
    const int nt = c.nt;
    // y0 (state at the step start), nw (candidate state) and the seven stage
    // slopes kp (positions' = velocities) and kv (velocities' = accelerations):
    // component k of particle i at Y0[k * Emax + i], KP(s)[k * E + i]
    double* const Y0 = c.y0;
    double* const NW = c.nw_;
    auto KP = [&](int s_) { return c.kp + 3 * s_ * Emax; };
    auto KV = [&](int s_) { return c.kv + 3 * s_ * Emax; };

    // groups to process: all, or the compacted running ones (count written on the device)
    const int n_run = st.n_active ? *st.n_active : st.n_groups;
    for (;;) {
        if (tid == 0) s_g = atomicAdd(work, 1);
        __syncthreads();
        const int gi = s_g;
        __syncthreads();
        if (gi >= n_run) break;
        const int g = st.group_order ? st.group_order[gi] : gi;
        const long long base = st.group_offset[g];
        const int E = (int)(st.group_offset[g + 1] - base);
        if (tid == 0) {
            gs.status = st.status[g];
            gs.t = st.t[g];
            gs.h = st.h[g];
            gs.n_acc = st.n_accepted[g];
            gs.n_rej = st.n_rejected[g];
            s_flag = 0;
        }
        __syncthreads();
        if (E <= 0 || gs.status >= SPT_GROUP_DONE) continue;
        // the layout keeps the Emax offsets; the stage routines use this group's E
        c.E = E;
        for (int i = tid; i < E; i += nt) {
            Y0[0 * Emax + i] = st.x[base + i]; Y0[1 * Emax + i] = st.y[base + i]; Y0[2 * Emax + i] = st.z[base + i];
            Y0[3 * Emax + i] = st.vx[base + i]; Y0[4 * Emax + i] = st.vy[base + i]; Y0[5 * Emax + i] = st.vz[base + i];
            c.tb[i] = st.t_birth[base + i];
            c.td[i] = st.t_death[base + i];
            c.q[i] = st.charge[base + i];
            c.m[i] = st.mass[base + i];
        }
        __syncthreads();
        // sorted birth times (batched_rk45.py:164): rank sort, ties by index
        for (int i = tid; i < E; i += nt) {
            const double v = c.tb[i];
            int r = 0;
            for (int j = 0; j < E; ++j) { const double u = c.tb[j]; r += (u < v) || (u == v && j < i); }
            c.cps[r] = v;
        }
        __syncthreads();
        if (tid == 0) {
            gs.fire_out = -1;
            if (gs.status == SPT_GROUP_NEW) {
                gs.t = c.cps[0];
                gs.h = (prm.t_max - gs.t) * prm.initial_step_fraction;
                // a group born entirely at or after t_max has nothing to integrate: it is
                // done as it stands (the reference would take a backward step to t_max)
                gs.status = gs.t < prm.t_max ? SPT_GROUP_RUNNING : SPT_GROUP_DONE;
                // an output time equal to the start time fires here (batched_rk45.py:191-209)
                if (prm.n_outputs > 0) {
                    const int last = count_le(prm.output_times, prm.n_outputs, gs.t) - 1;
                    if (last >= 0 && prm.output_times[last] == gs.t) gs.fire_out = last;
                }
            }
        }
        __syncthreads();
        if (gs.fire_out >= 0) {
            for (int i = tid; i < E; i += nt) {
                if (c.tb[i] <= gs.t) {
                    const double sv[6] = {Y0[i], Y0[Emax + i], Y0[2 * Emax + i], Y0[3 * Emax + i], Y0[4 * Emax + i],
                                          Y0[5 * Emax + i]};
                    write_output(prm, st.n_particles, gs.fire_out, base + i, gs.t, sv);
                }
            }
        }
        for (long long att = 0; att < prm.max_attempts; ++att) {
            if (gs.status != SPT_GROUP_RUNNING) break;
            if (tid == 0) {
                // next checkpoint (batched_rk45.py:228-242)
                int lo = 0, hi = E;
                while (lo < hi) { const int mid = (lo + hi) >> 1; if (c.cps[mid] <= gs.t) lo = mid + 1; else hi = mid; }
                gs.exhausted = lo >= E;
                gs.next_cp = gs.exhausted ? prm.t_max : c.cps[lo];
                double target = fmin(gs.next_cp, prm.t_max);
                if (prm.n_outputs > 0) {
                    const int optr = count_le(prm.output_times, prm.n_outputs, gs.t);
                    gs.out_ptr = optr;
                    gs.out_exh = optr >= prm.n_outputs;
                    gs.next_out = gs.out_exh ? prm.t_max : prm.output_times[optr];
                    target = fmin(target, gs.next_out);
                }
                gs.hr = fmin(gs.h, target - gs.t);
                if (!(gs.hr > 0.0) || !isfinite(gs.hr)) gs.status = SPT_GROUP_NONFINITE;
            }
            __syncthreads();
            if (gs.status != SPT_GROUP_RUNNING) break;
            const double t = gs.t, hr = gs.hr;
            for (int i = tid; i < E; i += nt) c.live[i] = (t >= c.tb[i]) && (t < c.td[i]);
            __syncthreads();
            // seven stage evaluations through one call site of stage_accel (a second
            // inlined copy of the stage code would double the kernel's instruction footprint)
            for (int s = 0; s < 7; ++s) {
                double* const kps = KP(s);
                if (s < 6) {
                    for (int i = tid; i < E; i += nt) {
                        double p[6];
#pragma unroll
                        for (int k = 0; k < 6; ++k) p[k] = Y0[k * Emax + i];
                        for (int j = 0; j < s; ++j) {
                            const double a = kA[s][j];
                            if (a == 0.0) continue;
                            const double ha = __dmul_rn(hr, a);
                            const double* kpj = KP(j);
                            const double* kvj = KV(j);
#pragma unroll
                            for (int k = 0; k < 3; ++k) {
                                p[k] = __dadd_rn(p[k], __dmul_rn(ha, kpj[k * E + i]));
                                p[3 + k] = __dadd_rn(p[3 + k], __dmul_rn(ha, kvj[k * E + i]));
                            }
                        }
                        const bool lv = c.live[i];
#pragma unroll
                        for (int k = 0; k < 3; ++k) {
                            c.sp[k * E + i] = p[k];
                            kps[k * E + i] = lv ? p[3 + k] : 0.0;
                        }
                    }
                } else {
                    // 5th-order solution and the endpoint stage (batched_rk45.py:365-370)
                    for (int i = tid; i < E; i += nt) {
#pragma unroll
                        for (int k = 0; k < 3; ++k) {
                            double sp = 0.0, sv = 0.0;
#pragma unroll
                            for (int j = 0; j < 6; ++j) {
                                sp = __dadd_rn(sp, __dmul_rn(kB[j], KP(j)[k * E + i]));
                                sv = __dadd_rn(sv, __dmul_rn(kB[j], KV(j)[k * E + i]));
                            }
                            const double pn = __dadd_rn(Y0[k * Emax + i], __dmul_rn(hr, sp));
                            const double vn = __dadd_rn(Y0[(3 + k) * Emax + i], __dmul_rn(hr, sv));
                            NW[k * Emax + i] = pn;
                            NW[(3 + k) * Emax + i] = vn;
                            c.sp[k * E + i] = pn;
                            kps[k * E + i] = c.live[i] ? vn : 0.0;
                        }
                    }
                }
                __syncthreads();
                c.key = (uint32_t)g * 2654435761u ^ (uint32_t)(gs.n_acc + gs.n_rej) * 40503u ^ (uint32_t)s * 97u;
                stage_accel<KIND, FORM, FAR>(c, KV(s), &s_flag);
            }
            // embedded error norm (batched_rk45.py:372-393)
            double part = 0.0;
            for (int i = tid; i < E; i += nt) {
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    double ep = 0.0, ev = 0.0;
#pragma unroll
                    for (int j = 0; j < 7; ++j) {
                        ep = __dadd_rn(ep, __dmul_rn(kE[j], KP(j)[k * E + i]));
                        ev = __dadd_rn(ev, __dmul_rn(kE[j], KV(j)[k * E + i]));
                    }
                    ep = __dmul_rn(hr, ep);
                    ev = __dmul_rn(hr, ev);
                    const double y0p = Y0[k * Emax + i], nwp = NW[k * Emax + i];
                    const double y0v = Y0[(3 + k) * Emax + i], nwv = NW[(3 + k) * Emax + i];
                    const double scp = __dadd_rn(prm.atol, __dmul_rn(prm.rtol, fmax(fabs(y0p), fabs(nwp))));
                    const double scv = __dadd_rn(kSpeedOfLight * prm.atol, __dmul_rn(prm.rtol, fmax(fabs(y0v), fabs(nwv))));
                    const double a = __ddiv_rn(ep, scp), b = __ddiv_rn(ev, scv);
                    part = __dadd_rn(part, __dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)));
                }
            }
            part = warp_sum(part);
            if ((tid & 31) == 0) s_red[tid >> 5] = part;
            __syncthreads();
            if (tid == 0) {
                double sq = 0.0;
                for (int w = 0; w < c.nw; ++w) sq += s_red[w];
                double err = sqrt(sq / (double)(6 * E));
                if (err == 0.0) err = kTiny;
                const bool acc = err <= 1.0;
                double fac = prm.safety * pow(err, -1.0 / 5.0);
                fac = fmin(fmax(fac, prm.min_factor), prm.max_factor);
                gs.err = err;
                gs.accepted = acc;
                gs.h_next = hr * fac;
                const long long k_att = gs.n_acc + gs.n_rej;
                if (prm.log_capacity > 0 && k_att < prm.log_capacity) {
                    prm.log_h[(size_t)g * prm.log_capacity + k_att] = hr;
                    prm.log_err[(size_t)g * prm.log_capacity + k_att] = err;
                }
                c.cnt[SPT_CNT_ATTEMPTS] += 1;
                c.cnt[SPT_CNT_STAGE_EVALS] += 7ull * E;
            }
            __syncthreads();
            if (gs.accepted) {
                const double t_new = t + hr;
                const double dt = t_new - t;
                const double tol_out = 1e-9 * fmax(prm.t_max, 1e-30);
                const bool hit = prm.n_outputs > 0 && !gs.out_exh && t_new >= gs.next_out - tol_out;
                unsigned long long n_live = 0;
                for (int i = tid; i < E; i += nt) {
                    const bool was = c.live[i];
                    n_live += was;
                    if (was && kill_test<KIND>(NW[i], NW[Emax + i], NW[2 * Emax + i], geo)) c.td[i] = t_new;
                    if (hit || prm.n_screens > 0) {
                        double o[6], nv[6];
                        for (int k = 0; k < 6; ++k) { o[k] = Y0[k * Emax + i]; nv[k] = NW[k * Emax + i]; }
                        if (hit && c.tb[i] <= t_new) write_output(prm, st.n_particles, gs.out_ptr, base + i, t_new, nv);
                        if (prm.n_screens > 0) screen_crossings(prm, o, nv, t, dt, base + i);
                    }
#pragma unroll
                    for (int k = 0; k < 6; ++k) Y0[k * Emax + i] = NW[k * Emax + i];
                }
                count_add(c, SPT_CNT_LIVE_STEPS, n_live);
                if (tid == 0) {
                    gs.t = t_new;
                    gs.n_acc += 1;
                    const double tol = 1e-9 * fmax(prm.t_max, 1e-30);
                    if (!gs.exhausted && t_new >= gs.next_cp - tol)
                        gs.h = (prm.t_max - t_new) * prm.initial_step_fraction;
                    else
                        gs.h = gs.h_next;
                    if (!(t_new < prm.t_max * (1 - 1e-14))) gs.status = SPT_GROUP_DONE;
                    c.cnt[SPT_CNT_ACCEPTED] += 1;
                    c.cnt[SPT_CNT_PARTICLE_STEPS] += (unsigned long long)E;
                }
            } else if (tid == 0) {
                gs.h = gs.h_next;
                gs.n_rej += 1;
            }
            if (tid == 0) {
                if (isnan(gs.err)) gs.status = SPT_GROUP_NONFINITE;
                if (s_flag) gs.status = s_flag;
            }
            __syncthreads();
        }
        // write back
        for (int i = tid; i < E; i += nt) {
            st.x[base + i] = Y0[i]; st.y[base + i] = Y0[Emax + i]; st.z[base + i] = Y0[2 * Emax + i];
            st.vx[base + i] = Y0[3 * Emax + i]; st.vy[base + i] = Y0[4 * Emax + i]; st.vz[base + i] = Y0[5 * Emax + i];
            st.t_death[base + i] = c.td[i];
        }
        if (tid == 0) {
            st.t[g] = gs.t;
            st.h[g] = gs.h;
            st.status[g] = gs.status;
            st.n_accepted[g] = gs.n_acc;
            st.n_rejected[g] = gs.n_rej;
        }
        __syncthreads();
        flush_counters(c, prm.counters);
        __syncthreads();
        // A timed-out barrier wait leaves this CTA's barrier phases unknown:
        // stop taking groups (the remaining ones stay NEW/RUNNING for the host).
        if (s_flag == SPT_GROUP_TIMEOUT) break;
    }
    if constexpr (sur) release_surrogate(c);
}

// one stage evaluation per group (spt_accel), one CTA per group
template <int KIND, int FORM, int FAR>
__global__ void __launch_bounds__(kMaxThreads, 2)
accel_kernel(const __grid_constant__ SptAccelArgs a, const __grid_constant__ SptGeometry geo,
             const __grid_constant__ SptBem bem) {
    extern __shared__ __align__(16) double smem[];
    __shared__ int s_flag;
    __shared__ unsigned long long s_cnt[SPT_N_COUNTERS];
    const int tid = threadIdx.x;
    const int g = blockIdx.x;
    Ctx c(geo, bem);
    c.cm = a.charge_to_mass;
    c.kc = a.coulomb_constant;
    c.soft2 = a.plummer_radius * a.plummer_radius;
    const int Emax = a.max_group_size;
    bind(c, smem, Emax, FAR, nullptr, s_cnt);
    init_barriers(c);
    const long long base = a.group_offset[g];
    const int E = (int)(a.group_offset[g + 1] - base);
    c.E = E;
    if (tid == 0) s_flag = 0;
    for (int i = tid; i < E; i += c.nt) {
        c.sp[i] = a.x[base + i];
        c.sp[E + i] = a.y[base + i];
        c.sp[2 * E + i] = a.z[base + i];
        c.live[i] = a.active[base + i];
        c.q[i] = a.charge[base + i];
        c.m[i] = a.mass[base + i];
    }
    __syncthreads();
    double* out = c.kv;  // slope storage is free on this path (groups here are at most kSmallGroup)
    stage_accel<KIND, FORM, FAR>(c, out, &s_flag);
    for (int i = tid; i < E; i += c.nt) {
        a.ax[base + i] = out[i];
        a.ay[base + i] = out[E + i];
        a.az[base + i] = out[2 * E + i];
    }
}

// ---------------------------------------------------------------------------
// One group per warp, several groups per CTA, the CTA's BEM points pooled
// (groups of at most 32 particles, BEM geometries without the BEM
// image-charge force, float64 form, adaptive far rule).
//
// Lane i of a warp is particle i of the warp's group: stage combination,
// pair sums (one target per lane, sources in order), error norm, controller,
// kills, screens and output times run per warp, with the group scalars held
// alike by every lane (sums over the group taken in lane 0 and broadcast).
// The CTA's warps advance their groups through each stage in step, and the
// BEM points of all of them go into one CTA-wide task pool that every warp
// draws from (closest segment, near quadrature, adaptive far sum -- the CTA
// team's warp routines, so the same field to the bit -- and the rotation,
// written back to the owning group).  With one group per CTA, warps that had
// finished their share of a stage's points idled at the barrier behind the
// slowest point; with one free-running group per warp, the warps' scattered
// positions in the stage code thrashed the instruction cache.  Here the pool
// of ~W x 17 points balances to within one point, warps share their
// instruction stream, and warps whose group is done help with the others'
// points until the work queue is empty.  The step's state -- y0, the
// 5th-order solution and the seven stage slopes -- lives in a per-warp slot
// in global memory (component k of lane i at slot[k * 32 + i], coalesced),
// read and written past L1 so that L1 keeps the BEM tables.

constexpr int kWarpSlotComps = 54;  // y0 6, 5th-order solution 6, stage velocities 21, stage accelerations 21
constexpr int kWarpSlotDoubles = kWarpSlotComps * 32;
// per-warp shared doubles: BEM record 8, near-sum scratch 4, stage positions
// and charges 4 x 32, sphere images 4 x 32, BEM fields 3 x 32, live flags 32 ints
constexpr int kWarpTeamDoubles = 8 + 4 + 4 * 32 + 4 * 32 + 3 * 32 + 16;

__host__ __device__ inline size_t warp_team_smem(int warps) {
    return (size_t)warps * ((size_t)kWarpScratchInts * 4 + (size_t)kWarpTeamDoubles * 8);
}

__device__ __forceinline__ double warp_min_all(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;  // min is exact and order-free: every lane holds the same value
}

// per-warp shared region of warp w
struct WarpTeam {
    double *rec, *nfld, *sx, *sy, *sz, *q, *img, *fld;
    int* live;
    __device__ WarpTeam(double* smem, int nw, int w) {
        double* t = smem + (size_t)nw * kWarpScratchInts / 2 + (size_t)w * kWarpTeamDoubles;
        rec = t;
        nfld = t + 8;
        sx = t + 12;
        sy = sx + 32;
        sz = sy + 32;
        q = sz + 32;
        img = q + 32;
        fld = img + 128;
        live = reinterpret_cast<int*>(fld + 96);
    }
};

// The CTA's BEM task pool of one stage: entries (warp << 5 | particle),
// drawn one per warp task; every warp calls, between the barriers that close
// the appends and open the next stage.
template <int FORM>
__device__ __forceinline__ void pool_bem_points(Ctx& c, double* smem, const int* entries, int count, int* next) {
    const int lane = threadIdx.x & 31;
    double* const P = c.bpt;
    unsigned long long n_near = 0, n_ring_near = 0, far_evals = 0, cl_evals = 0;
    for (;;) {
        int t = 0;
        if (lane == 0) t = atomicAdd(next, 1);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= count) break;
        const int e = entries[t];
        const WarpTeam own(smem, c.nw, e >> 5);
        const int k = e & 31;
        if (lane == 0) {
            P[0] = own.sx[k];
            P[1] = own.sy[k];
            P[2] = own.sz[k];
        }
        __syncwarp();
        closest_point(c, 0, false);
        __syncwarp();
        near_point(c, 0, n_near, n_ring_near);
        __syncwarp();
        far_point<FORM>(c, 0, far_evals, cl_evals);
        __syncwarp();
        if (lane == 0) {  // rotation to (x, y), as bem_points_fused
            const double x = P[0], y = P[1];
            const double rho = hypot(x, y);
            const double e_rho = P[5];
            double ex = 0.0, ey = 0.0;
            if (rho != 0.0) {
                ex = e_rho * (x / rho);
                ey = e_rho * (y / rho);
            }
            own.fld[3 * k + 0] = ex;
            own.fld[3 * k + 1] = ey;
            own.fld[3 * k + 2] = P[6];
        }
        __syncwarp();
    }
    count_add(c, SPT_CNT_NEAR_PAIRS, n_near);
    count_add(c, SPT_CNT_RING_NEAR, n_ring_near);
    count_add(c, SPT_CNT_RING_FAR, far_evals);
    count_add(c, SPT_CNT_CLUSTER_EVALS, cl_evals);
}

// The rest of a stage for this warp's group, after the pool: images, pair
// sums and the blended external field into this lane's acceleration.
template <int KIND>
__device__ __forceinline__ void stage_finish_warp(Ctx& c, const WarpTeam& w, bool live, bool need, double xi,
                                                  double yi, double zi, double mi, double& ax, double& ay,
                                                  double& az) {
    const int lane = threadIdx.x & 31, E = c.E;
    const SptGeometry& g = c.g;
    // image sources of the sphere-on-plane construction (forces.py:170-183)
    const bool three_img = KIND == SPT_GEOM_POST_BEM && g.has_image;
    const double zc = (KIND == SPT_GEOM_POST_BEM) ? g.L : 0.0;
    if (three_img) {
        if (lane < E) {
            const double a = g.R - g.z0;
            const double x = xi, y = yi, z = zi - zc;
            const double d = sqrt(x * x + y * y + z * z);
            const double ds = d > 0.0 ? d : a;
            const double sh = (a * a) / (ds * ds);
            w.img[lane] = x * sh;
            w.img[32 + lane] = y * sh;
            w.img[64 + lane] = z * sh;
            w.img[96 + lane] = -w.q[lane] * (a / ds);
        }
        __syncwarp();
    }
    // pair sums, one target per lane, sources in order (forces.py:16-57,
    // 101-191), and the blended external field
    ax = ay = az = 0.0;
    unsigned long long pairs = 0;
    if (live) {
        const double qk = c.kc * w.q[lane];
        double fcx = 0.0, fcy = 0.0, fcz = 0.0, fix = 0.0, fiy = 0.0, fiz = 0.0;
        if (E > 1) {
            auto real = [&](int j, double& x, double& y, double& z, double& q) {
                x = w.sx[j]; y = w.sy[j]; z = w.sz[j]; q = w.q[j];
            };
            pair_sum<false>(c, E, 0, 1, xi, yi, zi, qk, real, fcx, fcy, fcz);
            pairs += E;
        }
        if (three_img) {
            const double pz0 = g.L + g.z0;
            const double zl = zi - zc;
            double s1x, s1y, s1z, s2x, s2y, s2z, s3x, s3y, s3z;
            auto sphere = [&](int j, double& x, double& y, double& z, double& q) {
                x = w.img[j]; y = w.img[32 + j]; z = w.img[64 + j]; q = w.img[96 + j];
            };
            auto plane = [&](int j, double& x, double& y, double& z, double& q) {
                x = w.sx[j]; y = w.sy[j]; z = -2.0 * pz0 - (w.sz[j] - zc); q = -w.q[j];
            };
            auto plane_sphere = [&](int j, double& x, double& y, double& z, double& q) {
                x = w.img[j]; y = w.img[32 + j]; z = -2.0 * pz0 - w.img[64 + j]; q = -w.img[96 + j];
            };
            pair_sum<false>(c, E, 0, 1, xi, yi, zl, qk, sphere, s1x, s1y, s1z);
            pair_sum<false>(c, E, 0, 1, xi, yi, zl, qk, plane, s2x, s2y, s2z);
            pair_sum<false>(c, E, 0, 1, xi, yi, zl, qk, plane_sphere, s3x, s3y, s3z);
            fix = (s1x + s2x) + s3x;
            fiy = (s1y + s2y) + s3y;
            fiz = (s1z + s2z) + s3z;
            pairs += 3 * E;
        }
        // blend(near, far) with near = where(valid, uniform + pert, 0) (bem/geometry.py:44-55, bem/fields.py:186-211)
        const double wgt = blend_weight(zi, g.z_handoff);
        const bool valid = bem_valid<KIND>(xi, yi, zi, g);
        const double fz = (zi >= 0.0) ? g.E_gun : 0.0;
        double nx = 0.0, ny = 0.0, nz = 0.0;
        if (valid && wgt > 0.0) {
            const double bx = need ? w.fld[3 * lane + 0] : 0.0;
            const double by = need ? w.fld[3 * lane + 1] : 0.0;
            const double bz = need ? w.fld[3 * lane + 2] : 0.0;
            nx = 0.0 + bx;
            ny = 0.0 + by;
            nz = g.E_gun + bz;
        } else if (valid) {
            nx = 0.0; ny = 0.0; nz = g.E_gun;
        }
        const double ex = wgt * nx + (1.0 - wgt) * 0.0;
        const double ey = wgt * ny + (1.0 - wgt) * 0.0;
        const double ez = wgt * nz + (1.0 - wgt) * fz;
        ax = (c.cm * ex + fcx / mi) + fix / mi;
        ay = (c.cm * ey + fcy / mi) + fiy / mi;
        az = (c.cm * ez + fcz / mi) + fiz / mi;
    }
    count_add(c, SPT_CNT_PAIR_EVALS, pairs);
}

template <int KIND, int FORM>
__global__ void __launch_bounds__(kMaxThreads, 2)
trace_warp_kernel(const __grid_constant__ SptState st, const __grid_constant__ SptTraceParams prm,
                  const __grid_constant__ SptGeometry geo, const __grid_constant__ SptBem bem, int* work,
                  double* slots) {
    static_assert(FORM == SPT_FORM_FP64, "the warp team runs the float64 form");
    extern __shared__ __align__(16) double smem[];
    __shared__ unsigned long long s_cnt[SPT_N_COUNTERS];
    __shared__ int s_pool[2][kMaxThreads];  // two stages' task pools, used alternately
    __shared__ int s_pool_n[2], s_pool_next[2];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int k = threadIdx.x; k < SPT_N_COUNTERS; k += blockDim.x) s_cnt[k] = 0;
    if (threadIdx.x < 2) s_pool_n[threadIdx.x] = s_pool_next[threadIdx.x] = 0;
    Ctx c(geo, bem);
    c.cm = prm.charge_to_mass;
    c.kc = prm.coulomb_constant;
    c.soft2 = prm.plummer_radius * prm.plummer_radius;
    c.kappa = prm.kappa_max > 0.0 ? prm.kappa_max : kKappa;
    c.round_pts = 1;
    c.cnt = s_cnt;
    c.nt = blockDim.x;
    c.nw = nw;
    c.tiles = smem;  // far-rule scratch of every warp (far_adaptive_warp takes its own by warp index)
    const WarpTeam w(smem, nw, warp);
    c.bpt = w.rec;
    c.fld = w.nfld;
    c.live = w.live;
    double* const slot = slots + ((size_t)blockIdx.x * nw + warp) * kWarpSlotDoubles + lane;
    auto ld = [&](int k) { return __ldcg(slot + 32 * k); };
    auto sto = [&](int k, double v) { __stcg(slot + 32 * k, v); };
    constexpr int Y0 = 0, NW = 6, KP = 12, KV = 33;
    __syncthreads();

    const int n_run = st.n_active ? *st.n_active : st.n_groups;
    // this warp's group and its scalars (alike in every lane)
    bool have = false, queue_empty = false;
    int g = 0, E = 0, status = 0;
    long long base = 0, pi = 0, n_acc = 0, n_rej = 0, att = 0;
    bool in = false;
    double tb = INFINITY, td = INFINITY, mi = 1.0, t = 0.0, h = 0.0;
    auto write_back = [&]() {
        if (in) {
            st.x[pi] = ld(Y0 + 0); st.y[pi] = ld(Y0 + 1); st.z[pi] = ld(Y0 + 2);
            st.vx[pi] = ld(Y0 + 3); st.vy[pi] = ld(Y0 + 4); st.vz[pi] = ld(Y0 + 5);
            st.t_death[pi] = td;
        }
        if (lane == 0) {
            st.t[g] = t;
            st.h[g] = h;
            st.status[g] = status;
            st.n_accepted[g] = n_acc;
            st.n_rejected[g] = n_rej;
        }
        have = false;
    };
    int tick = 0;  // stages taken by the CTA (the pool parity)
    for (;;) {
        // ready this warp's group for an attempt: take groups from the work
        // queue until one is running and within this call's attempt budget
        double hr = 0.0, next_cp = 0.0, next_out = 0.0;
        bool exhausted = true, out_exh = true;
        int out_ptr = 0;
        for (;;) {
            if (!have) {
                if (queue_empty) break;
                int gi = 0;
                if (lane == 0) gi = atomicAdd(work, 1);
                gi = __shfl_sync(0xffffffffu, gi, 0);
                if (gi >= n_run) { queue_empty = true; break; }
                g = st.group_order ? st.group_order[gi] : gi;
                base = st.group_offset[g];
                E = (int)(st.group_offset[g + 1] - base);
                status = st.status[g];
                if (E <= 0 || E > 32 || status >= SPT_GROUP_DONE) continue;
                in = lane < E;
                pi = base + (in ? lane : 0);
                tb = in ? st.t_birth[pi] : INFINITY;
                td = in ? st.t_death[pi] : INFINITY;
                mi = in ? st.mass[pi] : 1.0;
                __syncwarp();  // the previous group's last pair sums have read q
                w.q[lane] = in ? st.charge[pi] : 0.0;
                if (in) {
                    sto(Y0 + 0, st.x[pi]); sto(Y0 + 1, st.y[pi]); sto(Y0 + 2, st.z[pi]);
                    sto(Y0 + 3, st.vx[pi]); sto(Y0 + 4, st.vy[pi]); sto(Y0 + 5, st.vz[pi]);
                }
                t = st.t[g];
                h = st.h[g];
                n_acc = st.n_accepted[g];
                n_rej = st.n_rejected[g];
                att = 0;
                have = true;
                int fire_out = -1;
                if (status == SPT_GROUP_NEW) {
                    // start at the first birth (batched_rk45.py:164-178)
                    t = warp_min_all(tb);
                    h = (prm.t_max - t) * prm.initial_step_fraction;
                    status = t < prm.t_max ? SPT_GROUP_RUNNING : SPT_GROUP_DONE;
                    if (prm.n_outputs > 0) {
                        const int last = count_le(prm.output_times, prm.n_outputs, t) - 1;
                        if (last >= 0 && prm.output_times[last] == t) fire_out = last;
                    }
                }
                if (fire_out >= 0 && in && tb <= t) {
                    double sv[6];
                    for (int k = 0; k < 6; ++k) sv[k] = ld(Y0 + k);
                    write_output(prm, st.n_particles, fire_out, base + lane, t, sv);
                }
            }
            if (status != SPT_GROUP_RUNNING || att >= prm.max_attempts) {
                write_back();
                continue;
            }
            // next checkpoint: the first birth after t (batched_rk45.py:228-242)
            const double ncp = warp_min_all(tb > t ? tb : INFINITY);
            exhausted = !(ncp < INFINITY);
            next_cp = exhausted ? prm.t_max : ncp;
            double target = fmin(next_cp, prm.t_max);
            out_ptr = 0;
            out_exh = true;
            next_out = prm.t_max;
            if (prm.n_outputs > 0) {
                out_ptr = count_le(prm.output_times, prm.n_outputs, t);
                out_exh = out_ptr >= prm.n_outputs;
                next_out = out_exh ? prm.t_max : prm.output_times[out_ptr];
                target = fmin(target, next_out);
            }
            hr = fmin(h, target - t);
            if (!(hr > 0.0) || !isfinite(hr)) {
                status = SPT_GROUP_NONFINITE;
                write_back();
                continue;
            }
            break;
        }
        const bool run = have;
        if (!__syncthreads_or(run)) break;
        c.E = E;
        const bool live = run && in && (t >= tb) && (t < td);
        // seven stage evaluations (batched_rk45.py:326-370), in step across the CTA
        for (int s = 0; s < 7; ++s, ++tick) {
            const int pp = tick & 1;
            double px = 0.0, py = 0.0, pz = 0.0;
            bool need = false;
            if (run) {
                if (in) {
                    if (s < 6) {
                        double p[6];
#pragma unroll
                        for (int k = 0; k < 6; ++k) p[k] = ld(Y0 + k);
                        for (int j = 0; j < s; ++j) {
                            const double a = kA[s][j];
                            if (a == 0.0) continue;
                            const double ha = __dmul_rn(hr, a);
#pragma unroll
                            for (int k = 0; k < 3; ++k) {
                                p[k] = __dadd_rn(p[k], __dmul_rn(ha, ld(KP + 3 * j + k)));
                                p[3 + k] = __dadd_rn(p[3 + k], __dmul_rn(ha, ld(KV + 3 * j + k)));
                            }
                        }
                        px = p[0]; py = p[1]; pz = p[2];
#pragma unroll
                        for (int k = 0; k < 3; ++k) sto(KP + 3 * s + k, live ? p[3 + k] : 0.0);
                    } else {
                        double pn[3];
#pragma unroll
                        for (int k = 0; k < 3; ++k) {
                            double sp = 0.0, sv = 0.0;
#pragma unroll
                            for (int j = 0; j < 6; ++j) {
                                sp = __dadd_rn(sp, __dmul_rn(kB[j], ld(KP + 3 * j + k)));
                                sv = __dadd_rn(sv, __dmul_rn(kB[j], ld(KV + 3 * j + k)));
                            }
                            pn[k] = __dadd_rn(ld(Y0 + k), __dmul_rn(hr, sp));
                            const double vn = __dadd_rn(ld(Y0 + 3 + k), __dmul_rn(hr, sv));
                            sto(NW + k, pn[k]);
                            sto(NW + 3 + k, vn);
                            sto(KP + 18 + k, live ? vn : 0.0);
                        }
                        px = pn[0]; py = pn[1]; pz = pn[2];
                    }
                }
                w.sx[lane] = px;
                w.sy[lane] = py;
                w.sz[lane] = pz;
                w.live[lane] = live;
                // the BEM field of the live particles inside the valid region
                // with blend weight > 0 goes to the CTA's pool
                need = live && bem_valid<KIND>(px, py, pz, geo) && blend_weight(pz, geo.z_handoff) > 0.0;
                const unsigned m = __ballot_sync(0xffffffffu, need);
                int at = 0;
                if (lane == 0 && m) at = atomicAdd(&s_pool_n[pp], __popc(m));
                at = __shfl_sync(0xffffffffu, at, 0);
                if (need) s_pool[pp][at + __popc(m & ((1u << lane) - 1u))] = (warp << 5) | lane;
            }
            __syncthreads();
            // the other pool is free until the next stage's appends, which follow the barrier below
            if (threadIdx.x == 0) {
                s_pool_n[pp ^ 1] = 0;
                s_pool_next[pp ^ 1] = 0;
            }
            pool_bem_points<FORM>(c, smem, s_pool[pp], s_pool_n[pp], &s_pool_next[pp]);
            __syncthreads();
            if (run) {
                double ax, ay, az;
                stage_finish_warp<KIND>(c, w, live, need, px, py, pz, mi, ax, ay, az);
                if (in) {
                    sto(KV + 3 * s + 0, ax);
                    sto(KV + 3 * s + 1, ay);
                    sto(KV + 3 * s + 2, az);
                }
                __syncwarp();  // the positions and images are rewritten by the next stage
            }
        }
        if (!run) continue;
        // embedded error norm (batched_rk45.py:372-393); the sum over the
        // group in lane 0, as the CTA kernel's fixed-order block sum
        double part = 0.0;
        if (in) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                double ep = 0.0, ev = 0.0;
#pragma unroll
                for (int j = 0; j < 7; ++j) {
                    ep = __dadd_rn(ep, __dmul_rn(kE[j], ld(KP + 3 * j + k)));
                    ev = __dadd_rn(ev, __dmul_rn(kE[j], ld(KV + 3 * j + k)));
                }
                ep = __dmul_rn(hr, ep);
                ev = __dmul_rn(hr, ev);
                const double y0p = ld(Y0 + k), nwp = ld(NW + k);
                const double y0v = ld(Y0 + 3 + k), nwv = ld(NW + 3 + k);
                const double scp = __dadd_rn(prm.atol, __dmul_rn(prm.rtol, fmax(fabs(y0p), fabs(nwp))));
                const double scv = __dadd_rn(kSpeedOfLight * prm.atol, __dmul_rn(prm.rtol, fmax(fabs(y0v), fabs(nwv))));
                const double a = __ddiv_rn(ep, scp), b = __ddiv_rn(ev, scv);
                part = __dadd_rn(part, __dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)));
            }
        }
        const double sq = 0.0 + __shfl_sync(0xffffffffu, warp_sum(part), 0);
        double err = sqrt(sq / (double)(6 * E));
        if (err == 0.0) err = kTiny;
        const bool accepted = err <= 1.0;
        double fac = prm.safety * pow(err, -1.0 / 5.0);
        fac = fmin(fmax(fac, prm.min_factor), prm.max_factor);
        const double h_next = hr * fac;
        if (lane == 0) {
            const long long k_att = n_acc + n_rej;
            if (prm.log_capacity > 0 && k_att < prm.log_capacity) {
                prm.log_h[(size_t)g * prm.log_capacity + k_att] = hr;
                prm.log_err[(size_t)g * prm.log_capacity + k_att] = err;
            }
            atomicAdd(c.cnt + SPT_CNT_ATTEMPTS, 1ull);
            atomicAdd(c.cnt + SPT_CNT_STAGE_EVALS, 7ull * E);
        }
        if (accepted) {
            const double t_new = t + hr;
            const double dt = t_new - t;
            const double tol_out = 1e-9 * fmax(prm.t_max, 1e-30);
            const bool hit = prm.n_outputs > 0 && !out_exh && t_new >= next_out - tol_out;
            if (in) {
                double o[6], nv[6];
#pragma unroll
                for (int k = 0; k < 6; ++k) { o[k] = ld(Y0 + k); nv[k] = ld(NW + k); }
                if (live && kill_test<KIND>(nv[0], nv[1], nv[2], geo)) td = t_new;
                if (hit && tb <= t_new) write_output(prm, st.n_particles, out_ptr, base + lane, t_new, nv);
                if (prm.n_screens > 0) screen_crossings(prm, o, nv, t, dt, base + lane);
#pragma unroll
                for (int k = 0; k < 6; ++k) sto(Y0 + k, nv[k]);
            }
            count_add(c, SPT_CNT_LIVE_STEPS, live ? 1ull : 0ull);
            t = t_new;
            n_acc += 1;
            const double tol = 1e-9 * fmax(prm.t_max, 1e-30);
            if (!exhausted && t_new >= next_cp - tol)
                h = (prm.t_max - t_new) * prm.initial_step_fraction;
            else
                h = h_next;
            if (!(t_new < prm.t_max * (1 - 1e-14))) status = SPT_GROUP_DONE;
            if (lane == 0) {
                atomicAdd(c.cnt + SPT_CNT_ACCEPTED, 1ull);
                atomicAdd(c.cnt + SPT_CNT_PARTICLE_STEPS, (unsigned long long)E);
            }
        } else {
            h = h_next;
            n_rej += 1;
        }
        if (isnan(err)) status = SPT_GROUP_NONFINITE;
        ++att;
    }
    __syncthreads();
    flush_counters(c, prm.counters);
}

// ---------------------------------------------------------------------------
// host-side launchers of the kernels above, instantiated per geometry kind in
// spt_trace_<kind>.cu (kept out of the C ABI's translation unit so that the
// kinds compile in parallel)

struct TraceLaunch {
    const SptState* s;
    const SptTraceParams* p;
    const SptGeometry* g;
    SptBem bem;
    int threads;                 // CTA width
    int* work;                   // zeroed work-queue counter
    double* slots;               // big-group slots (or null)
    long long max_slots;         // largest grid: the CTAs the slot buffer holds, or a caller's cap (0: no limit)
    cudaStream_t stream;
    bool warp_team;              // one group per warp (trace_warp_kernel), slope slots at `slots`
};

// Shared memory and grid of a trace launch; returns 0 or a cudaError_t.
template <int KIND, int FORM, int FAR>
int trace_grid(int max_group_size, int threads, int n_groups, long long max_slots, int img_doubles, size_t* smem,
               int* grid, int* per_sm) {
    const Layout L = make_layout(max_group_size, FAR, FORM == SPT_FORM_SURROGATE, true, threads / 32, img_doubles);
    auto kern = trace_kernel<KIND, FORM, FAR>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.bytes);
    if (e != cudaSuccess) return (int)e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, kern, threads, L.bytes);
    if (e != cudaSuccess) return (int)e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    long long cap = (long long)sms * (*per_sm);
    if (max_slots > 0 && cap > max_slots) cap = max_slots;
    *grid = (int)(n_groups < cap ? n_groups : cap);
    *smem = L.bytes;
    return 0;
}

// Shared memory and grid of a warp-team launch (trace_warp_kernel): as many
// CTAs as the SMs hold, no more than the groups need, capped by max_slots.
template <int KIND, int FORM>
int trace_warp_grid(int threads, int n_groups, long long max_slots, size_t* smem, int* grid, int* per_sm) {
    const size_t bytes = warp_team_smem(threads / 32);
    auto kern = trace_warp_kernel<KIND, FORM>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return (int)e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, kern, threads, bytes);
    if (e != cudaSuccess) return (int)e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    long long cap = (long long)sms * (*per_sm);
    if (max_slots > 0 && cap > max_slots) cap = max_slots;
    const long long need = ((long long)n_groups + threads / 32 - 1) / (threads / 32);
    *grid = (int)(need < cap ? need : cap);
    *smem = bytes;
    return 0;
}

template <int KIND, int FORM>
int trace_warp_launch(const TraceLaunch& t, int grid, size_t smem) {
    trace_warp_kernel<KIND, FORM><<<grid, t.threads, smem, t.stream>>>(*t.s, *t.p, *t.g, t.bem, t.work, t.slots);
    return (int)cudaGetLastError();
}

template <int KIND, int FORM, int FAR>
int trace_launch(const TraceLaunch& t, int grid, size_t smem) {
    trace_kernel<KIND, FORM, FAR><<<grid, t.threads, smem, t.stream>>>(*t.s, *t.p, *t.g, t.bem, t.work, t.slots);
    return (int)cudaGetLastError();
}

template <int KIND, int FORM, int FAR>
int accel_launch(const SptAccelArgs* a, const SptGeometry* g, const SptBem& bem, cudaStream_t stream) {
    const Layout L = make_layout(a->max_group_size, FAR, false, true, kMaxWarps,
                                 image_scratch(*g, bem, a->max_group_size, kMaxThreads));
    auto kern = accel_kernel<KIND, FORM, FAR>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.bytes);
    if (e != cudaSuccess) return (int)e;
    kern<<<a->n_groups, kMaxThreads, L.bytes, stream>>>(*a, *g, bem);
    return (int)cudaGetLastError();
}

// Trace dispatch over the (form, far rule) instantiations of one geometry
// kind: with launch false, only the shared memory, grid and occupancy of the
// launch t describes; with launch true, also the launch on that grid.
// Returns 0, a cudaError_t, or -1 for a (form, far rule) this kind does not
// offer.  Defined here, instantiated once per kind in spt_trace_<kind>.cu.
template <int KIND>
int trace_dispatch(const TraceLaunch& t, int form, int far, bool launch, int* grid, size_t* smem, int* per_sm) {
    constexpr bool kBem = KIND == SPT_GEOM_TIP_BEM || KIND == SPT_GEOM_WELL_BEM || KIND == SPT_GEOM_POST_BEM;
    const int n = t.s->n_groups, E = t.s->max_group_size;
    const int img = image_scratch(*t.g, t.bem, E, t.threads);
#define SPT_TRACE_CASE(F, R)                                                                            \
    {                                                                                                   \
        int rc = trace_grid<KIND, F, R>(E, t.threads, n, t.max_slots, img, smem, grid, per_sm);         \
        if (rc || !launch) return rc;                                                                   \
        return trace_launch<KIND, F, R>(t, *grid, *smem);                                               \
    }
    if constexpr (kBem) {
        if (t.warp_team) {
            if (form != SPT_FORM_FP64 || far != SPT_FAR_ADAPTIVE || E > 32 || img > 0) return -1;
            int rc = trace_warp_grid<KIND, SPT_FORM_FP64>(t.threads, n, t.max_slots, smem, grid, per_sm);
            if (rc || !launch) return rc;
            return trace_warp_launch<KIND, SPT_FORM_FP64>(t, *grid, *smem);
        }
        if (form == SPT_FORM_FP64 && far == SPT_FAR_REFERENCE) SPT_TRACE_CASE(SPT_FORM_FP64, SPT_FAR_REFERENCE)
        if (form == SPT_FORM_FP64 && far == SPT_FAR_ADAPTIVE) SPT_TRACE_CASE(SPT_FORM_FP64, SPT_FAR_ADAPTIVE)
        if (form == SPT_FORM_MIXED && far == SPT_FAR_REFERENCE) SPT_TRACE_CASE(SPT_FORM_MIXED, SPT_FAR_REFERENCE)
        if (form == SPT_FORM_MIXED && far == SPT_FAR_ADAPTIVE) SPT_TRACE_CASE(SPT_FORM_MIXED, SPT_FAR_ADAPTIVE)
        if (form == SPT_FORM_SURROGATE && far == SPT_FAR_REFERENCE) SPT_TRACE_CASE(SPT_FORM_SURROGATE, SPT_FAR_REFERENCE)
        if (form == SPT_FORM_SURROGATE && far == SPT_FAR_ADAPTIVE) SPT_TRACE_CASE(SPT_FORM_SURROGATE, SPT_FAR_ADAPTIVE)
    } else {
        // no BEM field: the far rule plays no part
        if (t.warp_team) return -1;
        if (form == SPT_FORM_FP64) SPT_TRACE_CASE(SPT_FORM_FP64, SPT_FAR_REFERENCE)
        if (form == SPT_FORM_MIXED) SPT_TRACE_CASE(SPT_FORM_MIXED, SPT_FAR_REFERENCE)
    }
#undef SPT_TRACE_CASE
    return -1;
}

// spt_accel dispatch, as trace_dispatch (forms FP64 and MIXED).
template <int KIND>
int accel_dispatch(const SptAccelArgs* a, const SptGeometry* g, const SptBem& bem, cudaStream_t stream) {
    constexpr bool kBem = KIND == SPT_GEOM_TIP_BEM || KIND == SPT_GEOM_WELL_BEM || KIND == SPT_GEOM_POST_BEM;
    const int far = kBem ? bem.far_rule : SPT_FAR_REFERENCE;
    if constexpr (kBem) {
        if (a->form == SPT_FORM_FP64 && far == SPT_FAR_REFERENCE)
            return accel_launch<KIND, SPT_FORM_FP64, SPT_FAR_REFERENCE>(a, g, bem, stream);
        if (a->form == SPT_FORM_FP64 && far == SPT_FAR_ADAPTIVE)
            return accel_launch<KIND, SPT_FORM_FP64, SPT_FAR_ADAPTIVE>(a, g, bem, stream);
        if (a->form == SPT_FORM_MIXED && far == SPT_FAR_REFERENCE)
            return accel_launch<KIND, SPT_FORM_MIXED, SPT_FAR_REFERENCE>(a, g, bem, stream);
        if (a->form == SPT_FORM_MIXED && far == SPT_FAR_ADAPTIVE)
            return accel_launch<KIND, SPT_FORM_MIXED, SPT_FAR_ADAPTIVE>(a, g, bem, stream);
    } else {
        if (a->form == SPT_FORM_FP64) return accel_launch<KIND, SPT_FORM_FP64, SPT_FAR_REFERENCE>(a, g, bem, stream);
        if (a->form == SPT_FORM_MIXED) return accel_launch<KIND, SPT_FORM_MIXED, SPT_FAR_REFERENCE>(a, g, bem, stream);
    }
    return -1;
}

#define SPT_DECLARE_KIND(KIND)                                                                                  \
    extern template int trace_dispatch<KIND>(const TraceLaunch&, int, int, bool, int*, size_t*, int*);         \
    extern template int accel_dispatch<KIND>(const SptAccelArgs*, const SptGeometry*, const SptBem&, cudaStream_t);
#define SPT_INSTANTIATE_KIND(KIND)                                                                              \
    template int trace_dispatch<KIND>(const TraceLaunch&, int, int, bool, int*, size_t*, int*);                \
    template int accel_dispatch<KIND>(const SptAccelArgs*, const SptGeometry*, const SptBem&, cudaStream_t);

}  // namespace spt
