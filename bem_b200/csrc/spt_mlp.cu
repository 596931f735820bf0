// BF16 tensor-core kernels (tcgen05, sm_100a) for the learned field
// surrogate: an MLP (rho, z) -> (E_rho, E_z) with four hidden layers of width
// 128 and SiLU activations, BF16 weights and activations, FP32 accumulation.
//
// gemm_kernel: D[M x N] = A[M x K] * B[N x K]^T for tiles of 128 x 128, one
// CTA of 128 threads per tile (and per K split).  Each K chunk of 64 is
// copied by the threads from global memory into shared memory in the
// canonical no-swizzle UMMA layout (8 x 16-byte core matrices), K-major or
// MN-major as the operand is stored, so no transpose is ever materialised;
// one thread issues four tcgen05.mma (K = 16 each) into a 128-lane x
// 128-column FP32 accumulator in tensor memory and commits them to an
// mbarrier; after the last chunk every warp reads its 32 lanes back with
// tcgen05.ld and applies the epilogue:
//   EPI_STORE    C (FP32), optionally one partial per K split;
//   EPI_BIAS_SILU z = acc + bias (FP32 out) and h = SiLU(z) (BF16 out);
//   EPI_DSILU    delta = acc * SiLU'(z) (BF16 out).
// The host builds the training step from these and the small kernels below
// (first and last layers, loss, bias sums, Adam); all of them are this
// library's own code.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "../../include/spt_b200.h"
#include "spt_umma.cuh"

namespace spt_mlp {

constexpr int kTile = 128;   // M and N tile
constexpr int kChunk = 64;   // K per shared-memory chunk
constexpr int kThreads = 128;

using spt_umma::dsilu;
using spt_umma::silu;
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return spt_umma::smem_addr(p); }
__device__ __forceinline__ uint64_t umma_desc(const void* smem, uint32_t lbo, uint32_t sbo) {
    return spt_umma::desc(smem, lbo, sbo);
}
__host__ __device__ constexpr uint32_t umma_idesc(int a_mn, int b_mn) { return spt_umma::idesc_bf16_128(a_mn, b_mn); }
__device__ __forceinline__ void mma_bf16(uint32_t d, uint64_t a, uint64_t b, uint32_t i, uint32_t acc) {
    spt_umma::mma(d, a, b, i, acc);
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) { spt_umma::commit(bar); }
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) { spt_umma::ld16(taddr, v); }

__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t phase) {
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

// Copy a 128 (rows: M or N) x 64 (K) chunk of a BF16 operand into the
// canonical layout.  mn == 0: global element (r, k) at g[r*ld + k] (K
// contiguous) -> K-major core matrices, LBO = 128 B (next 8 k), SBO = 1024 B
// (next 8 rows).  mn == 1: element (r, k) at g[k*ld + r] (rows contiguous) ->
// MN-major core matrices, LBO = 128 B (next 8 k), SBO = 1024 B (next 8 rows).
// Every 16-byte vector stays whole in both cases.  rows_valid/k_valid pad
// with zeros beyond the matrix.
__device__ __forceinline__ void load_chunk(uint8_t* dst, const __nv_bfloat16* g, int64_t ld, int mn, int r0, int k0,
                                           int rows_valid, int k_valid) {
    for (int v = threadIdx.x; v < kTile * kChunk / 8; v += kThreads) {
        uint4 val = make_uint4(0, 0, 0, 0);
        uint32_t off;
        if (mn == 0) {
            const int r = v >> 3, kg = v & 7;  // 8 vectors of 8 k per row
            if (r < rows_valid && kg * 8 < k_valid)
                val = *reinterpret_cast<const uint4*>(g + (int64_t)(r0 + r) * ld + k0 + kg * 8);
            off = (uint32_t)(((r >> 3) * 8 + kg) * 128 + (r & 7) * 16);
        } else {
            const int k = v >> 4, rg = v & 15;  // 16 vectors of 8 rows per k
            if (k < k_valid && rg * 8 < rows_valid)
                val = *reinterpret_cast<const uint4*>(g + (int64_t)(k0 + k) * ld + r0 + rg * 8);
            off = (uint32_t)(rg * 1024 + (k >> 3) * 128 + (k & 7) * 16);
        }
        *reinterpret_cast<uint4*>(dst + off) = val;
    }
}

__global__ void __launch_bounds__(kThreads, 1) gemm_kernel(SptGemmArgs args) {
    struct View {
        int M, N, K, a_mn, b_mn, epi;
        int64_t lda, ldb, ldc, split_stride;
        const __nv_bfloat16 *A, *B;
        float* C;
        const float *bias, *Z;
        __nv_bfloat16* H;
        int32_t* status;
    } a{args.M, args.N, args.K, args.a_mn, args.b_mn, args.epi, args.lda, args.ldb, args.ldc, args.split_stride,
        static_cast<const __nv_bfloat16*>(args.A), static_cast<const __nv_bfloat16*>(args.B), args.C, args.bias,
        args.Z, static_cast<__nv_bfloat16*>(args.H), args.status};
    __shared__ __align__(1024) uint8_t sa[kTile * kChunk * 2];
    __shared__ __align__(1024) uint8_t sb[kTile * kChunk * 2];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t s_tmem;
    __shared__ int s_fail;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int m0 = blockIdx.x * kTile, n0 = blockIdx.y * kTile;
    const int ksplit = a.K / gridDim.z;
    const int kbeg = blockIdx.z * ksplit;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(kTile));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_fail = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    const uint32_t idesc = umma_idesc(a.a_mn, a.b_mn);
    uint32_t phase = 0;
    for (int kc = 0; kc < ksplit; kc += kChunk) {
        const int k0 = kbeg + kc;
        load_chunk(sa, a.A, a.lda, a.a_mn, m0, k0, min(kTile, a.M - m0), min(kChunk, a.K - k0));
        load_chunk(sb, a.B, a.ldb, a.b_mn, n0, k0, min(kTile, a.N - n0), min(kChunk, a.K - k0));
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int kk = 0; kk < kChunk / 16; ++kk) {
                // K-major: the next 16 k are two core matrices (2 x LBO) further;
                // MN-major: two 8-deep k groups (2 x LBO) further as well.
                const uint64_t da = umma_desc(sa + kk * 256, 128, 1024);
                const uint64_t db = umma_desc(sb + kk * 256, 128, 1024);
                mma_bf16(tmem, da, db, idesc, (kc > 0 || kk > 0) ? 1u : 0u);
            }
            mma_commit(&bar);
        }
        if (!bar_wait(&bar, phase)) s_fail = 1;
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        __syncthreads();
    }
    // epilogue: warp w owns accumulator rows (TMEM lanes) 32w..32w+31; thread = one row
    const int row = m0 + warp * 32 + (tid & 31);
    const bool row_ok = row < a.M && !s_fail;
    for (int c0 = 0; c0 < kTile; c0 += 16) {
        float v[16];
        tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
        if (!row_ok) continue;
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const int col = n0 + c0 + i;
            if (col >= a.N) continue;
            const int64_t idx = (int64_t)row * a.ldc + col;
            if (a.epi == SPT_EPI_STORE) {
                a.C[(int64_t)blockIdx.z * a.split_stride + idx] = v[i];
            } else if (a.epi == SPT_EPI_BIAS_SILU) {
                const float z = v[i] + a.bias[col];
                if (a.C) a.C[idx] = z;
                a.H[idx] = __float2bfloat16_rn(silu(z));
            } else {
                a.H[idx] = __float2bfloat16_rn(v[i] * dsilu(a.Z[idx]));
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTile));
    if (tid == 0 && s_fail && a.status) *a.status = 1;
}

}  // namespace spt_mlp

extern "C" int spt_mlp_gemm(const SptGemmArgs* a, void* stream) {
    if (!a || !a->A || !a->B) return 1;
    if (a->M <= 0 || a->N <= 0 || a->K <= 0 || a->K % (spt_mlp::kChunk) != 0) return 1;
    if (a->lda % 8 || a->ldb % 8) return 1;
    // MN-major operands are read in 8-row vectors: whole vectors only
    if ((a->a_mn && a->M % 8) || (a->b_mn && a->N % 8)) return 1;
    if ((reinterpret_cast<uintptr_t>(a->A) & 15) || (reinterpret_cast<uintptr_t>(a->B) & 15)) return 1;
    const int split = a->split_k > 0 ? a->split_k : 1;
    if ((a->K / split) % spt_mlp::kChunk != 0 || a->K % split != 0) return 1;
    if (a->epi != SPT_EPI_STORE && split != 1) return 1;
    if (a->epi == SPT_EPI_STORE && !a->C) return 1;
    if (a->epi != SPT_EPI_STORE && !a->H) return 1;
    if (a->epi == SPT_EPI_BIAS_SILU && !a->bias) return 1;
    if (a->epi == SPT_EPI_DSILU && !a->Z) return 1;
    dim3 grid((a->M + 127) / 128, (a->N + 127) / 128, split);
    spt_mlp::gemm_kernel<<<grid, spt_mlp::kThreads, 0, static_cast<cudaStream_t>(stream)>>>(*a);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// ---------------------------------------------------------------------------
// CUDA-core pieces of the network and of its training step.
namespace spt_mlp {

// first layer: z = W1 x + b1 (W1 [128 x 2], FP32), h = SiLU(z) (BF16)
__global__ void first_layer_kernel(const float* x, int64_t n, const float* W1, const float* b1, float* z,
                                   __nv_bfloat16* h) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n * 128) return;
    const int64_t s = i >> 7;
    const int j = (int)(i & 127);
    const float v = fmaf(W1[2 * j], x[2 * s], fmaf(W1[2 * j + 1], x[2 * s + 1], b1[j]));
    if (z) z[i] = v;
    h[i] = __float2bfloat16_rn(silu(v));
}

// last layer: y = W5 h + b5 (W5 [2 x 128], BF16-rounded weights given as FP32);
// with a target: loss partials, dy = 2 (y - t) / n_batch, and the gradient at
// the last hidden layer delta4 = (W5^T dy) * SiLU'(z4) (BF16), dW5/db5 sums.
// One warp per sample.
__global__ void last_layer_kernel(const __nv_bfloat16* h, const float* z, int64_t n, const float* W5, const float* b5,
                                  float* y, const float* target, float inv_batch, __nv_bfloat16* delta, float* dW5,
                                  float* db5, float* loss) {
    const int64_t s = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (s >= n) return;
    float a0 = 0.f, a1 = 0.f, hv[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int j = lane + 32 * q;
        hv[q] = __bfloat162float(h[s * 128 + j]);
        a0 = fmaf(W5[j], hv[q], a0);
        a1 = fmaf(W5[128 + j], hv[q], a1);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, o);
        a1 += __shfl_xor_sync(0xffffffffu, a1, o);
    }
    const float y0 = a0 + b5[0], y1 = a1 + b5[1];
    if (y && lane == 0) { y[2 * s] = y0; y[2 * s + 1] = y1; }
    if (!target) return;
    const float e0 = y0 - target[2 * s], e1 = y1 - target[2 * s + 1];
    const float g0 = 2.f * e0 * inv_batch, g1 = 2.f * e1 * inv_batch;
    if (lane == 0) {
        atomicAdd(loss, (e0 * e0 + e1 * e1) * inv_batch);
        atomicAdd(db5, g0);
        atomicAdd(db5 + 1, g1);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int j = lane + 32 * q;
        const float d = (W5[j] * g0 + W5[128 + j] * g1) * dsilu(z[s * 128 + j]);
        delta[s * 128 + j] = __float2bfloat16_rn(d);
        atomicAdd(dW5 + j, g0 * hv[q]);
        atomicAdd(dW5 + 128 + j, g1 * hv[q]);
    }
}

// column sums of a BF16 [n x 128] matrix (bias gradients); dW1 = sum delta1 x^T
__global__ void colsum_kernel(const __nv_bfloat16* d, int64_t n, const float* x, float* db, float* dW1) {
    const int j = threadIdx.x;  // 128 threads: one column each
    float acc = 0.f, w0 = 0.f, w1 = 0.f;
    for (int64_t s = blockIdx.x; s < n; s += gridDim.x) {
        const float v = __bfloat162float(d[s * 128 + j]);
        acc += v;
        if (dW1) { w0 = fmaf(v, x[2 * s], w0); w1 = fmaf(v, x[2 * s + 1], w1); }
    }
    atomicAdd(db + j, acc);
    if (dW1) { atomicAdd(dW1 + 2 * j, w0); atomicAdd(dW1 + 2 * j + 1, w1); }
}

__global__ void reduce_splits_kernel(const float* part, int splits, int64_t n, float* out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    float acc = 0.f;
    for (int k = 0; k < splits; ++k) acc += part[k * n + i];
    out[i] = acc;
}

// Adam (decoupled from any framework): FP32 master weights p, moments m, v;
// optional BF16 copy of the updated weights for the tensor-core GEMMs.
__global__ void adam_kernel(float* p, const float* g, float* m, float* v, int64_t n, float lr, float b1, float b2,
                            float eps, float bc1, float bc2, __nv_bfloat16* p16, float* p_rounded) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float pi = p[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    p[i] = pi;
    if (p16) p16[i] = __float2bfloat16_rn(pi);
    if (p_rounded) p_rounded[i] = __bfloat162float(__float2bfloat16_rn(pi));
}

}  // namespace spt_mlp

extern "C" int spt_mlp_first_layer(const float* x, int64_t n, const float* W1, const float* b1, float* z, void* h,
                                   void* stream) {
    if (n <= 0) return 0;
    const int64_t tot = n * 128;
    spt_mlp::first_layer_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        x, n, W1, b1, z, static_cast<__nv_bfloat16*>(h));
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

extern "C" int spt_mlp_last_layer(const void* h, const float* z, int64_t n, const float* W5, const float* b5, float* y,
                                  const float* target, float inv_batch, void* delta, float* dW5, float* db5,
                                  float* loss, void* stream) {
    if (n <= 0) return 0;
    if (target && (!z || !delta || !dW5 || !db5 || !loss)) return 1;
    const int64_t threads = n * 32;
    spt_mlp::last_layer_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const __nv_bfloat16*>(h), z, n, W5, b5, y, target, inv_batch, static_cast<__nv_bfloat16*>(delta),
        dW5, db5, loss);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

extern "C" int spt_mlp_colsum(const void* delta, int64_t n, const float* x, float* db, float* dW1, void* stream) {
    if (n <= 0) return 0;
    const unsigned blocks = (unsigned)(n < 1184 ? n : 1184);
    spt_mlp::colsum_kernel<<<blocks, 128, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const __nv_bfloat16*>(delta), n, x, db, dW1);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

extern "C" int spt_mlp_reduce_splits(const float* part, int32_t splits, int64_t n, float* out, void* stream) {
    if (n <= 0) return 0;
    spt_mlp::reduce_splits_kernel<<<(unsigned)((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        part, splits, n, out);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

extern "C" int spt_mlp_adam(float* p, const float* g, float* m, float* v, int64_t n, float lr, float beta1, float beta2,
                            float eps, int32_t step, void* p_bf16, float* p_rounded, void* stream) {
    if (n <= 0) return 0;
    float bc1 = 1.f, bc2 = 1.f;
    for (int i = 0; i < step; ++i) { bc1 *= beta1; bc2 *= beta2; }
    bc1 = 1.f - bc1;
    bc2 = 1.f - bc2;
    spt_mlp::adam_kernel<<<(unsigned)((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        p, g, m, v, n, lr, beta1, beta2, eps, bc1, bc2, static_cast<__nv_bfloat16*>(p_bf16), p_rounded);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}
