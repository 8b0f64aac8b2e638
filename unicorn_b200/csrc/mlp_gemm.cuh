// BF16 tensor-core GEMM for the surrogate network (sm_100a, tcgen05).
//
//   C[M, N] = A[M, K] * B[N, K]^T      (A, B bf16, row-major, K contiguous; FP32 accumulate)
//
// One CTA of 4 warps computes a 128 x Nt tile (Nt <= 256, a multiple of 16)
// with the accumulator in tensor memory (TMEM, Nt columns of 128 lanes):
//   1. all threads copy (cp.async, 16 B each) a 128 x 64 chunk of A and an
//      Nt x 64 chunk of B from global memory into shared memory in the canonical K-major layout
//      without swizzle (8 x 8 "core matrices" of 128 contiguous bytes; core
//      matrices adjacent in K are 128 B apart, 8-row groups 1024 B apart);
//   2. one thread issues four tcgen05.mma (K = 16 each) and commits them to an
//      mbarrier; the CTA waits (bounded) before the chunk's shared memory is
//      rewritten;
//   3. after the last chunk each warp reads its 32 TMEM lanes (rows) with
//      tcgen05.ld and applies the epilogue (bias, GELU, its derivative,
//      conversions) on the way to global memory.
// The epilogues are those the network needs: forward layers (bias + GELU,
// keeping the pre-activation for the backward pass), the output layer (bias,
// FP32 out), the input gradient of a hidden layer (times GELU'(z)) and the
// weight gradient (FP32 out).
#pragma once
#include <cuda_bf16.h>
#include <cstdint>

#include "uc_device.cuh"

namespace uc {

constexpr int GM = 128;          // rows of a CTA tile (TMEM lanes)
constexpr int GK = 64;           // K chunk staged in shared memory
constexpr int GN_MAX = 256;      // columns of a CTA tile (TMEM columns)
constexpr int GEMM_THREADS = 128;
constexpr size_t GEMM_SMEM = (size_t)(GM + GN_MAX) * GK * 2 + 64;
// dynamic shared memory asked at launch: above the tile's need, so that at most two
// CTAs (2 x 256 TMEM columns) share an SM
constexpr size_t GEMM_SMEM_LAUNCH = 100 * 1024;

enum GemmEpi : int {
    EPI_F32 = 0,        // C as FP32 (out_f32, ldo)
    EPI_BIAS_GELU = 1,  // z = C + bias -> z_save (FP32, if given), gelu(z) -> out_bf16
    EPI_BIAS_F32 = 2,   // C + bias -> out_f32
    EPI_DGELU = 3,      // C * gelu'(z_in) -> out_bf16 (gradient w.r.t. a hidden pre-activation)
    EPI_BIAS_BF16 = 4,  // C + bias -> out_bf16 (no activation)
};

struct GemmArgs {
    const __nv_bfloat16 *A;
    const __nv_bfloat16 *B;
    int lda, ldb;                 // row strides in elements (multiples of 8)
    int M, N, K;                  // N, K multiples of 16 and 64 respectively
    int epi;
    const float *bias;            // [N]
    const float *z_in;            // [M][ldz] (EPI_DGELU)
    float *z_save;                // [M][ldz] (EPI_BIAS_GELU)
    int ldz;
    float *out_f32;               // [M][ldo]
    __nv_bfloat16 *out_bf16;      // [M][ldo]
    int ldo;
    int *status;
};

// GELU in its tanh form, gelu(x) = x/2 (1 + tanh(u)), u = sqrt(2/pi) (x + 0.044715 x^3),
// with the hardware tanh approximation (relative error ~1e-3, below the BF16 rounding
// of the activations it feeds); gelu'(x) = (1 + t)/2 + x/2 (1 - t^2) du/dx.
__device__ __forceinline__ float tanh_hw(float x)
{
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float gelu_f(float x)
{
    const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
    return 0.5f * x * (1.0f + tanh_hw(u));
}
__device__ __forceinline__ float gelu_grad_f(float x)
{
    const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
    const float t = tanh_hw(u);
    const float du = 0.7978845608028654f * (1.0f + 3.0f * 0.044715f * x * x);
    return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * du;
}

// shared-memory matrix descriptor: K-major, no swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;                        // descriptor version of sm_100
    return d;                                      // base offset 0, layout type 0 (no swizzle)
}

// instruction descriptor of kind::f16: BF16 x BF16 -> FP32, both K-major, M x N
__host__ __device__ constexpr uint32_t mma_idesc(int m, int n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// 16-byte asynchronous global -> shared copy (zero-filled when !valid)
__device__ __forceinline__ void cp_async16(void *dst, const void *src, bool valid)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(valid ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__global__ void __launch_bounds__(GEMM_THREADS) gemm_bf16_tc_kernel(const GemmArgs g)
{
    extern __shared__ __align__(1024) unsigned char gsm[];
    unsigned char *sA = gsm;                                  // 128 x 64 bf16 = 16 KB
    unsigned char *sB = gsm + GM * GK * 2;                    // Nt x 64 bf16 <= 32 KB
    uint64_t *bar = reinterpret_cast<uint64_t *>(gsm + (GM + GN_MAX) * GK * 2);
    __shared__ uint32_t s_tmem;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * GM, n0 = blockIdx.y * GN_MAX;
    const int nt = min(GN_MAX, g.N - n0);                     // multiple of 16
    const uint32_t ncols = nt <= 32 ? 32 : nt <= 64 ? 64 : nt <= 128 ? 128 : 256;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(ncols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) mbar_init(bar, 1);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const uint32_t idesc = mma_idesc(GM, nt);
    const int nchunk = g.K / GK;
    bool ok = true;

    for (int kc = 0; kc < nchunk; ++kc) {
        const int k0 = kc * GK;
        // ---- stage A (128 x 64) and B (nt x 64), 16-byte pieces, canonical K-major layout
        for (int i = tid; i < GM * (GK / 8); i += GEMM_THREADS) {
            const int r = i >> 3, kb = i & 7;
            const bool in = m0 + r < g.M;
            cp_async16(sA + ((r >> 3) * (GK / 8) + kb) * 128 + (r & 7) * 16,
                       g.A + (size_t)(in ? m0 + r : 0) * g.lda + k0 + kb * 8, in);
        }
        for (int i = tid; i < nt * (GK / 8); i += GEMM_THREADS) {
            const int r = i >> 3, kb = i & 7;
            cp_async16(sB + ((r >> 3) * (GK / 8) + kb) * 128 + (r & 7) * 16, g.B + (size_t)(n0 + r) * g.ldb + k0 + kb * 8,
                       true);
        }
        cp_async_wait_all();
        // generic-proxy writes -> visible to the tensor core (async proxy)
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (tid == 0) {
            const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
#pragma unroll
            for (int kk = 0; kk < GK / 16; ++kk) {
                const uint64_t ad = smem_desc(a0 + kk * 256, 128, (GK / 8) * 128);
                const uint64_t bd = smem_desc(b0 + kk * 256, 128, (GK / 8) * 128);
                const uint32_t acc = (kc > 0 || kk > 0) ? 1u : 0u;
                asm volatile(
                    "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                    " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                    "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(bar))
                         : "memory");
        }
        // the chunk's shared memory is read by the MMAs until they complete
        const bool done = mbar_wait_bounded(bar, (uint32_t)(kc & 1), 1 << 22);
        if (!done) {
            if (tid == 0) atomicExch(g.status, ST_MMA_TIMEOUT);
            mbar_wait_bounded(bar, (uint32_t)(kc & 1), 1 << 22);   // let work in flight land
        }
        tc_fence_after();
        if (!__syncthreads_and(done)) { ok = false; break; }    // the same decision in every thread
    }

    // ---- epilogue: warp w reads TMEM lanes 32w..32w+31 (rows), 16 columns at a time
    const int row = m0 + warp * 32 + lane;
    if (ok) {
        for (int c0 = 0; c0 < nt; c0 += 16) {
            uint32_t v[16];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                  "=r"(v[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < g.M) {
                const int n = n0 + c0;
                float x[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) x[j] = __uint_as_float(v[j]);
                if (g.epi == EPI_F32) {
#pragma unroll
                    for (int j = 0; j < 16; ++j) g.out_f32[(size_t)row * g.ldo + n + j] = x[j];
                } else if (g.epi == EPI_BIAS_F32) {
#pragma unroll
                    for (int j = 0; j < 16; ++j) g.out_f32[(size_t)row * g.ldo + n + j] = x[j] + g.bias[n + j];
                } else if (g.epi == EPI_BIAS_GELU) {
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const float z = x[j] + g.bias[n + j];
                        if (g.z_save) g.z_save[(size_t)row * g.ldz + n + j] = z;
                        g.out_bf16[(size_t)row * g.ldo + n + j] = __float2bfloat16_rn(gelu_f(z));
                    }
                } else if (g.epi == EPI_DGELU) {
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const float z = g.z_in[(size_t)row * g.ldz + n + j];
                        g.out_bf16[(size_t)row * g.ldo + n + j] = __float2bfloat16_rn(x[j] * gelu_grad_f(z));
                    }
                } else {
#pragma unroll
                    for (int j = 0; j < 16; ++j)
                        g.out_bf16[(size_t)row * g.ldo + n + j] = __float2bfloat16_rn(x[j] + g.bias[n + j]);
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
}

}  // namespace uc

namespace uc {

// ---------------------------------------------------------------------------
// One layer of the network over many rows, weights resident in shared memory:
//   out[M, N] = epi(A[M, K] * W[N, K]^T + bias),   N <= 256, K in {64, 128, 256}
// A persistent CTA per SM (8 warps) stages W once in the canonical K-major
// layout, then walks 128-row tiles of A: it stages the tile, one thread
// issues K/16 tcgen05.mma into one of two TMEM accumulators (2 x 256 columns)
// and commits them to that accumulator's mbarrier, and while they run the
// warps drain the previous tile's accumulator through tcgen05.ld (32 columns
// at a time) into the epilogue (bias from shared memory, GELU -> BF16, or
// bias -> FP32, 16-byte stores). Warp w reads TMEM lanes 32 (w % 4) .. +31
// and half w / 4 of the columns (N / 2 a multiple of 32).
constexpr int LW_THREADS = 256;
constexpr size_t LW_SMEM = (size_t)256 * 256 * 2 + (size_t)128 * 256 * 2 + 64;

__global__ void __launch_bounds__(LW_THREADS, 1) gemm_w_resident_kernel(const GemmArgs g)
{
    extern __shared__ __align__(1024) unsigned char lsm[];
    const int N = g.N, K = g.K;
    unsigned char *sW = lsm;                                   // N x K bf16
    unsigned char *sA = lsm + (size_t)N * K * 2;               // 128 x K bf16
    uint64_t *bar = reinterpret_cast<uint64_t *>(lsm + LW_SMEM - 64);   // two mbarriers
    __shared__ uint32_t s_tmem;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int kb8 = K / 8;                                     // core matrices along K
    const int ntiles = (g.M + GM - 1) / GM;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        mbar_init(bar, 1);
        mbar_init(bar + 1, 1);
    }
    // weights, once per CTA
    for (int i = tid; i < N * kb8; i += LW_THREADS) {
        const int r = i / kb8, kb = i % kb8;
        cp_async16(sW + ((size_t)(r >> 3) * kb8 + kb) * 128 + (r & 7) * 16, g.B + (size_t)r * g.ldb + kb * 8, true);
    }
    cp_async_wait_all();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const uint32_t idesc = mma_idesc(GM, N);
    bool ok = true;
    int it = 0;

    // bias of the layer in shared memory (read by every row)
    __shared__ float s_bias[256];
    for (int i = tid; i < N; i += LW_THREADS) s_bias[i] = g.bias[i];
    __syncthreads();

    auto epilogue = [&](int tile, int buf) {
        const int row = tile * GM + (warp & 3) * 32 + lane;
        const int half = N / 2;                                // 128 or 32 columns per warp
        const int cbeg = (warp >> 2) * half, cend = cbeg + half;
        for (int c0 = cbeg; c0 < cend; c0 += 32) {
            uint32_t v[32];
            const uint32_t taddr = tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)(buf * 256 + c0);
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
                  "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
                  "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < g.M) {
                if (g.epi == EPI_BIAS_GELU) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        __align__(16) __nv_bfloat16 o[8];
#pragma unroll
                        for (int j = 0; j < 8; ++j) {
                            const int c = q * 8 + j;
                            const float z = __uint_as_float(v[c]) + s_bias[c0 + c];
                            if (g.z_save) g.z_save[(size_t)row * g.ldz + c0 + c] = z;
                            o[j] = __float2bfloat16_rn(gelu_f(z));
                        }
                        *reinterpret_cast<uint4 *>(g.out_bf16 + (size_t)row * g.ldo + c0 + q * 8) =
                            *reinterpret_cast<uint4 *>(o);
                    }
                } else {
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        float4 o;
                        o.x = __uint_as_float(v[q * 4 + 0]) + s_bias[c0 + q * 4 + 0];
                        o.y = __uint_as_float(v[q * 4 + 1]) + s_bias[c0 + q * 4 + 1];
                        o.z = __uint_as_float(v[q * 4 + 2]) + s_bias[c0 + q * 4 + 2];
                        o.w = __uint_as_float(v[q * 4 + 3]) + s_bias[c0 + q * 4 + 3];
                        *reinterpret_cast<float4 *>(g.out_f32 + (size_t)row * g.ldo + c0 + q * 4) = o;
                    }
                }
            }
        }
    };

    int prev_tile = -1;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
        const int buf = it & 1;
        // the previous tile's MMAs read sA: wait for them before restaging it
        if (prev_tile >= 0) {
            const bool done = mbar_wait_bounded(bar + (buf ^ 1), (uint32_t)(((it - 1) >> 1) & 1), 1 << 22);
            if (!done) {
                if (tid == 0) atomicExch(g.status, ST_MMA_TIMEOUT);
                mbar_wait_bounded(bar + (buf ^ 1), (uint32_t)(((it - 1) >> 1) & 1), 1 << 22);
            }
            tc_fence_after();
            if (!__syncthreads_and(done)) { ok = false; break; }
        }
        const int m0 = tile * GM;
        for (int i = tid; i < GM * kb8; i += LW_THREADS) {
            const int r = i / kb8, kb = i % kb8;
            const bool in = m0 + r < g.M;
            cp_async16(sA + ((size_t)(r >> 3) * kb8 + kb) * 128 + (r & 7) * 16,
                       g.A + (size_t)(in ? m0 + r : 0) * g.lda + kb * 8, in);
        }
        cp_async_wait_all();
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        __syncthreads();                 // also: the epilogue of tile it-2 (same accumulator) is finished
        tc_fence_after();
        if (tid == 0) {
            const uint32_t a0 = smem_u32(sA), w0 = smem_u32(sW);
            for (int kk = 0; kk < K / 16; ++kk) {
                const uint64_t ad = smem_desc(a0 + kk * 256, 128, kb8 * 128);
                const uint64_t bd = smem_desc(w0 + kk * 256, 128, kb8 * 128);
                const uint32_t acc = kk > 0 ? 1u : 0u;
                asm volatile(
                    "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                    " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem + (uint32_t)(buf * 256)),
                    "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(bar + buf))
                         : "memory");
        }
        // drain the previous accumulator while these MMAs run
        if (prev_tile >= 0) epilogue(prev_tile, buf ^ 1);
        tc_fence_before();
        prev_tile = tile;
    }
    if (ok && prev_tile >= 0) {
        const int buf = (it - 1) & 1;
        const bool done = mbar_wait_bounded(bar + buf, (uint32_t)(((it - 1) >> 1) & 1), 1 << 22);
        if (!done) {
            if (tid == 0) atomicExch(g.status, ST_MMA_TIMEOUT);
            mbar_wait_bounded(bar + buf, (uint32_t)(((it - 1) >> 1) & 1), 1 << 22);
        }
        tc_fence_after();
        if (__syncthreads_and(done)) epilogue(prev_tile, buf);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
}

}  // namespace uc
