// Learned surrogate of omega: a 54 -> 256 x 4 (GELU) -> 52 network with BF16
// weights and FP32 accumulation, trained and run on the tensor cores
// (mlp_gemm.cuh). This file holds the element-wise and reduction kernels
// around the GEMMs.
//
// Features of a cell (54, padded to 64 with zeros): (T - mu)/sd, (ln p - mu)/sd
// and (ln max(Y_k, 1e-12) - mu_k)/sd_k for the 52 species. Targets (52,
// padded to 64): t_k = (asinh(QDSP_k / s_k) - mu_k)/sd_k, a signed logarithm
// of the reference's QDSP (= -omega_k) with a per-species scale s_k.
#pragma once
#include <cuda_bf16.h>

#include "uc_device.cuh"

namespace uc {

constexpr int MLP_IN = 64;       // 54 features, padded
constexpr int MLP_NF = 54;
constexpr int MLP_H = 256;
constexpr int MLP_OUT = 64;      // 52 outputs, padded
constexpr int MLP_NO = 52;
constexpr int MLP_LAYERS = 5;

struct MlpNorm {
    float feat_mu[MLP_NF], feat_sd[MLP_NF];
    float hull_lo[MLP_NF], hull_hi[MLP_NF];   // training range of each feature (before scaling)
    float tgt_mu[MLP_NO], tgt_sd[MLP_NO], tgt_scale[MLP_NO];
};

// raw features of cell c (T in K, ln p, ln max(Y, 1e-12))
__device__ __forceinline__ float mlp_raw_feature(int f, double T, double lnp, const double *y, size_t np, size_t c)
{
    if (f == 0) return (float)T;
    if (f == 1) return (float)lnp;
    const double yk = y[(size_t)(f - 2) * np + c];
    return (float)log(yk > 1e-12 ? yk : 1e-12);
}

// Features of cells [c0, c0+rows) of a context's fields into X rows [r0, r0+rows);
// outside[c - c0] = 1 if any raw feature lies outside the training hull (optional).
__global__ void mlp_features_kernel(const DevParams *Pp, const MlpNorm *N, const double *tk, const double *pnd,
                                    const double *y, int npad, int c0, int rows, __nv_bfloat16 *X, int r0,
                                    int *outside)
{
    const DevParams &P = *Pp;
    const int nthreads = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += nthreads) {
        const size_t c = (size_t)c0 + i;
        const double T = tk[c] * P.TSTR;
        const double lnp = log(pnd[c] / P.PBACK);      // ln(p / reference pressure)
        int out = 0;
        uint4 *xr = reinterpret_cast<uint4 *>(X + (size_t)(r0 + i) * MLP_IN);
        for (int f0 = 0; f0 < MLP_IN; f0 += 8) {          // eight features -> one 16-byte store
            __align__(16) __nv_bfloat16 o[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int f = f0 + j;
                float v = 0.0f;
                if (f < MLP_NF) {
                    const float raw = mlp_raw_feature(f, T, lnp, y, npad, c);
                    out |= !(raw >= N->hull_lo[f] && raw <= N->hull_hi[f]);
                    v = (raw - N->feat_mu[f]) / N->feat_sd[f];
                }
                o[j] = __float2bfloat16_rn(v);
            }
            xr[f0 / 8] = *reinterpret_cast<const uint4 *>(o);
        }
        if (outside) outside[i] = out;
    }
}

// Targets of cells [c0, c0+rows) from QDSP rows [52][npad] into T rows [r0, ...)
__global__ void mlp_targets_kernel(const MlpNorm *N, const double *qdsp, int npad, int c0, int rows, float *Tg, int r0)
{
    const int nthreads = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows * MLP_OUT; i += nthreads) {
        const int r = i / MLP_OUT, k = i % MLP_OUT;
        float v = 0.0f;
        if (k < MLP_NO) {
            const double q = qdsp[(size_t)k * npad + c0 + r];
            v = ((float)asinh(q / N->tgt_scale[k]) - N->tgt_mu[k]) / N->tgt_sd[k];
        }
        Tg[(size_t)(r0 + r) * MLP_OUT + k] = v;
    }
}

// batch rows from the data set: X[b] = Xall[idx[b]], T[b] = Tall[idx[b]]
__global__ void mlp_gather_kernel(const __nv_bfloat16 *Xall, const float *Tall, const int *idx, const int *step,
                                  int batch, __nv_bfloat16 *X, float *T)
{
    const int base = *step * batch;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < batch * MLP_OUT; i += gridDim.x * blockDim.x) {
        const int b = i / MLP_OUT, f = i % MLP_OUT;
        const size_t src = (size_t)idx[base + b];
        X[(size_t)b * MLP_IN + f] = Xall[src * MLP_IN + f];
        T[(size_t)b * MLP_OUT + f] = Tall[src * MLP_OUT + f];
    }
}

// dLoss/dOut for the mean squared error over the 52 real outputs; per-block loss partials
__global__ void mlp_loss_grad_kernel(const float *Out, const float *T, int M, __nv_bfloat16 *G, double *partial)
{
    __shared__ double s[256];
    double acc = 0.0;
    const float scale = 2.0f / ((float)M * (float)MLP_NO);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < M * MLP_OUT; i += gridDim.x * blockDim.x) {
        const int k = i % MLP_OUT;
        float g = 0.0f;
        if (k < MLP_NO) {
            const float d = Out[i] - T[i];
            acc += (double)d * d;
            g = scale * d;
        }
        G[i] = __float2bfloat16_rn(g);
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = s[0];
}

// loss of the step = sum(partials) / (M * 52), stored at loss_hist[*step]
__global__ void mlp_loss_final_kernel(const double *partial, int nblk, int M, const int *step, float *loss_hist)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int b = 0; b < nblk; ++b) s += partial[b];
        loss_hist[*step] = (float)(s / ((double)M * MLP_NO));
    }
}

// out[C][R] = in[R][C] (bf16), 32 x 32 tiles through shared memory
__global__ void transpose_bf16_kernel(const __nv_bfloat16 *in, int R, int C, __nv_bfloat16 *out)
{
    __shared__ __nv_bfloat16 t[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;     // x: columns of in, y: rows of in
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int r = by + j, c = bx + threadIdx.x;
        if (r < R && c < C) t[j][threadIdx.x] = in[(size_t)r * C + c];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int c = bx + j, r = by + threadIdx.x;
        if (r < R && c < C) out[(size_t)c * R + r] = t[threadIdx.x][j];
    }
}

// db[j] = sum over the batch of Gt[j][m] (the transposed output gradient, rows contiguous): one warp per
// j, 16-byte loads, each lane's partial in a fixed order, then a fixed shuffle tree
__global__ void bias_grad_kernel(const __nv_bfloat16 *Gt, int M, int N, float *db)
{
    const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (j >= N) return;
    const __nv_bfloat16 *row = Gt + (size_t)j * M;
    float acc = 0.0f;
    int m = lane * 8;
    for (; m + 8 <= M; m += 256) {
        const uint4 q = *reinterpret_cast<const uint4 *>(row + m);
        const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&q);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float2 f = __bfloat1622float2(h[i]);
            acc += f.x + f.y;
        }
    }
    for (int r = m; r < M && r < m + 8; ++r) acc += __bfloat162float(row[r]);    // ragged tail
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) db[j] = acc;
}

struct AdamArgs {
    float *w, *g, *m, *v;        // flat FP32 parameters, gradients, moments
    int n;
    float lr, b1, b2, eps;
    const int *step;             // steps done before this one
    const int *iter;             // steps of this training call done before this one (null: constant lr)
    int total;                   // steps of this training call: lr decays to lr/100 along a half cosine
    // BF16 copies of the weight matrices: layer l occupies w[woff[l] .. + out*in]
    __nv_bfloat16 *wb, *wbt;     // [out][in] and [in][out] per layer, flat with the same offsets
    int woff[MLP_LAYERS], wout[MLP_LAYERS], win[MLP_LAYERS], bfoff[MLP_LAYERS];
};

__global__ void adam_kernel(const AdamArgs a)
{
    const int t = *a.step + 1;
    const float c1 = 1.0f - powf(a.b1, (float)t), c2 = 1.0f - powf(a.b2, (float)t);
    float lr = a.lr;
    if (a.iter && a.total > 1) {
        const float f = (float)*a.iter / (float)(a.total - 1);
        lr = 0.01f * a.lr + 0.5f * 0.99f * a.lr * (1.0f + cospif(f));
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        const float g = a.g[i];
        const float m = a.b1 * a.m[i] + (1.0f - a.b1) * g;
        const float v = a.b2 * a.v[i] + (1.0f - a.b2) * g * g;
        a.m[i] = m;
        a.v[i] = v;
        const float w = a.w[i] - lr * (m / c1) / (sqrtf(v / c2) + a.eps);
        a.w[i] = w;
        for (int l = 0; l < MLP_LAYERS; ++l) {
            const int rel = i - a.woff[l];
            if (rel >= 0 && rel < a.wout[l] * a.win[l]) {
                const int o = rel / a.win[l], in = rel % a.win[l];
                const __nv_bfloat16 b = __float2bfloat16_rn(w);
                a.wb[a.bfoff[l] + rel] = b;
                a.wbt[a.bfoff[l] + in * a.wout[l] + o] = b;
            }
        }
    }
}

__global__ void step_incr_kernel(int *step)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) *step += 1;
}

// Per-cell checks of the surrogate's omega. A cell falls back to the exact FP64
// kernel when it lies outside the training hull, or when the surrogate's omega
// breaks element conservation by more than the tolerance: every reaction of the
// mechanism conserves C, H and O, so the exact omega satisfies
// sum_k a_ek omega_k / W_k = 0 to rounding (1e-16 of sum_k |a_ek omega_k / W_k|),
// while the network's errors show up in that residual cell by cell. Every 32nd
// cell (position `off` within each group of 32) is recomputed as well, as a
// sample of the surrogate's true error: its prediction is kept (pred_s) and
// whether the checks accepted it (pass_s). Flagged cells are appended to `list`.
__global__ void mlp_cell_check_kernel(const DevParams *Pp, const double *qdsp, const int *outside, int n, int npad,
                                      double tol, int off, int *list, int *count, double *pred_s, int *pass_s)
{
    const DevParams &P = *Pp;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        double num[3] = {0.0, 0.0, 0.0}, den[3] = {0.0, 0.0, 0.0};
        for (int k = 0; k < LSP; ++k) {
            const double f = qdsp[(size_t)k * npad + c] / P.WM[k];
            for (int e = 0; e < 3; ++e) {
                const double t = (double)P.elem[k * 3 + e] * f;
                num[e] += t;
                den[e] += fabs(t);
            }
        }
        double r = 0.0;
        for (int e = 0; e < 3; ++e)
            if (den[e] > 0.0) r = fmax(r, fabs(num[e]) / den[e]);
        const bool ok = !outside[c] && r <= tol;           // NaN fails
        const bool sample = (c & 31) == off;
        if (sample) {
            const int sidx = c >> 5;
            for (int k = 0; k < LSP; ++k) pred_s[(size_t)sidx * LSP + k] = qdsp[(size_t)k * npad + c];
            pass_s[sidx] = ok ? 1 : 0;
        }
        if (!ok || sample) list[atomicAdd(count, 1)] = c;
    }
}

// The flagged cells as a compact field (cell t of the compact field is list[t]; the padding of the last
// 32-cell tile repeats the last flagged cell) and the tile list the exact kernel walks.
__global__ void mlp_gather_cells_kernel(const int *list, const int *count, const double *tk, const double *rho,
                                        const double *y, const double *soot, int npad, double *stk, double *srho,
                                        double *sy, double *ssoot, int snpad, int *tlist, int *tcount)
{
    const int cnt = *count, m = (cnt + 31) & ~31;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x) {
        const int c = list[t < cnt ? t : cnt - 1];
        stk[t] = tk[c];
        srho[t] = rho[c];
        for (int k = 0; k < LSP; ++k) sy[(size_t)k * snpad + t] = y[(size_t)k * npad + c];
        ssoot[t] = soot[c];
        ssoot[snpad + t] = soot[npad + c];
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m / 32; i += gridDim.x * blockDim.x) tlist[i] = i;
    if (blockIdx.x == 0 && threadIdx.x == 0) *tcount = m / 32;
}

// exact omega of the compact field back to the flagged cells
__global__ void mlp_scatter_cells_kernel(const int *list, const int *count, const double *sq, const double *sqd,
                                         int snpad, double *qdsp, double *qdot, int npad)
{
    const int cnt = *count;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += gridDim.x * blockDim.x) {
        const int c = list[t];
        for (int k = 0; k < LSP; ++k) qdsp[(size_t)k * npad + c] = sq[(size_t)k * snpad + t];
        if (qdot) qdot[c] = sqd[t];
    }
}

// the surrogate's error on each sampled cell: max over species with Y_k > 1e-8 of
// |predicted - exact| / max(|exact|, 1e-6 max_j |exact_j|); -1 for positions beyond n
__global__ void mlp_sample_error_kernel(const double *pred_s, const double *qdsp, const double *y, int n, int npad,
                                        int off, int ns, double *err_s)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < ns; s += gridDim.x * blockDim.x) {
        const int c = s * 32 + off;
        if (c >= n) { err_s[s] = -1.0; continue; }
        double wmax = 0.0;
        for (int k = 0; k < LSP; ++k) wmax = fmax(wmax, fabs(qdsp[(size_t)k * npad + c]));
        double r = 0.0;
        for (int k = 0; k < LSP; ++k) {
            if (!(y[(size_t)k * npad + c] > 1e-8)) continue;
            const double e = qdsp[(size_t)k * npad + c];
            const double d = fabs(pred_s[(size_t)s * LSP + k] - e) / fmax(fabs(e), 1e-6 * wmax + 1e-300);
            r = fmax(r, d != d ? 1e300 : d);
        }
        err_s[s] = r;
    }
}

}  // namespace uc
