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
        __nv_bfloat16 *xr = X + (size_t)(r0 + i) * MLP_IN;
        for (int f = 0; f < MLP_IN; ++f) {
            float v = 0.0f;
            if (f < MLP_NF) {
                const float raw = mlp_raw_feature(f, T, lnp, y, npad, c);
                out |= !(raw >= N->hull_lo[f] && raw <= N->hull_hi[f]);
                v = (raw - N->feat_mu[f]) / N->feat_sd[f];
            }
            xr[f] = __float2bfloat16_rn(v);
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

// Network output rows [0, rows) -> QDSP of cells [c0, c0+rows) ([52][npad], FP64)
__global__ void mlp_decode_kernel(const MlpNorm *N, const float *Out, int rows, double *qdsp, int npad, int c0)
{
    const int nthreads = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows * MLP_NO; i += nthreads) {
        const int k = i / rows, r = i % rows;     // consecutive threads -> consecutive cells of a row
        const float t = Out[(size_t)r * MLP_OUT + k] * N->tgt_sd[k] + N->tgt_mu[k];
        qdsp[(size_t)k * npad + c0 + r] = (double)N->tgt_scale[k] * sinh((double)t);
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

// db[j] = sum over rows of G[m][j] (fixed order per column)
__global__ void bias_grad_kernel(const __nv_bfloat16 *G, int M, int N, float *db)
{
    __shared__ float s[8][33];
    const int j = blockIdx.x * 32 + threadIdx.x;
    float acc = 0.0f;
    if (j < N)
        for (int m = threadIdx.y; m < M; m += blockDim.y) acc += __bfloat162float(G[(size_t)m * N + j]);
    s[threadIdx.y][threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.y == 0 && j < N) {
        float t = 0.0f;
        for (int r = 0; r < (int)blockDim.y; ++r) t += s[r][threadIdx.x];
        db[j] = t;
    }
}

struct AdamArgs {
    float *w, *g, *m, *v;        // flat FP32 parameters, gradients, moments
    int n;
    float lr, b1, b2, eps;
    const int *step;             // steps done before this one
    // BF16 copies of the weight matrices: layer l occupies w[woff[l] .. + out*in]
    __nv_bfloat16 *wb, *wbt;     // [out][in] and [in][out] per layer, flat with the same offsets
    int woff[MLP_LAYERS], wout[MLP_LAYERS], win[MLP_LAYERS], bfoff[MLP_LAYERS];
};

__global__ void adam_kernel(const AdamArgs a)
{
    const int t = *a.step + 1;
    const float c1 = 1.0f - powf(a.b1, (float)t), c2 = 1.0f - powf(a.b2, (float)t);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        const float g = a.g[i];
        const float m = a.b1 * a.m[i] + (1.0f - a.b1) * g;
        const float v = a.b2 * a.v[i] + (1.0f - a.b2) * g * g;
        a.m[i] = m;
        a.v[i] = v;
        const float w = a.w[i] - a.lr * (m / c1) / (sqrtf(v / c2) + a.eps);
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

// Sampled residual check: one cell per 32-cell tile of the field (position
// tile*32 + (hash(tile) & 31), clamped to n-1) is gathered into a compact
// field; after the exact omega of the compact field, each tile's flag is set
// if the surrogate's relative error on that cell exceeds tol over the species
// with Y_k > 1e-8 (relative to max(|w_k|, 1e-6 max_j |w_j|)), or if any of its
// cells lies outside the training hull.
__device__ __forceinline__ int sample_pos(int tile, int n)
{
    unsigned h = (unsigned)tile * 2654435761u;
    h ^= h >> 15;
    const int p = tile * 32 + (int)(h & 31u);
    return p < n ? p : n - 1;
}

__global__ void sample_gather_kernel(const double *tk, const double *rho, const double *y, const double *soot,
                                     int npad, int n, int ntile, double *stk, double *srho, double *sy, double *ssoot,
                                     int snpad)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < snpad; t += gridDim.x * blockDim.x) {
        const int p = sample_pos(t < ntile ? t : ntile - 1, n);
        stk[t] = tk[p];
        srho[t] = rho[p];
        for (int k = 0; k < LSP; ++k) sy[(size_t)k * snpad + t] = y[(size_t)k * npad + p];
        ssoot[t] = soot[p];
        ssoot[snpad + t] = soot[npad + p];
    }
}

__global__ void residual_flag_kernel(const double *qdsp_pred, const double *y, int npad, int n, int ntile,
                                     const double *sq_exact, int snpad, const int *outside, double tol, int *tile_flag,
                                     double *tile_resid)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntile; t += gridDim.x * blockDim.x) {
        const int p = sample_pos(t, n);
        double wmax = 0.0;
        for (int k = 0; k < LSP; ++k) wmax = fmax(wmax, fabs(sq_exact[(size_t)k * snpad + t]));
        double r = 0.0;
        for (int k = 0; k < LSP; ++k) {
            if (!(y[(size_t)k * npad + p] > 1e-8)) continue;
            const double e = sq_exact[(size_t)k * snpad + t];
            const double d = fabs(qdsp_pred[(size_t)k * npad + p] - e) / fmax(fabs(e), 1e-6 * wmax + 1e-300);
            r = fmax(r, d != d ? 1e300 : d);
        }
        int out = 0;
        for (int i = 0; i < 32; ++i) {
            const int c = t * 32 + i;
            if (c < n) out |= outside[c];
        }
        tile_resid[t] = r;
        tile_flag[t] = (out || !(r <= tol)) ? 1 : 0;
    }
}

}  // namespace uc
