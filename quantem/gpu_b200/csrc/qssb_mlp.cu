// qssb_mlp.cu - training and inference kernels of the learned aberration
// proposer: BF16 tensor-core GEMMs with FP32 accumulation and fused bias/GELU
// epilogues, the GELU backward, the MSE loss and its gradient, bias-gradient
// reductions and an Adam step on FP32 master weights that refreshes the BF16
// copies. No counterpart in the reference (it has no learned component).
//
// GEMM: C[M][N] = op(A)[M][K] * op(B)[K][N] (+ C when accumulate), A and B
// BF16 with a per-operand transpose flag, FP32 accumulation in the tensor
// cores (warp-level 16x16x16 BF16 MMA), M, N, K multiples of 16. Each warp
// owns a 32x32 output tile; each CTA of 4 warps a 64x64 tile. The epilogue
// adds a bias, stores the FP32 pre-activation and/or a BF16 copy of
// GELU(pre) for the next layer.
#include <cuda_bf16.h>
#include <math.h>
#include <mma.h>

#include "qssb_internal.h"

namespace qssb {

using namespace nvcuda;

constexpr int kGemmWarpTile = 32;
constexpr int kGemmCtaTile = 64;

// GELU with the tanh form: 0.5 x (1 + tanh(s (x + 0.044715 x^3))), s = sqrt(2/pi).
__device__ __forceinline__ float gelu_f(float x) {
    const float s = 0.7978845608028654f;
    const float u = s * fmaf(0.044715f * x * x, x, x);
    return 0.5f * x * (1.0f + tanhf(u));
}

__device__ __forceinline__ float gelu_grad(float x) {
    const float s = 0.7978845608028654f;
    const float x2 = x * x;
    const float u = s * fmaf(0.044715f * x2, x, x);
    const float t = tanhf(u);
    const float du = s * fmaf(3.0f * 0.044715f, x2, 1.0f);
    return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * du;
}

template <bool TA, bool TB>
__global__ void __launch_bounds__(128) k_gemm_bf16(
    const __nv_bfloat16* __restrict__ A, int lda, const __nv_bfloat16* __restrict__ B, int ldb,
    int M, int N, int K, const float* __restrict__ bias, int accumulate,
    float* __restrict__ C, int ldc, __nv_bfloat16* __restrict__ act, int ld_act) {
    using LA = typename std::conditional<TA, wmma::col_major, wmma::row_major>::type;
    using LB = typename std::conditional<TB, wmma::col_major, wmma::row_major>::type;
    __shared__ float stage[4][16 * 16];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int m0 = blockIdx.y * kGemmCtaTile + (warp >> 1) * kGemmWarpTile;
    const int n0 = blockIdx.x * kGemmCtaTile + (warp & 1) * kGemmWarpTile;
    if (m0 >= M || n0 >= N) return;  // warp-uniform; no block barrier below
    wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc[2][2];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) wmma::fill_fragment(acc[i][j], 0.0f);
    const bool mi1 = m0 + 16 < M;
    const bool nj1 = n0 + 16 < N;
    for (int k = 0; k < K; k += 16) {
        wmma::fragment<wmma::matrix_a, 16, 16, 16, __nv_bfloat16, LA> fa[2];
        wmma::fragment<wmma::matrix_b, 16, 16, 16, __nv_bfloat16, LB> fb[2];
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            if (i == 1 && !mi1) break;
            const int m = m0 + 16 * i;
            const __nv_bfloat16* pa = TA ? A + (size_t)k * lda + m : A + (size_t)m * lda + k;
            wmma::load_matrix_sync(fa[i], pa, lda);
        }
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            if (j == 1 && !nj1) break;
            const int n = n0 + 16 * j;
            const __nv_bfloat16* pb = TB ? B + (size_t)n * ldb + k : B + (size_t)k * ldb + n;
            wmma::load_matrix_sync(fb[j], pb, ldb);
        }
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 2; ++j)
                if ((i == 0 || mi1) && (j == 0 || nj1)) wmma::mma_sync(acc[i][j], fa[i], fb[j], acc[i][j]);
    }
    float* st = stage[warp];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            if ((i == 1 && !mi1) || (j == 1 && !nj1)) continue;
            wmma::store_matrix_sync(st, acc[i][j], 16, wmma::mem_row_major);
            __syncwarp();
            for (int e = lane; e < 256; e += 32) {
                const int r = m0 + 16 * i + (e >> 4);
                const int c = n0 + 16 * j + (e & 15);
                float v = st[e];
                if (bias) v += bias[c];
                if (C) {
                    float* pc = C + (size_t)r * ldc + c;
                    *pc = accumulate ? *pc + v : v;
                }
                if (act) act[(size_t)r * ld_act + c] = __float2bfloat16_rn(gelu_f(v));
            }
            __syncwarp();
        }
    }
}

// dZ = dY * GELU'(pre), as BF16 for the next GEMMs and FP32 for the bias gradient.
__global__ void k_gelu_backward(const float* __restrict__ dy, const float* __restrict__ pre,
                                long long n, __nv_bfloat16* __restrict__ dz_bf,
                                float* __restrict__ dz) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float g = dy[i] * gelu_grad(pre[i]);
        dz[i] = g;
        dz_bf[i] = __float2bfloat16_rn(g);
    }
}

// db[c] = sum over rows of dz[r][c]: 32 columns per CTA (one per lane, so a
// warp reads 128 contiguous bytes of a row), eight warps over interleaved row
// slices in FP64, folded in warp order (a fixed order).
constexpr int kBiasWarps = 8;
__global__ void __launch_bounds__(32 * kBiasWarps) k_bias_grad(const float* __restrict__ dz,
                                                               int rows, int cols,
                                                               float* __restrict__ db) {
    __shared__ double part[kBiasWarps][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int c = blockIdx.x * 32 + lane;
    double s = 0.0;
    if (c < cols)
        for (int r = w; r < rows; r += kBiasWarps) s += (double)dz[(size_t)r * cols + c];
    part[w][lane] = s;
    __syncthreads();
    if (w == 0 && c < cols) {
        double t = 0.0;
        for (int k = 0; k < kBiasWarps; ++k) t += part[k][lane];
        db[c] = (float)t;
    }
}

// MSE over the first n_out of ld columns: loss = mean (y - t)^2 over rows x n_out,
// dy = 2 (y - t) / (rows * n_out) (zero in the padding columns).
__global__ void __launch_bounds__(256) k_mse(const float* __restrict__ y, const float* __restrict__ t,
                                             int rows, int n_out, int ld, float* __restrict__ dy,
                                             float* __restrict__ loss) {
    __shared__ double red[256];
    const double scale = 1.0 / ((double)rows * n_out);
    double acc = 0.0;
    for (int i = threadIdx.x; i < rows * ld; i += 256) {
        const int r = i / ld;
        const int c = i - r * ld;
        float g = 0.0f;
        if (c < n_out) {
            const float d = y[i] - t[(size_t)r * n_out + c];
            acc += (double)d * d;
            g = (float)(2.0 * scale) * d;
        }
        dy[i] = g;
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0 && loss) *loss = (float)(red[0] * scale);
}

// Multi-head (winner-takes-all) MSE. Row r of y holds `heads` groups of n_out
// outputs (columns h n_out .. h n_out + n_out - 1, padding up to ld). The
// winning head of a row is the one with the least squared error over its
// first n_select outputs (ties: the lowest index); the loss is the mean over
// rows of sum_c w_c (y_win,c - t_c)^2 / n_out and the gradient of head h is
// dy_h,c = 2 s_h w_c (y_h,c - t_c) / (rows n_out), with s = 1 - eps for the
// winner and eps / (heads - 1) for the others (s = 1 with one head). One
// thread per row; the loss sums in FP64 in a fixed order.
__global__ void __launch_bounds__(256) k_mse_heads(
    const float* __restrict__ y, const float* __restrict__ t, int rows, int n_out, int heads,
    int ld, const float* __restrict__ w_out, int n_select, float eps, float* __restrict__ dy,
    float* __restrict__ loss, int* __restrict__ winner) {
    __shared__ double red[256];
    const double scale = 1.0 / ((double)rows * n_out);
    double acc = 0.0;
    for (int r = threadIdx.x; r < rows; r += 256) {
        const float* yr = y + (size_t)r * ld;
        const float* tr = t + (size_t)r * n_out;
        int win = 0;
        float best = 0.0f;
        for (int h = 0; h < heads; ++h) {
            float e = 0.0f;
            for (int c = 0; c < n_select; ++c) {
                const float d = yr[h * n_out + c] - tr[c];
                e = fmaf(d, d, e);
            }
            if (h == 0 || e < best) {
                best = e;
                win = h;
            }
        }
        if (winner) winner[r] = win;
        float* dr = dy + (size_t)r * ld;
        for (int c = heads * n_out; c < ld; ++c) dr[c] = 0.0f;
        for (int h = 0; h < heads; ++h) {
            const float s = heads == 1 ? 1.0f : (h == win ? 1.0f - eps : eps / (float)(heads - 1));
            for (int c = 0; c < n_out; ++c) {
                const float wc = w_out ? w_out[c] : 1.0f;
                const float d = yr[h * n_out + c] - tr[c];
                if (h == win) acc += (double)wc * d * d;
                dr[h * n_out + c] = (float)(2.0 * scale) * s * wc * d;
            }
        }
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0 && loss) *loss = (float)(red[0] * scale);
}

// Adam on FP32 master weights (bias-corrected), then the BF16 copy. With
// `hyper` the learning rate and the bias corrections come from the device
// ({lr, c1, c2}, written by k_adam_schedule) instead of the arguments.
__global__ void k_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ g, long long n, float lr, float b1, float b2,
                       float eps, float wd, float c1, float c2, __nv_bfloat16* __restrict__ w_bf,
                       const float* __restrict__ hyper) {
    if (hyper) {
        lr = hyper[0];
        c1 = hyper[1];
        c2 = hyper[2];
    }
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = fmaf(b1, m[i], (1.0f - b1) * gi);
        const float vi = fmaf(b2, v[i], (1.0f - b2) * gi * gi);
        m[i] = mi;
        v[i] = vi;
        const float upd = (mi / c1) / (sqrtf(vi / c2) + eps) + wd * w[i];
        const float wi = w[i] - lr * upd;
        w[i] = wi;
        if (w_bf) w_bf[i] = __float2bfloat16_rn(wi);
    }
}

// One training step's schedule on the device (for graph-replayed steps):
// step += 1; hyper = {lr0 (1 + cos(pi (step - 1 - first) / total)) / 2,
// 1 - beta1^step, 1 - beta2^step} (the cosine schedule of a run that began
// after step `first`, and Adam's bias corrections, as the host computes them
// for qssb_adam).
__global__ void k_adam_schedule(float* __restrict__ hyper, int* __restrict__ step, int first,
                                int total, float lr0, float beta1, float beta2) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const int t = *step + 1;
    *step = t;
    const double frac = (double)(t - 1 - first) / (double)total;
    hyper[0] = (float)((double)lr0 * 0.5 * (1.0 + cos(3.141592653589793 * frac)));
    hyper[1] = 1.0f - powf(beta1, (float)t);
    hyper[2] = 1.0f - powf(beta2, (float)t);
}

__global__ void k_to_bf16(const float* __restrict__ x, long long n, __nv_bfloat16* __restrict__ y) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        y[i] = __float2bfloat16_rn(x[i]);
}

static int grid_for(long long n) {
    long long g = (n + 255) / 256;
    const long long cap = 148LL * 16;
    return (int)(g < 1 ? 1 : (g > cap ? cap : g));
}

}  // namespace qssb

using namespace qssb;

extern "C" int qssb_gemm_bf16(const void* A, int32_t lda, int32_t trans_a, const void* B,
                              int32_t ldb, int32_t trans_b, int32_t M, int32_t N, int32_t K,
                              const float* bias, int32_t accumulate, float* C, int32_t ldc,
                              void* act_bf16, int32_t ld_act, void* stream) {
    if (!A || !B || (!C && !act_bf16))
        return set_error(QSSB_ERR_INVALID, "qssb_gemm_bf16: null operand or no output");
    if (M <= 0 || N <= 0 || K <= 0 || (M % 16) || (N % 16) || (K % 16))
        return set_error(QSSB_ERR_INVALID, "qssb_gemm_bf16: M, N, K must be positive multiples of 16");
    const int rows_a = trans_a ? K : M, cols_a = trans_a ? M : K;
    const int rows_b = trans_b ? N : K, cols_b = trans_b ? K : N;
    (void)rows_a;
    (void)rows_b;
    if (lda < cols_a || ldb < cols_b || (C && ldc < N) || (act_bf16 && ld_act < N) ||
        (lda % 8) || (ldb % 8))
        return set_error(QSSB_ERR_INVALID, "qssb_gemm_bf16: leading dimensions too small or not multiples of 8");
    if (((uintptr_t)A & 31u) || ((uintptr_t)B & 31u))
        return set_error(QSSB_ERR_INVALID, "qssb_gemm_bf16: A and B must be 32-byte aligned");
    const dim3 grid((N + kGemmCtaTile - 1) / kGemmCtaTile, (M + kGemmCtaTile - 1) / kGemmCtaTile);
    const auto* a = static_cast<const __nv_bfloat16*>(A);
    const auto* b = static_cast<const __nv_bfloat16*>(B);
    auto* act = static_cast<__nv_bfloat16*>(act_bf16);
    cudaStream_t s = (cudaStream_t)stream;
    if (trans_a) {
        if (trans_b) { k_gemm_bf16<true, true><<<grid, 128, 0, s>>>(a, lda, b, ldb, M, N, K, bias, accumulate, C, ldc, act, ld_act); note_launch(); }
        else { k_gemm_bf16<true, false><<<grid, 128, 0, s>>>(a, lda, b, ldb, M, N, K, bias, accumulate, C, ldc, act, ld_act); note_launch(); }
    } else {
        if (trans_b) { k_gemm_bf16<false, true><<<grid, 128, 0, s>>>(a, lda, b, ldb, M, N, K, bias, accumulate, C, ldc, act, ld_act); note_launch(); }
        else { k_gemm_bf16<false, false><<<grid, 128, 0, s>>>(a, lda, b, ldb, M, N, K, bias, accumulate, C, ldc, act, ld_act); note_launch(); }
    }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}

extern "C" int qssb_gelu_backward(const float* dy, const float* pre, int64_t n, void* dz_bf16,
                                  float* dz, void* stream) {
    if (!dy || !pre || !dz_bf16 || !dz || n <= 0)
        return set_error(QSSB_ERR_INVALID, "qssb_gelu_backward: null pointer or empty");
    { k_gelu_backward<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(
        dy, pre, n, static_cast<__nv_bfloat16*>(dz_bf16), dz); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}

extern "C" int qssb_bias_grad(const float* dz, int32_t rows, int32_t cols, float* db, void* stream) {
    if (!dz || !db || rows <= 0 || cols <= 0)
        return set_error(QSSB_ERR_INVALID, "qssb_bias_grad: null pointer or empty");
    { k_bias_grad<<<(cols + 31) / 32, 32 * kBiasWarps, 0, (cudaStream_t)stream>>>(dz, rows, cols, db); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}

extern "C" int qssb_mse(const float* y, const float* target, int32_t rows, int32_t n_out,
                        int32_t ld, float* dy, float* loss, void* stream) {
    if (!y || !target || !dy || rows <= 0 || n_out <= 0 || ld < n_out)
        return set_error(QSSB_ERR_INVALID, "qssb_mse: null pointer or bad shape");
    { k_mse<<<1, 256, 0, (cudaStream_t)stream>>>(y, target, rows, n_out, ld, dy, loss); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}

extern "C" int qssb_mse_heads(const float* y, const float* target, int32_t rows, int32_t n_out,
                              int32_t heads, int32_t ld, const float* out_weight,
                              int32_t n_select, float eps, float* dy, float* loss,
                              int32_t* winner, void* stream) {
    if (!y || !target || !dy || rows <= 0 || n_out <= 0 || heads <= 0 ||
        (int64_t)heads * n_out > ld || n_select <= 0 || n_select > n_out)
        return set_error(QSSB_ERR_INVALID, "qssb_mse_heads: null pointer or bad shape");
    if (!(eps >= 0.0f && eps < 1.0f))
        return set_error(QSSB_ERR_INVALID, "qssb_mse_heads: eps must be in [0, 1)");
    { k_mse_heads<<<1, 256, 0, (cudaStream_t)stream>>>(y, target, rows, n_out, heads, ld,
                                                      out_weight, n_select, eps, dy, loss,
                                                      winner); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}

extern "C" int qssb_adam(float* w, float* m, float* v, const float* grad, int64_t n, float lr,
                         float beta1, float beta2, float eps, float weight_decay, int32_t step,
                         void* w_bf16, void* stream) {
    if (!w || !m || !v || !grad || n <= 0 || step < 1)
        return set_error(QSSB_ERR_INVALID, "qssb_adam: null pointer, empty or step < 1");
    const float c1 = 1.0f - powf(beta1, (float)step);
    const float c2 = 1.0f - powf(beta2, (float)step);
    { k_adam<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(
        w, m, v, grad, n, lr, beta1, beta2, eps, weight_decay, c1, c2,
        static_cast<__nv_bfloat16*>(w_bf16), nullptr); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}

extern "C" int qssb_adam_schedule(float* hyper, int32_t* step, int32_t first_step,
                                  int32_t total_steps, float lr0, float beta1, float beta2,
                                  void* stream) {
    if (!hyper || !step || total_steps <= 0 || first_step < 0)
        return set_error(QSSB_ERR_INVALID,
                         "qssb_adam_schedule: null pointer, total_steps < 1 or first_step < 0");
    { k_adam_schedule<<<1, 32, 0, (cudaStream_t)stream>>>(hyper, step, first_step, total_steps, lr0,
                                                         beta1, beta2); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}

extern "C" int qssb_adam_dev(float* w, float* m, float* v, const float* grad, int64_t n,
                             const float* hyper, float beta1, float beta2, float eps,
                             float weight_decay, void* w_bf16, void* stream) {
    if (!w || !m || !v || !grad || !hyper || n <= 0)
        return set_error(QSSB_ERR_INVALID, "qssb_adam_dev: null pointer or empty");
    { k_adam<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(
        w, m, v, grad, n, 0.0f, beta1, beta2, eps, weight_decay, 1.0f, 1.0f,
        static_cast<__nv_bfloat16*>(w_bf16), hyper); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}

extern "C" int qssb_to_bf16(const float* x, int64_t n, void* y, void* stream) {
    if (!x || !y || n <= 0) return set_error(QSSB_ERR_INVALID, "qssb_to_bf16: null pointer or empty");
    { k_to_bf16<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(x, n, static_cast<__nv_bfloat16*>(y)); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}
