// qssb_temporal.cu - joining a time series of SSB object waves (sm_100a).
//
// Restates the drift-corrected complex mean of the reference's temporal
// helpers (ssb/temporal.py:77-257 of bobleesj/quantem.gpu):
//   fourier_shift: O'_t = ifft2(fft2(O_t) exp(-2 pi i (f_r s_r + f_c s_c))),
//     f = fftfreq(n, 1) (temporal.py:77-107), as three passes over the stack:
//     row FFTs; per column strip: FFT along the rows, the ramp, inverse FFT;
//     inverse row FFTs with the 1 / (R C) scale;
//   join: with phase reference "first", frames t > 0 are multiplied by
//     exp(-i angle(sum_p O'_t conj O'_0)) (temporal.py:154-160; the overlap
//     summed in FP64 in a fixed order), then joined = sum_t w_t O'_t
//     (temporal.py:234).
// Line transforms: the warp FFT at 256..1024 points, the shared-memory
// Stockham transform at 64 and 128.
#include <math.h>

#include "qssb_internal.h"

namespace qssb {

constexpr int kTmpWarps = 8;

template <int N>
__host__ __device__ constexpr int tmp_line() {
    // room for the line and, at N >= 256, the warp FFT's transpose scratch
    return N >= 256 ? (warp_fft_scratch<N>() > N ? warp_fft_scratch<N>() : N) : N;
}

// In-place transform of one line held in shared memory (natural order).
template <int N, int DIR>
__device__ __forceinline__ void line_transform(float2* line, const float2* tw, int lane) {
    if constexpr (N >= 256) {
        constexpr int RPL = N / 32;
        float2 v[RPL];
#pragma unroll
        for (int t = 0; t < RPL; ++t) v[t] = line[lane + 32 * t];
        __syncwarp();
        warp_fft<N, DIR>(v, line, tw, lane);
#pragma unroll
        for (int j = 0; j < RPL; ++j) line[warp_fft_index<N>(lane, j)] = v[j];
        __syncwarp();
    } else {
        line_fft<N, DIR>(line, 1, tw, lane);
    }
}

// One warp per row of every frame: out = (scale) * FFT_DIR(row of in).
template <int C, int DIR>
__global__ void __launch_bounds__(32 * kTmpWarps) k_tmp_rows(const float2* __restrict__ in,
                                                             float2* __restrict__ out, int rows,
                                                             float scale) {
    constexpr int L = tmp_line<C>();
    extern __shared__ float2 tmp_rows_smem[];
    float2* tw = tmp_rows_smem;
    float2* lines = tw + C;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    fill_twiddles<C>(tw, tid, 32 * kTmpWarps);
    __syncthreads();
    const int r = blockIdx.x * kTmpWarps + warp;
    if (r >= rows) return;
    const size_t base = ((size_t)blockIdx.y * rows + r) * C;
    float2* line = lines + warp * L;
    for (int i = lane; i < C; i += 32) line[i] = in[base + i];
    __syncwarp();
    line_transform<C, DIR>(line, tw, lane);
    for (int i = lane; i < C; i += 32) {
        const float2 v = line[i];
        out[base + i] = make_float2(v.x * scale, v.y * scale);
    }
}

// Per strip of columns of every frame: FFT along the rows, the frame's
// shift ramp, inverse FFT along the rows (in place). The ramp phase
// -2 pi (f_r s_r + f_c s_c) is formed in FP64 and reduced before the
// float32 sincos.
template <int R>
__global__ void __launch_bounds__(32 * kTmpWarps) k_tmp_cols(float2* __restrict__ data, int cols,
                                                             const float* __restrict__ shifts) {
    constexpr int L = tmp_line<R>();
    constexpr int P = L | 1;
    extern __shared__ float2 tmp_cols_smem[];
    float2* tile = tmp_cols_smem;
    float2* tw = tile + kTmpWarps * P;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int frame = blockIdx.y;
    const int c0 = blockIdx.x * kTmpWarps;
    const int nc = min(kTmpWarps, cols - c0);
    fill_twiddles<R>(tw, tid, 32 * kTmpWarps);
    float2* d = data + (size_t)frame * R * cols;
    for (int e = tid; e < R * kTmpWarps; e += 32 * kTmpWarps) {
        const int r = e / kTmpWarps;
        const int c = e - r * kTmpWarps;
        if (c < nc) tile[c * P + r] = d[(size_t)r * cols + c0 + c];
    }
    __syncthreads();
    if (warp < nc) {
        float2* line = tile + warp * P;
        line_transform<R, -1>(line, tw, lane);
        const double sr = (double)__ldg(shifts + 2 * frame);
        const double sc = (double)__ldg(shifts + 2 * frame + 1);
        const int c = c0 + warp;
        const double fc = (double)(c < (cols + 1) / 2 ? c : c - cols) / (double)cols;
        for (int r = lane; r < R; r += 32) {
            const double fr = (double)(r < (R + 1) / 2 ? r : r - R) / (double)R;
            double ph = -(fr * sr + fc * sc);  // in turns
            ph -= rint(ph);
            float s, co;
            sincospif((float)(2.0 * ph), &s, &co);
            line[r] = cmul(line[r], make_float2(co, s));
        }
        __syncwarp();
        line_transform<R, +1>(line, tw, lane);
    }
    __syncthreads();
    for (int e = tid; e < R * kTmpWarps; e += 32 * kTmpWarps) {
        const int r = e / kTmpWarps;
        const int c = e - r * kTmpWarps;
        if (c < nc) d[(size_t)r * cols + c0 + c] = tile[c * P + r];
    }
}

constexpr int kJoinBlocks = 64;   // overlap partial sums per frame
constexpr int kJoinThreads = 256;

// partial[t][blk] = sum over this block's pixels of a_t conj(a_0), FP64.
__global__ void __launch_bounds__(kJoinThreads) k_overlap_partial(const float2* __restrict__ a,
                                                                  long long n_pix,
                                                                  double2* __restrict__ partial) {
    __shared__ double2 red[kJoinThreads];
    const int t = blockIdx.y;
    const float2* at = a + (size_t)t * n_pix;
    double sr = 0.0, si = 0.0;
    for (long long p = (long long)blockIdx.x * kJoinThreads + threadIdx.x; p < n_pix;
         p += (long long)kJoinBlocks * kJoinThreads) {
        const float2 v = at[p];
        const float2 r = a[p];
        sr += (double)v.x * r.x + (double)v.y * r.y;
        si += (double)v.y * r.x - (double)v.x * r.y;
    }
    red[threadIdx.x] = make_double2(sr, si);
    __syncthreads();
    for (int w = kJoinThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            red[threadIdx.x].x += red[threadIdx.x + w].x;
            red[threadIdx.x].y += red[threadIdx.x + w].y;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[(size_t)t * kJoinBlocks + blockIdx.x] = red[0];
}

// rot[t] = exp(-i angle(overlap_t)) for t > 0, 1 for frame 0.
__global__ void k_overlap_rotation(const double2* __restrict__ partial, int n_frames,
                                   float2* __restrict__ rot) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_frames) return;
    if (t == 0) {
        rot[0] = make_float2(1.0f, 0.0f);
        return;
    }
    double sr = 0.0, si = 0.0;
    for (int b = 0; b < kJoinBlocks; ++b) {
        sr += partial[(size_t)t * kJoinBlocks + b].x;
        si += partial[(size_t)t * kJoinBlocks + b].y;
    }
    const double ang = atan2(si, sr);
    rot[t] = make_float2((float)cos(ang), (float)-sin(ang));
}

// joined[p] = sum_t w_t rot_t a_t[p] (FP32, frames in order); the rotated
// frames are written back when requested.
__global__ void __launch_bounds__(kJoinThreads) k_join(float2* __restrict__ a,
                                                       const float* __restrict__ w,
                                                       const float2* __restrict__ rot,
                                                       int n_frames, long long n_pix,
                                                       float2* __restrict__ joined,
                                                       int write_back) {
    const long long p = (long long)blockIdx.x * kJoinThreads + threadIdx.x;
    if (p >= n_pix) return;
    float sr = 0.0f, si = 0.0f;
    for (int t = 0; t < n_frames; ++t) {
        float2 v = a[(size_t)t * n_pix + p];
        if (rot) v = cmul(v, __ldg(rot + t));
        if (write_back) a[(size_t)t * n_pix + p] = v;
        const float wt = __ldg(w + t);
        sr = fmaf(wt, v.x, sr);
        si = fmaf(wt, v.y, si);
    }
    joined[p] = make_float2(sr, si);
}

template <int C, int DIR>
static void launch_rows(const float2* in, float2* out, int n_frames, int rows, float scale,
                        cudaStream_t s) {
    const size_t smem = sizeof(float2) * ((size_t)kTmpWarps * tmp_line<C>() + C);
    cudaFuncSetAttribute(k_tmp_rows<C, DIR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    { k_tmp_rows<C, DIR><<<dim3((rows + kTmpWarps - 1) / kTmpWarps, n_frames), 32 * kTmpWarps, smem, s>>>(
        in, out, rows, scale); note_launch(); }
}

static int rows_pass(int cols, int dir, const float2* in, float2* out, int n_frames, int rows,
                     float scale, cudaStream_t s) {
    switch (cols) {
#define QSSB_ROWS_CASE(n)                                                              \
    case n:                                                                           \
        if (dir < 0) launch_rows<n, -1>(in, out, n_frames, rows, scale, s);            \
        else launch_rows<n, +1>(in, out, n_frames, rows, scale, s);                    \
        break;
        QSSB_ROWS_CASE(64)
        QSSB_ROWS_CASE(128)
        QSSB_ROWS_CASE(256)
        QSSB_ROWS_CASE(512)
        QSSB_ROWS_CASE(1024)
#undef QSSB_ROWS_CASE
        default:
            return set_error(QSSB_ERR_UNSUPPORTED, "qssb_fourier_shift: sizes must be 64..1024, powers of two");
    }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}

template <int R>
static int launch_cols(float2* data, int n_frames, int cols, const float* shifts, cudaStream_t s) {
    const size_t smem = sizeof(float2) * ((size_t)kTmpWarps * (tmp_line<R>() | 1) + R);
    CUDA_TRY(cudaFuncSetAttribute(k_tmp_cols<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    { k_tmp_cols<R><<<dim3((cols + kTmpWarps - 1) / kTmpWarps, n_frames), 32 * kTmpWarps, smem, s>>>(
        data, cols, shifts); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}

static bool tmp_size_ok(int n) {
    return n == 64 || n == 128 || n == 256 || n == 512 || n == 1024;
}

}  // namespace qssb

using namespace qssb;

extern "C" int qssb_fourier_shift(const float* in, float* out, int32_t n_frames, int32_t rows,
                                  int32_t cols, const float* shifts, void* stream) {
    if (!in || !out || !shifts || n_frames <= 0 || n_frames > 65535)
        return set_error(QSSB_ERR_INVALID, "qssb_fourier_shift: null pointer or n_frames outside [1, 65535]");
    if (!tmp_size_ok(rows) || !tmp_size_ok(cols))
        return set_error(QSSB_ERR_UNSUPPORTED, "qssb_fourier_shift: sizes must be 64..1024, powers of two");
    cudaStream_t s = (cudaStream_t)stream;
    auto* o = reinterpret_cast<float2*>(out);
    int rc = rows_pass(cols, -1, reinterpret_cast<const float2*>(in), o, n_frames, rows, 1.0f, s);
    if (rc) return rc;
    switch (rows) {
        case 64: rc = launch_cols<64>(o, n_frames, cols, shifts, s); break;
        case 128: rc = launch_cols<128>(o, n_frames, cols, shifts, s); break;
        case 256: rc = launch_cols<256>(o, n_frames, cols, shifts, s); break;
        case 512: rc = launch_cols<512>(o, n_frames, cols, shifts, s); break;
        default: rc = launch_cols<1024>(o, n_frames, cols, shifts, s); break;
    }
    if (rc) return rc;
    return rows_pass(cols, +1, o, o, n_frames, rows, 1.0f / ((float)rows * (float)cols), s);
}

extern "C" int qssb_join_workspace_bytes(int32_t n_frames, size_t* bytes) {
    if (!bytes || n_frames <= 0 || n_frames > 65535)
        return set_error(QSSB_ERR_INVALID, "qssb_join_workspace_bytes: n_frames must be in [1, 65535]");
    const size_t part = (sizeof(double2) * (size_t)n_frames * kJoinBlocks + 255) & ~(size_t)255;
    *bytes = part + sizeof(float2) * (size_t)n_frames;
    return QSSB_OK;
}

extern "C" int qssb_join_object_waves(float* frames, const float* weights, int32_t n_frames,
                                      int64_t n_pix, int32_t phase_reference, void* workspace,
                                      size_t workspace_bytes, float* joined, int32_t write_back,
                                      void* stream) {
    if (!frames || !weights || !joined || n_frames <= 0 || n_frames > 65535 || n_pix <= 0)
        return set_error(QSSB_ERR_INVALID, "qssb_join_object_waves: null pointer or empty shape");
    if (phase_reference != 0 && phase_reference != 1)
        return set_error(QSSB_ERR_INVALID, "qssb_join_object_waves: phase_reference must be 0 (none) or 1 (first)");
    cudaStream_t s = (cudaStream_t)stream;
    auto* a = reinterpret_cast<float2*>(frames);
    float2* rot = nullptr;
    if (phase_reference == 1) {
        size_t need = 0;
        int rc = qssb_join_workspace_bytes(n_frames, &need);
        if (rc) return rc;
        if (!workspace || workspace_bytes < need)
            return set_error(QSSB_ERR_WORKSPACE, "qssb_join_object_waves: workspace too small");
        if (((uintptr_t)workspace & 255u) != 0)
            return set_error(QSSB_ERR_INVALID, "qssb_join_object_waves: workspace must be 256-byte aligned");
        auto* partial = static_cast<double2*>(workspace);
        const size_t part = (sizeof(double2) * (size_t)n_frames * kJoinBlocks + 255) & ~(size_t)255;
        rot = reinterpret_cast<float2*>(static_cast<char*>(workspace) + part);
        { k_overlap_partial<<<dim3(kJoinBlocks, n_frames), kJoinThreads, 0, s>>>(a, n_pix, partial); note_launch(); }
        CUDA_TRY(cudaGetLastError());
        { k_overlap_rotation<<<(n_frames + 127) / 128, 128, 0, s>>>(partial, n_frames, rot); note_launch(); }
        CUDA_TRY(cudaGetLastError());
    }
    const long long blocks = (n_pix + kJoinThreads - 1) / kJoinThreads;
    if (blocks > 0x7fffffffLL) return set_error(QSSB_ERR_INVALID, "qssb_join_object_waves: too many pixels");
    { k_join<<<(unsigned)blocks, kJoinThreads, 0, s>>>(a, weights, rot, n_frames, n_pix,
                                                     reinterpret_cast<float2*>(joined), write_back); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}
