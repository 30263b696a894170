// qssb_box.cu - the BF columns written by the frame-sum pass itself.
//
// The cold path reads every count once for the exact u64 frame sums and,
// after the BF selection, again for the BF-column gather (whole 128-byte
// lines of every detector row the disk touches: 198 MB at 128^4 for 58 MB of
// BF data). Here a superset box of the disk is estimated first from the sums
// of the first frames, and the sum pass writes the box's columns
// ([box pixel][frame], u16) while it streams the counts; after the real
// selection a map from BF index to box pixel replaces the gather. A BF pixel
// outside the box (a disk that moved, an explicit larger bf_radius) clears
// the map's ok flag and the caller gathers as before, so the result never
// depends on the estimate.
//
// Box record (device int32[8]): r0, r1, c0, c1 (rows [r0, r1), columns
// [c0, c1), c0 and c1 multiples of 8), width c1 - c0, pixel count, valid,
// unused.
#include "qssb_internal.h"

using namespace qssb;

namespace {

constexpr int kBoxThreads = 1024;

// Largest sum, then the bounding box of the pixels at >= 1/4 of it (or, with
// radius_px > 0, their centroid +- radius), widened by margin, clamped, and
// its columns rounded out to 8 pixels.
__global__ void __launch_bounds__(kBoxThreads) k_box_estimate(
    const unsigned long long* __restrict__ sums, int k0, int k1, float radius_px, int margin,
    long long capacity, int* __restrict__ box) {
    __shared__ unsigned long long s_max[kBoxThreads / 32];
    __shared__ int s_box[4][kBoxThreads / 32];
    __shared__ double s_cen[3][kBoxThreads / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int npix = k0 * k1;
    unsigned long long m = 0;
    for (int p = tid; p < npix; p += kBoxThreads) m = max(m, sums[p]);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, off));
    if (lane == 0) s_max[warp] = m;
    __syncthreads();
    if (tid < 32) {
        unsigned long long v = s_max[tid];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, off));
        if (tid == 0) s_max[0] = v;
    }
    __syncthreads();
    const unsigned long long mx = s_max[0];
    int rmin = k0, rmax = -1, cmin = k1, cmax = -1;
    double sw = 0.0, sr = 0.0, sc = 0.0;
    for (int p = tid; p < npix; p += kBoxThreads) {
        if (mx > 0 && sums[p] >= (mx + 3) / 4) {
            const int r = p / k1, c = p - r * k1;
            rmin = min(rmin, r);
            rmax = max(rmax, r);
            cmin = min(cmin, c);
            cmax = max(cmax, c);
            sw += 1.0;
            sr += r;
            sc += c;
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        rmin = min(rmin, __shfl_xor_sync(0xffffffffu, rmin, off));
        rmax = max(rmax, __shfl_xor_sync(0xffffffffu, rmax, off));
        cmin = min(cmin, __shfl_xor_sync(0xffffffffu, cmin, off));
        cmax = max(cmax, __shfl_xor_sync(0xffffffffu, cmax, off));
        sw += __shfl_xor_sync(0xffffffffu, sw, off);
        sr += __shfl_xor_sync(0xffffffffu, sr, off);
        sc += __shfl_xor_sync(0xffffffffu, sc, off);
    }
    if (lane == 0) {
        s_box[0][warp] = rmin;
        s_box[1][warp] = rmax;
        s_box[2][warp] = cmin;
        s_box[3][warp] = cmax;
        s_cen[0][warp] = sw;
        s_cen[1][warp] = sr;
        s_cen[2][warp] = sc;
    }
    __syncthreads();
    if (tid != 0) return;
    rmin = k0, rmax = -1, cmin = k1, cmax = -1;
    sw = sr = sc = 0.0;
    for (int w = 0; w < kBoxThreads / 32; ++w) {
        rmin = min(rmin, s_box[0][w]);
        rmax = max(rmax, s_box[1][w]);
        cmin = min(cmin, s_box[2][w]);
        cmax = max(cmax, s_box[3][w]);
        sw += s_cen[0][w];
        sr += s_cen[1][w];
        sc += s_cen[2][w];
    }
    int r0, r1, c0, c1;
    if (rmax < 0) {
        r0 = r1 = c0 = c1 = 0;
    } else if (radius_px > 0.0f) {
        const double cr = sr / sw, cc = sc / sw, ext = (double)radius_px + margin;
        r0 = (int)floor(cr - ext);
        r1 = (int)ceil(cr + ext) + 1;
        c0 = (int)floor(cc - ext);
        c1 = (int)ceil(cc + ext) + 1;
    } else {
        r0 = rmin - margin;
        r1 = rmax + 1 + margin;
        c0 = cmin - margin;
        c1 = cmax + 1 + margin;
    }
    r0 = max(r0, 0);
    r1 = min(r1, k0);
    c0 = max(c0, 0) & ~7;
    c1 = min((c1 + 7) & ~7, k1);
    const long long n = (r1 > r0 && c1 > c0) ? (long long)(r1 - r0) * (c1 - c0) : 0;
    box[0] = r0;
    box[1] = r1;
    box[2] = c0;
    box[3] = c1;
    box[4] = c1 - c0;
    box[5] = (int)n;
    box[6] = (n > 0 && n <= capacity) ? 1 : 0;
    box[7] = 0;
}

// u64 frame sums as k_sum_frames_vec8 (one thread: 8 pixels, a chunk of
// frames; frames_per_chunk a multiple of 8) and, for vectors inside the box,
// the 8 x 8 (frames x pixels) u16 tile transposed in registers (byte
// permutes) and stored as one 16-byte run of 8 frames per pixel.
constexpr int kSumBoxThreads = 256;

// A box record is used only if it is valid and consistent: inside the
// detector, 8-pixel columns, its pixel count within the buffer's capacity.
__device__ __forceinline__ bool box_usable(const int* box, int k0, int k1, long long capacity) {
    return box[6] != 0 && box[0] >= 0 && box[1] <= k0 && box[0] < box[1] && box[2] >= 0 &&
           box[3] <= k1 && box[2] < box[3] && (box[2] & 7) == 0 && (box[3] & 7) == 0 &&
           box[4] == box[3] - box[2] && (long long)box[5] == (long long)(box[1] - box[0]) * box[4] &&
           (long long)box[5] <= capacity;
}

__global__ void __launch_bounds__(kSumBoxThreads) k_sum_frames_box(
    const uint4* __restrict__ counts, long long n_frames, int nvec, int k0, int k1,
    int frames_per_chunk, unsigned long long* __restrict__ sums, const int* __restrict__ box,
    long long capacity, uint16_t* __restrict__ box_cols) {
    const int vec = blockIdx.x * kSumBoxThreads + threadIdx.x;
    if (vec >= nvec) return;
    const long long f0 = (long long)blockIdx.y * frames_per_chunk;
    long long f1 = f0 + frames_per_chunk;
    if (f1 > n_frames) f1 = n_frames;
    const int p0 = vec * 8;
    const int row = p0 / k1, col = p0 - row * k1;
    const bool in_box = box_usable(box, k0, k1, capacity) && row >= box[0] && row < box[1] &&
                        col >= box[2] && col < box[3];
    uint4* out = nullptr;  // this vector's 8 box columns, frame f0 onwards
    long long stride = 0;  // one box column, in uint4 (8 frames)
    if (in_box) {
        const long long bp = (long long)(row - box[0]) * box[4] + (col - box[2]);
        stride = n_frames / 8;
        out = reinterpret_cast<uint4*>(box_cols + bp * n_frames + f0);
    }
    uint32_t acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    auto add = [&](uint4 v) {
        acc[0] += v.x & 0xffffu; acc[1] += v.x >> 16;
        acc[2] += v.y & 0xffffu; acc[3] += v.y >> 16;
        acc[4] += v.z & 0xffffu; acc[5] += v.z >> 16;
        acc[6] += v.w & 0xffffu; acc[7] += v.w >> 16;
    };
    const uint4* p = counts + f0 * (long long)nvec + vec;
    long long f = f0;
    for (; f + 8 <= f1; f += 8) {
        uint4 v[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] = __ldcs(p + j * (long long)nvec);
        p += 8 * (long long)nvec;
#pragma unroll
        for (int j = 0; j < 8; ++j) add(v[j]);
        if (in_box) {
            // word w of frame j holds pixels 2w (low) and 2w + 1 (high)
            const uint32_t* wv = reinterpret_cast<const uint32_t*>(v);
#pragma unroll
            for (int w = 0; w < 4; ++w) {
                uint4 lo, hi;
                lo.x = __byte_perm(wv[0 * 4 + w], wv[1 * 4 + w], 0x5410);
                hi.x = __byte_perm(wv[0 * 4 + w], wv[1 * 4 + w], 0x7632);
                lo.y = __byte_perm(wv[2 * 4 + w], wv[3 * 4 + w], 0x5410);
                hi.y = __byte_perm(wv[2 * 4 + w], wv[3 * 4 + w], 0x7632);
                lo.z = __byte_perm(wv[4 * 4 + w], wv[5 * 4 + w], 0x5410);
                hi.z = __byte_perm(wv[4 * 4 + w], wv[5 * 4 + w], 0x7632);
                lo.w = __byte_perm(wv[6 * 4 + w], wv[7 * 4 + w], 0x5410);
                hi.w = __byte_perm(wv[6 * 4 + w], wv[7 * 4 + w], 0x7632);
                out[(2 * w) * stride] = lo;
                out[(2 * w + 1) * stride] = hi;
            }
            ++out;
        }
    }
    for (; f < f1; ++f) {  // a partial last group (n_frames not a multiple of 8)
        const uint4 v = __ldcs(p);
        p += nvec;
        add(v);
        if (in_box) {
            uint16_t* o = box_cols + ((long long)(row - box[0]) * box[4] + (col - box[2])) * n_frames + f;
            const uint32_t w4[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int q = 0; q < 8; ++q) o[q * n_frames] = (uint16_t)(w4[q >> 1] >> (16 * (q & 1)));
        }
    }
#pragma unroll
    for (int i = 0; i < 8; ++i)
        if (acc[i]) atomicAdd(&sums[vec * 8 + i], (unsigned long long)acc[i]);
}

// map[b] = box pixel of BF pixel b (-1 outside); ok = every BF pixel inside.
__global__ void __launch_bounds__(kBoxThreads) k_box_map(
    const int32_t* __restrict__ bf_linear, const qssb_bf_info_t* __restrict__ info, int k0, int k1,
    int capacity, long long box_capacity, const int* __restrict__ box, int32_t* __restrict__ map,
    int* __restrict__ ok) {
    const int n_bf = info->n_bf;
    const bool usable = box_usable(box, k0, k1, box_capacity);
    int inside = usable && n_bf > 0 && n_bf <= capacity;
    for (int b = threadIdx.x; b < n_bf && b < capacity; b += kBoxThreads) {
        const int p = bf_linear[b];
        const int r = p / k1, c = p - r * k1;
        int m = -1;
        if (usable && r >= box[0] && r < box[1] && c >= box[2] && c < box[3])
            m = (r - box[0]) * box[4] + (c - box[2]);
        map[b] = m;
        inside &= (m >= 0);
    }
    inside = __syncthreads_and(inside);
    if (threadIdx.x == 0) *ok = inside;
}

}  // namespace

extern "C" int qssb_bf_box_estimate(const uint64_t* sums, int32_t det_rows, int32_t det_cols,
                                    float radius_px, int32_t margin, int64_t capacity,
                                    int32_t* box, void* stream) {
    if (!sums || !box || det_rows <= 0 || det_cols <= 0 || margin < 0 || capacity < 0)
        return set_error(QSSB_ERR_INVALID, "qssb_bf_box_estimate: invalid arguments");
    if ((int64_t)det_rows * det_cols > (1 << 26))
        return set_error(QSSB_ERR_UNSUPPORTED, "qssb_bf_box_estimate: detector too large");
    { k_box_estimate<<<1, kBoxThreads, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<const unsigned long long*>(sums), det_rows, det_cols, radius_px, margin,
        capacity, box); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}

extern "C" int qssb_mean_dp_u64_box(const uint16_t* counts, int64_t n_frames, int32_t det_rows,
                                    int32_t det_cols, uint64_t* sums, const int32_t* box,
                                    int64_t capacity, uint16_t* box_cols, void* stream) {
    if (!counts || !sums || !box || !box_cols || n_frames <= 0 || det_rows <= 0 || det_cols <= 0 ||
        capacity < 0)
        return set_error(QSSB_ERR_INVALID, "qssb_mean_dp_u64_box: null pointer or empty shape");
    if (det_cols % 8 != 0 || n_frames % 8 != 0 || ((uintptr_t)counts & 15u) ||
        ((uintptr_t)box_cols & 15u))
        return set_error(QSSB_ERR_UNSUPPORTED,
                         "qssb_mean_dp_u64_box: needs det_cols and n_frames multiples of 8 and "
                         "16-byte aligned counts and box columns");
    if (n_frames > (int64_t)1 << 40)
        return set_error(QSSB_ERR_INVALID, "qssb_mean_dp_u64_box: n_frames too large");
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t det_pixels = (int64_t)det_rows * det_cols;
    CUDA_TRY(cudaMemsetAsync(sums, 0, sizeof(uint64_t) * (size_t)det_pixels, s));
    const int nvec = (int)(det_pixels / 8);
    const int gx = (nvec + kSumBoxThreads - 1) / kSumBoxThreads;
    long long want = (long long)device_sm_count() * 16 / gx;
    if (want < 1) want = 1;
    long long chunk = (n_frames + want - 1) / want;
    chunk = (chunk + 7) & ~7LL;
    if (chunk > 32768) chunk = 32768;
    if (chunk < 8) chunk = 8;
    const long long gy = (n_frames + chunk - 1) / chunk;
    if (gy > 65535) return set_error(QSSB_ERR_INVALID, "qssb_mean_dp_u64_box: too many frames");
    { k_sum_frames_box<<<dim3(gx, (unsigned)gy), kSumBoxThreads, 0, s>>>(
        reinterpret_cast<const uint4*>(counts), n_frames, nvec, det_rows, det_cols, (int)chunk,
        reinterpret_cast<unsigned long long*>(sums), box, (long long)capacity, box_cols); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}

extern "C" int qssb_bf_box_map(const int32_t* bf_linear, const qssb_bf_info_t* info,
                               int32_t det_rows, int32_t det_cols, int32_t capacity,
                               int64_t box_capacity, const int32_t* box, int32_t* map,
                               int32_t* ok, void* stream) {
    if (!bf_linear || !info || !box || !map || !ok || det_rows <= 0 || det_cols <= 0 ||
        capacity <= 0 || box_capacity < 0)
        return set_error(QSSB_ERR_INVALID, "qssb_bf_box_map: invalid arguments");
    { k_box_map<<<1, kBoxThreads, 0, (cudaStream_t)stream>>>(bf_linear, info, det_rows, det_cols,
                                                           capacity, (long long)box_capacity, box,
                                                           map, ok); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}
