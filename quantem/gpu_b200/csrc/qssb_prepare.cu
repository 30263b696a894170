// qssb_prepare.cu - dataset preparation: exact u64 mean diffraction pattern,
// BF-column gather and the per-BF Hermitian scan FFT (sm_100a).
//
// HBM layout: counts[f][k] u16 with k = k_row * K1 + k_col contiguous per
// frame (the reference's data.reshape(-1, K0, K1), backend.py:432); BF
// columns [b][f] u16 (BF-major, one 32 KB scan image per BF pixel at 128^2);
// spectra [b][r][c] complex64 with c in [0, R1/2] (backend.py:547-554).
#include "qssb_internal.h"

namespace qssb {

// --------------------------------------------------------------- mean DP
// Each thread owns 8 detector pixels (one 16-byte vector per frame) and a
// contiguous range of frames; u32 partials (<= 65536 frames * 65535 fits)
// are folded into the u64 sums with one atomic per pixel per chunk. Integer
// addition commutes, so the result is exact and order-independent.
constexpr int kSumThreads = 256;

__global__ void __launch_bounds__(kSumThreads) k_sum_frames_vec8(
    const uint4* __restrict__ counts, long long n_frames, int nvec, int frames_per_chunk,
    unsigned long long* __restrict__ sums) {
    const int vec = blockIdx.x * kSumThreads + threadIdx.x;
    if (vec >= nvec) return;
    const long long f0 = (long long)blockIdx.y * frames_per_chunk;
    long long f1 = f0 + frames_per_chunk;
    if (f1 > n_frames) f1 = n_frames;
    uint32_t acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const uint4* p = counts + f0 * (long long)nvec + vec;
    long long f = f0;
    auto add = [&](uint4 v) {
        acc[0] += v.x & 0xffffu; acc[1] += v.x >> 16;
        acc[2] += v.y & 0xffffu; acc[3] += v.y >> 16;
        acc[4] += v.z & 0xffffu; acc[5] += v.z >> 16;
        acc[6] += v.w & 0xffffu; acc[7] += v.w >> 16;
    };
    for (; f + 4 <= f1; f += 4) {
        const uint4 v0 = __ldcs(p);
        const uint4 v1 = __ldcs(p + nvec);
        const uint4 v2 = __ldcs(p + 2 * (long long)nvec);
        const uint4 v3 = __ldcs(p + 3 * (long long)nvec);
        p += 4 * (long long)nvec;
        add(v0); add(v1); add(v2); add(v3);
    }
    for (; f < f1; ++f) {
        add(__ldcs(p));
        p += nvec;
    }
#pragma unroll
    for (int i = 0; i < 8; ++i)
        if (acc[i]) atomicAdd(&sums[vec * 8 + i], (unsigned long long)acc[i]);
}

// Fallback for detector sizes that are not a multiple of 8 pixels or
// unaligned bases: one pixel per thread.
__global__ void k_sum_frames_scalar(const uint16_t* __restrict__ counts, long long n_frames,
                                    int npix, int frames_per_chunk,
                                    unsigned long long* __restrict__ sums) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= npix) return;
    const long long f0 = (long long)blockIdx.y * frames_per_chunk;
    long long f1 = f0 + frames_per_chunk;
    if (f1 > n_frames) f1 = n_frames;
    uint32_t acc = 0;
    for (long long f = f0; f < f1; ++f) acc += counts[f * npix + k];
    if (acc) atomicAdd(&sums[k], (unsigned long long)acc);
}

__global__ void k_mean_from_sums(const unsigned long long* __restrict__ sums, int npix,
                                 float n_frames_f, float* __restrict__ mean_dp) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < npix) mean_dp[k] = __fdiv_rn(__ull2float_rn(sums[k]), n_frames_f);
}

// ---------------------------------------------------------------- gather
// Tile of 64 frames x 64 BF pixels through shared memory: each warp reads 32
// BF entries of one frame (mostly contiguous within a detector row) and
// writes 64 consecutive frames (128 bytes) of one BF column.
constexpr int kGatherF = 64;
constexpr int kGatherB = 64;

__global__ void __launch_bounds__(256) k_gather_columns(
    const uint16_t* __restrict__ counts, long long n_frames, int npix,
    const int32_t* __restrict__ bf_linear, int n_bf, uint16_t* __restrict__ columns) {
    __shared__ uint16_t tile[kGatherB][kGatherF + 2];
    const int tid = threadIdx.x;
    const long long f0 = (long long)blockIdx.x * kGatherF;
    const int b0 = blockIdx.y * kGatherB;
    const int bl = tid & (kGatherB - 1);
    const int b = b0 + bl;
    const int lin = b < n_bf ? __ldg(bf_linear + b) : 0;
    // an index outside the detector reads nothing (its column stays zero);
    // the host wrapper rejects such indices before launch
    const bool ok = b < n_bf && lin >= 0 && lin < npix;
    for (int fl = tid >> 6; fl < kGatherF; fl += 4) {
        const long long f = f0 + fl;
        uint16_t v = 0;
        if (ok && f < n_frames) v = __ldcs(counts + f * npix + lin);
        tile[bl][fl] = v;
    }
    __syncthreads();
    // write: 64 BF rows x 32 u32 words (2 frames each)
    const bool full = (f0 + kGatherF <= n_frames) && ((n_frames & 1) == 0);
    for (int w = tid; w < kGatherB * (kGatherF / 2); w += 256) {
        const int row = w >> 5;
        const int word = w & 31;
        const int bb = b0 + row;
        if (bb >= n_bf) continue;
        const long long f = f0 + 2 * word;
        uint16_t* dst = columns + (long long)bb * n_frames + f;
        if (full) {
            const uint32_t packed = (uint32_t)tile[row][2 * word] | ((uint32_t)tile[row][2 * word + 1] << 16);
            *reinterpret_cast<uint32_t*>(dst) = packed;
        } else {
            if (f < n_frames) dst[0] = tile[row][2 * word];
            if (f + 1 < n_frames) dst[1] = tile[row][2 * word + 1];
        }
    }
}

// ----------------------------------------------------- Hermitian scan FFT
// One CTA per BF image (N x N real). Rows 2j and 2j+1 are packed as the real
// and imaginary parts of one complex line, transformed together and split:
// X_2j(c) = (Z(c) + conj Z(-c)) / 2, X_2j+1(c) = (Z(c) - conj Z(-c)) / (2i),
// keeping c in [0, N/2]. The N/2+1 columns are then transformed along rows.
template <int N>
struct ScanFftSmem {
    static constexpr int H = N / 2 + 1;
    static constexpr int PP = N + 1;          // packed-line pitch (odd)
    static constexpr int HP = H;              // half-plane pitch (odd for N=128,256)
    static constexpr size_t bytes = sizeof(float2) * ((size_t)(N / 2) * PP + (size_t)N * HP + N);
};

template <int N>
__global__ void __launch_bounds__(512, 1) k_scan_fft_half(const uint16_t* __restrict__ columns,
                                                          int n_bf, float2* __restrict__ g_half) {
    using S = ScanFftSmem<N>;
    extern __shared__ float2 smem[];
    float2* packed = smem;                         // [N/2][PP]
    float2* half = packed + (N / 2) * S::PP;       // [N][HP]
    float2* tw = half + N * S::HP;                 // [N]
    const int b = blockIdx.x;
    if (b >= n_bf) return;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    constexpr int NW = 16;
    fill_twiddles<N>(tw, tid, 512);
    // load N*N u16 as uint4 (8 values), pack row pairs
    const uint4* src = reinterpret_cast<const uint4*>(columns + (size_t)b * N * N);
    constexpr int NV = N * N / 8;
    for (int i = tid; i < NV; i += 512) {
        const uint4 v = __ldcs(src + i);
        const int e = i * 8;
        const int row = e / N;
        const int col = e % N;
        const int j = row >> 1;
        const bool odd = row & 1;
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float lo = (float)(w[q] & 0xffffu);
            const float hi = (float)(w[q] >> 16);
            float* d0 = reinterpret_cast<float*>(&packed[j * S::PP + col + 2 * q]);
            float* d1 = reinterpret_cast<float*>(&packed[j * S::PP + col + 2 * q + 1]);
            d0[odd ? 1 : 0] = lo;
            d1[odd ? 1 : 0] = hi;
        }
    }
    __syncthreads();
    for (int j = warp; j < N / 2; j += NW) {
        float2* line = packed + j * S::PP;
        line_fft<N, -1>(line, 1, tw, lane);
        for (int c = lane; c < S::H; c += 32) {
            const float2 z = line[c];
            const float2 zm = line[(N - c) & (N - 1)];
            // even = (z + conj zm)/2 ; odd = (z - conj zm)/(2i)
            const float2 ev = make_float2(0.5f * (z.x + zm.x), 0.5f * (z.y - zm.y));
            const float2 od = make_float2(0.5f * (z.y + zm.y), -0.5f * (z.x - zm.x));
            half[(2 * j) * S::HP + c] = ev;
            half[(2 * j + 1) * S::HP + c] = od;
        }
    }
    __syncthreads();
    for (int c = warp; c < S::H; c += NW) line_fft<N, -1>(half + c, S::HP, tw, lane);
    __syncthreads();
    float2* dst = g_half + (size_t)b * N * S::H;
    for (int i = tid; i < N * S::H; i += 512) {
        const int r = i / S::H;
        const int c = i - r * S::H;
        dst[i] = half[r * S::HP + c];
    }
}

// 128 x 128 scan FFT: persistent CTAs of 256 threads (32 groups of 8 lanes),
// two per SM (106 KB of shared memory each, so one CTA's barriers overlap
// the other's work), loop over BF images. Per image:
//  1. the u16 image is in shared memory (rows padded to 136 u16), copied in
//     by cp.async (16-byte global -> shared copies, L1 bypassed) while the
//     previous image's spectrum was stored; each group reads its two row
//     pairs (j = g, g + 32) into registers, after which the image region
//     serves as the groups' FFT scratch;
//  2. row pairs 2j, 2j+1 are transformed packed as one complex line
//     (fft128_g8) and split into the two real spectra of the half plane H
//     ([128][65], pitch 65);
//  3. the 65 columns of H are transformed in place, two jobs per group:
//     columns 0 and 64 (the DC and Nyquist bins of real rows) are real, so
//     they go packed as Z = H(:,0) + i H(:,64) in one transform, stored in
//     column 0; job (warp + 8 round, grp) takes a column chosen so the two
//     groups of each half-warp hit disjoint bank halves of H;
//  4. columns 0 and 64 are split from Z, F0(k) = (Z(k) + conj Z(-k)) / 2,
//     F64(k) = (Z(k) - conj Z(-k)) / (2i); the next image's copy is started
//     and H, which has G's [128][65] layout, is copied out with 16-byte
//     stores.
// (The 512-thread form with a separate scratch and a double-buffered image,
// one CTA per SM, took 80 us at 1781 BF pixels; this one 71 us.)
constexpr int kImgPitch = 136;  // u16 per staged image row
constexpr int kScanHalf = 65;
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

template <int NT>
__device__ __forceinline__ void stage_image_async(uint16_t* img, const uint16_t* columns, int b,
                                                  int tid) {
    const uint4* src = reinterpret_cast<const uint4*>(columns + (size_t)b * 128 * 128);
    for (int i = tid; i < 128 * 128 / 8; i += NT) {
        const int row = i >> 4;
        const int col = (i & 15) * 8;
        cp_async16(img + row * kImgPitch + col, src + i);
    }
    cp_async_commit();
}

struct ScanFft128PSmem {
    static constexpr size_t t_bytes = sizeof(float2) * 32 * kG8Scratch;
    static constexpr size_t img_bytes = sizeof(uint16_t) * 128 * kImgPitch;
    static constexpr size_t u_bytes = ((t_bytes > img_bytes ? t_bytes : img_bytes) + 15) & ~(size_t)15;
    static constexpr size_t h_bytes = sizeof(float2) * 128 * kScanHalf;
    static constexpr size_t tw_bytes = sizeof(float2) * 128;
    static constexpr size_t bytes = u_bytes + h_bytes + tw_bytes;
};

// map (optional): BF pixel b's image is column map[b] of the n_cols in
// `columns` (the box columns of qssb_mean_dp_u64_box); an index outside
// [0, n_cols) is clamped (callers pass only maps whose ok flag was set).
__device__ __forceinline__ int scan_column(const int32_t* map, int b, int n_cols) {
    if (!map) return b;
    const int c = __ldg(map + b);
    return c < 0 ? 0 : (c >= n_cols ? n_cols - 1 : c);
}

__global__ void __launch_bounds__(256, 2) k_scan_fft128p(const uint16_t* __restrict__ columns,
                                                         int n_bf, float2* __restrict__ g_half,
                                                         const int32_t* __restrict__ map,
                                                         int n_cols) {
    extern __shared__ float4 smem4[];
    char* base = reinterpret_cast<char*>(smem4);
    float2* T = reinterpret_cast<float2*>(base);       // FFT scratch ...
    uint16_t* img = reinterpret_cast<uint16_t*>(base);  // ... or the staged image
    float2* H = reinterpret_cast<float2*>(base + ScanFft128PSmem::u_bytes);
    float2* tw = H + 128 * kScanHalf;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int g = tid >> 3;  // group 0..31
    const int s = tid & 7;   // sub-lane
    const int grp = lane >> 3;
    float2* Tg = T + g * kG8Scratch;
    fill_twiddles<128>(tw, tid, 256);
    if (blockIdx.x < n_bf) stage_image_async<256>(img, columns, scan_column(map, blockIdx.x, n_cols), tid);
    for (int b = blockIdx.x; b < n_bf; b += gridDim.x) {
        cp_async_wait_all();
        __syncthreads();  // the image is in; the previous copy-out of H is done
        // row pairs j = g and g + 32 into registers
        float2 v0[16], v1[16];
        {
            const uint16_t* r0 = img + (2 * g) * kImgPitch + s;
            const uint16_t* r2 = r0 + 64 * kImgPitch;
#pragma unroll
            for (int n1 = 0; n1 < 16; ++n1) {
                v0[n1] = make_float2((float)r0[8 * n1], (float)r0[kImgPitch + 8 * n1]);
                v1[n1] = make_float2((float)r2[8 * n1], (float)r2[kImgPitch + 8 * n1]);
            }
        }
        __syncthreads();  // the image region becomes T
#pragma unroll
        for (int round = 0; round < 2; ++round) {
            float2(&v)[16] = round == 0 ? v0 : v1;
            const int j = g + 32 * round;
            fft128_g8<-1>(v, Tg, s, tw);
#pragma unroll
            for (int t = 0; t < 16; ++t) Tg[fft128_g8_index(s, t)] = v[t];
            __syncwarp();
            // X_2j(c) = (Z(c) + conj Z(-c)) / 2, X_2j+1(c) = (Z(c) - conj Z(-c)) / (2i)
#pragma unroll
            for (int m = 0; m < 9; ++m) {
                const int c = s + 8 * m;
                if (c <= 64) {
                    const float2 z = Tg[c];
                    const float2 zm = Tg[(128 - c) & 127];
                    H[(2 * j) * kScanHalf + c] = make_float2(0.5f * (z.x + zm.x), 0.5f * (z.y - zm.y));
                    H[(2 * j + 1) * kScanHalf + c] = make_float2(0.5f * (z.y + zm.y), -0.5f * (z.x - zm.x));
                }
            }
            __syncwarp();  // the group's reads of Tg precede its next transform
        }
        __syncthreads();
        // columns: 64 jobs (1..63 and the packed 0 / 64 pair), two per group
#pragma unroll
        for (int round = 0; round < 2; ++round) {
            const int w = warp + 8 * round;
            const int col = 16 * (w & 3) + 8 * (grp & 1) + 2 * (w >> 2) + (grp >> 1);
            float2 v[16];
            if (col == 0) {
#pragma unroll
                for (int n1 = 0; n1 < 16; ++n1) {
                    const float2* hr = H + (s + 8 * n1) * kScanHalf;
                    v[n1] = make_float2(hr[0].x, hr[64].x);  // both columns are real
                }
            } else {
#pragma unroll
                for (int n1 = 0; n1 < 16; ++n1) v[n1] = H[(s + 8 * n1) * kScanHalf + col];
            }
            fft128_g8<-1>(v, Tg, s, tw);
#pragma unroll
            for (int t = 0; t < 16; ++t) H[fft128_g8_index(s, t) * kScanHalf + col] = v[t];
            __syncwarp();
        }
        __syncthreads();
        // split Z into columns 0 and 64: thread k <= 64 owns rows k and -k
        if (tid <= 64) {
            const int km = (128 - tid) & 127;
            const float2 a = H[tid * kScanHalf];
            const float2 m = H[km * kScanHalf];
            const float2 f0 = make_float2(0.5f * (a.x + m.x), 0.5f * (a.y - m.y));
            const float2 f64 = make_float2(0.5f * (a.y + m.y), -0.5f * (a.x - m.x));
            H[tid * kScanHalf] = f0;
            H[tid * kScanHalf + 64] = f64;
            if (km != tid) {  // F(-k) = conj F(k) for real columns (k = 0, 64: real)
                H[km * kScanHalf] = cconj(f0);
                H[km * kScanHalf + 64] = cconj(f64);
            }
        }
        __syncthreads();  // T is free: the next image comes in during the copy-out
        const int nb = b + gridDim.x;
        if (nb < n_bf) stage_image_async<256>(img, columns, scan_column(map, nb, n_cols), tid);
        const float4* h4 = reinterpret_cast<const float4*>(H);
        float4* dst = reinterpret_cast<float4*>(g_half + (size_t)b * 128 * kScanHalf);
        for (int i = tid; i < 128 * kScanHalf / 2; i += 256) dst[i] = h4[i];
    }
    cp_async_wait_all();  // nothing left in flight at exit
}

}  // namespace qssb

using namespace qssb;

extern "C" int qssb_mean_dp_u64(const uint16_t* counts, int64_t n_frames, int32_t det_pixels,
                                uint64_t* sums, float* mean_dp, void* stream) {
    if (!counts || !sums || n_frames <= 0 || det_pixels <= 0)
        return set_error(QSSB_ERR_INVALID, "qssb_mean_dp_u64: null pointer or empty shape");
    if (n_frames > (int64_t)1 << 40)
        return set_error(QSSB_ERR_INVALID, "qssb_mean_dp_u64: n_frames too large");
    cudaStream_t s = (cudaStream_t)stream;
    CUDA_TRY(cudaMemsetAsync(sums, 0, sizeof(uint64_t) * (size_t)det_pixels, s));
    const int sms = device_sm_count();
    const bool vec = (det_pixels % 8 == 0) && (((uintptr_t)counts & 15u) == 0);
    if (vec) {
        const int nvec = det_pixels / 8;
        const int gx = (nvec + kSumThreads - 1) / kSumThreads;
        // about 8 resident CTAs per SM, two waves
        long long want = (long long)sms * 16 / gx;
        if (want < 1) want = 1;
        long long chunk = (n_frames + want - 1) / want;
        if (chunk > 32768) chunk = 32768;
        if (chunk < 4) chunk = 4;
        const long long gy = (n_frames + chunk - 1) / chunk;
        if (gy > 65535) return set_error(QSSB_ERR_INVALID, "qssb_mean_dp_u64: too many frames");
        { k_sum_frames_vec8<<<dim3(gx, (unsigned)gy), kSumThreads, 0, s>>>(
            reinterpret_cast<const uint4*>(counts), n_frames, nvec, (int)chunk,
            reinterpret_cast<unsigned long long*>(sums)); note_launch(); }
    } else {
        const int gx = (det_pixels + 255) / 256;
        long long want = (long long)sms * 16 / gx;
        if (want < 1) want = 1;
        long long chunk = (n_frames + want - 1) / want;
        if (chunk > 32768) chunk = 32768;
        const long long gy = (n_frames + chunk - 1) / chunk;
        if (gy > 65535) return set_error(QSSB_ERR_INVALID, "qssb_mean_dp_u64: too many frames");
        { k_sum_frames_scalar<<<dim3(gx, (unsigned)gy), 256, 0, s>>>(
            counts, n_frames, det_pixels, (int)chunk, reinterpret_cast<unsigned long long*>(sums)); note_launch(); }
    }
    CUDA_TRY(cudaGetLastError());
    if (mean_dp) {
        { k_mean_from_sums<<<(det_pixels + 255) / 256, 256, 0, s>>>(
            reinterpret_cast<const unsigned long long*>(sums), det_pixels, (float)n_frames, mean_dp); note_launch(); }
        CUDA_TRY(cudaGetLastError());
    }
    return QSSB_OK;
}

// Bounding-box gather. The BF pixels' bounding box (rows x columns rounded
// out to 8 pixels = 16 bytes) is read per frame with coalesced 16-byte copies
// into shared memory, F frames per tile; each BF column then receives its F
// frames as F/8 consecutive 16-byte stores. Persistent CTAs (two per SM) loop
// over frame tiles with the next tile's box arriving by cp.async into a second
// buffer while the current tile is written out. (DRAM fetches whole 128-byte
// lines, so the box rows are read in full either way: ~12.5 KB per 128^2
// frame.) A box larger than the tile buffer (MAXPIX pixels per frame) is taken
// in row bands (work item = frame tile x band); with ascending BF indices (the
// selection's order) each band writes only its own contiguous BF range. Boxes
// wider than one buffer fall back to direct element loads.
// Two shapes, same 98 KB of buffers: F = 32 frames x 768 pixels for detectors
// up to 768 columns (64-byte column writes: at 128^4, 60 us against 70 us for
// 16-byte ones), F = 8 x 3072 for wider ones.
template <int F, int MAXPIX, int CTAS = 2>
struct GbShape {
    static constexpr int kF = F;
    static constexpr int kMaxPix = MAXPIX;
    static constexpr int kCtas = CTAS;  // persistent CTAs per SM
    static constexpr size_t smem = sizeof(uint16_t) * 2 * F * MAXPIX;
};
using GbNarrow = GbShape<32, 768>;
using GbWide = GbShape<8, 3072>;
constexpr int kGbThreads = 256;
constexpr int kGbNarrowCols = 768;

__device__ __forceinline__ void gb_cp_async16(void* smem_dst, const void* gmem_src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem_src) : "memory");
}

constexpr int kGbMaxBands = 64;

template <typename SHAPE>
__global__ void __launch_bounds__(kGbThreads) k_gather_bbox(
    const uint16_t* __restrict__ counts, long long n_frames, int det_rows, int det_cols,
    const int32_t* __restrict__ bf_linear, int n_bf, uint16_t* __restrict__ columns) {
    constexpr int kGbF = SHAPE::kF;
    constexpr int kGbMaxPix = SHAPE::kMaxPix;
    extern __shared__ uint4 smem_u4[];
    uint16_t* tiles = reinterpret_cast<uint16_t*>(smem_u4);  // [2][kGbF][band area]
    __shared__ int s_box[4][kGbThreads / 32];
    __shared__ int s_band_lo[kGbMaxBands + 1];
    __shared__ int s_unsorted;
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int npix = det_rows * det_cols;
    int rmin = det_rows, rmax = -1, cmin = det_cols, cmax = -1;
    if (tid == 0) s_unsorted = 0;
    __syncthreads();
    for (int b = tid; b < n_bf; b += kGbThreads) {
        const int lin = __ldg(bf_linear + b);
        if (b + 1 < n_bf && __ldg(bf_linear + b + 1) <= lin) s_unsorted = 1;
        if (lin < 0 || lin >= npix) continue;
        const int r = lin / det_cols, c = lin - (lin / det_cols) * det_cols;
        rmin = min(rmin, r); rmax = max(rmax, r); cmin = min(cmin, c); cmax = max(cmax, c);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        rmin = min(rmin, __shfl_xor_sync(0xffffffffu, rmin, o));
        rmax = max(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
        cmin = min(cmin, __shfl_xor_sync(0xffffffffu, cmin, o));
        cmax = max(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
    }
    if (lane == 0) {
        s_box[0][warp] = rmin; s_box[1][warp] = rmax; s_box[2][warp] = cmin; s_box[3][warp] = cmax;
    }
    __syncthreads();
    rmin = det_rows; rmax = -1; cmin = det_cols; cmax = -1;
#pragma unroll
    for (int w = 0; w < kGbThreads / 32; ++w) {
        rmin = min(rmin, s_box[0][w]); rmax = max(rmax, s_box[1][w]);
        cmin = min(cmin, s_box[2][w]); cmax = max(cmax, s_box[3][w]);
    }
    const long long n_tiles = (n_frames + kGbF - 1) / kGbF;
    const int c0 = cmin & ~7;
    const int width = rmax >= 0 ? ((cmax + 8) & ~7) - c0 : 0;   // multiple of 8 pixels
    const int nr = rmax >= 0 ? rmax - rmin + 1 : 0;
    // row bands of at most kGbMaxPix box pixels
    const int band_rows = width > 0 ? min(nr, kGbMaxPix / width) : 0;
    const int n_bands = band_rows > 0 ? (nr + band_rows - 1) / band_rows : 0;
    if (width == 0 || band_rows == 0 || n_bands > kGbMaxBands) {
        // direct path: one element per (frame, BF pixel)
        for (long long t = blockIdx.x; t < n_tiles; t += gridDim.x) {
            const long long f0 = t * kGbF;
            const int nf = (int)min((long long)kGbF, n_frames - f0);
            for (int e = tid; e < nf * n_bf; e += kGbThreads) {
                const int f = e / n_bf, b = e - (e / n_bf) * n_bf;
                const int lin = __ldg(bf_linear + b);
                const bool ok = lin >= 0 && lin < npix;
                columns[(size_t)b * n_frames + f0 + f] =
                    ok ? __ldcs(counts + (size_t)(f0 + f) * npix + lin) : (uint16_t)0;
            }
        }
        return;
    }
    // BF range of each band when bf_linear is ascending (the selection's
    // row-major order): s_band_lo[k] = #{b : lin(b) < first pixel of band k}
    const bool sorted = s_unsorted == 0;
    if (sorted) {
        for (int k = tid; k <= n_bands; k += kGbThreads) {
            const int row = rmin + k * band_rows;
            const int key = row > rmax ? 0x7fffffff : row * det_cols;
            int lo = 0, hi = n_bf;  // first b with lin(b) >= key
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (__ldg(bf_linear + mid) < key) lo = mid + 1; else hi = mid;
            }
            s_band_lo[k] = lo;
        }
    }
    __syncthreads();
    const int vpr = width / 8;
    const long long n_items = n_tiles * n_bands;
    auto stage = [&](long long item, uint16_t* dst) {
        const long long t = item / n_bands;
        const int k = (int)(item - t * n_bands);
        const int r0 = rmin + k * band_rows;
        const int rows = min(band_rows, rmax + 1 - r0);
        const int per_frame = rows * vpr;
        const int area = rows * width;
        const long long f0 = t * kGbF;
        const int nf = (int)min((long long)kGbF, n_frames - f0);
        for (int e = tid; e < nf * per_frame; e += kGbThreads) {
            const int f = e / per_frame;
            const int rem = e - f * per_frame;
            const int i = rem / vpr;
            const int v = rem - i * vpr;
            const uint4* src = reinterpret_cast<const uint4*>(
                counts + (size_t)(f0 + f) * npix + (size_t)(r0 + i) * det_cols + c0) + v;
            gb_cp_async16(reinterpret_cast<uint4*>(dst + (size_t)f * area + i * width) + v, src);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
    const bool vec_out = (n_frames & 7) == 0;
    int buf = 0;
    if (blockIdx.x < n_items) stage(blockIdx.x, tiles);
    for (long long item = blockIdx.x; item < n_items; item += gridDim.x) {
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        __syncthreads();  // this item is in; everyone is done with the other buffer
        const long long nxt = item + gridDim.x;
        if (nxt < n_items) stage(nxt, tiles + (size_t)(buf ^ 1) * kGbF * kGbMaxPix);
        const uint16_t* tile = tiles + (size_t)buf * kGbF * kGbMaxPix;
        const long long t = item / n_bands;
        const int k = (int)(item - t * n_bands);
        const int r0 = rmin + k * band_rows;
        const int rows = min(band_rows, rmax + 1 - r0);
        const int area = rows * width;
        const long long f0 = t * kGbF;
        const int nf = (int)min((long long)kGbF, n_frames - f0);
        // sorted: the bands' BF ranges partition [0, n_bf) (out-of-detector
        // entries sit at the ends and go to the first / last band); unsorted:
        // every band scans all pixels and band 0 zero-fills invalid ones
        const int b_lo = sorted && k > 0 ? s_band_lo[k] : 0;
        const int b_hi = sorted && k + 1 < n_bands ? s_band_lo[k + 1] : n_bf;
        const bool owns_invalid = sorted || k == 0;
        for (int b = b_lo + tid; b < b_hi; b += kGbThreads) {
            const int lin = __ldg(bf_linear + b);
            const bool valid = lin >= 0 && lin < npix;
            const int r = valid ? lin / det_cols : -1;
            if (valid ? (r < r0 || r >= r0 + rows) : !owns_invalid) continue;
            const bool ok = valid;
            const int c = ok ? lin - r * det_cols : c0;
            const int pos = ok ? (r - r0) * width + (c - c0) : 0;
            uint16_t* dst = columns + (size_t)b * n_frames + f0;
            if (vec_out && nf == kGbF) {
#pragma unroll
                for (int h = 0; h < kGbF / 8; ++h) {  // 8 frames per 16-byte store
                    uint32_t w[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        w[q] = ok ? ((uint32_t)tile[(8 * h + 2 * q) * area + pos] |
                                     ((uint32_t)tile[(8 * h + 2 * q + 1) * area + pos] << 16)) : 0u;
                    reinterpret_cast<uint4*>(dst)[h] = make_uint4(w[0], w[1], w[2], w[3]);
                }
            } else {
                for (int f = 0; f < nf; ++f) dst[f] = ok ? tile[f * area + pos] : (uint16_t)0;
            }
        }
        buf ^= 1;
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// 64-frame tiles for outputs that do not stay in L2 (512^2 scans and up): a
// work item is (64 frames, a row band of the bounding box). Lane pairs read a
// 32-byte box segment of one frame (16 frames per warp load) and scatter the
// pixels into a pixel-major shared tile (pitch 72 frames = 144 bytes, 16-byte
// aligned rows); each BF column then receives its 64 frames as one 128-byte
// line written by 8 lanes. Needs n_frames % 8 == 0 and 16-byte aligned rows.
// Two tile sizes: 320 band pixels per item (45 KB, four CTAs per SM) for
// detectors up to 320 columns - 0.90 ms against 1.22 ms for the 704-pixel
// form on a 256^2 x 192^2 scan with 8921 BF pixels - and 704 (99 KB, two
// per SM) beyond.
constexpr int kT64F = 64;
constexpr int kT64P = 72;  // frames per smem pixel row (64 + 8)
constexpr int kT64SmallCols = 320;

template <int MAXPIX>
__global__ void __launch_bounds__(kGbThreads) k_gather_t64(
    const uint16_t* __restrict__ counts, long long n_frames, int det_rows, int det_cols,
    const int32_t* __restrict__ bf_linear, int n_bf, uint16_t* __restrict__ columns) {
    constexpr int kT64MaxPix = MAXPIX;  // band pixels per item (x 144 B of shared memory)
    extern __shared__ uint4 smem_u4[];
    uint16_t* tile = reinterpret_cast<uint16_t*>(smem_u4);  // [band pixel][kT64P]
    __shared__ int s_box[4][kGbThreads / 32];
    __shared__ int s_band_lo[kGbMaxBands + 1];
    __shared__ int s_unsorted;
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int npix = det_rows * det_cols;
    if (tid == 0) s_unsorted = 0;
    __syncthreads();
    int rmin = det_rows, rmax = -1, cmin = det_cols, cmax = -1;
    for (int b = tid; b < n_bf; b += kGbThreads) {
        const int lin = __ldg(bf_linear + b);
        if (b + 1 < n_bf && __ldg(bf_linear + b + 1) <= lin) s_unsorted = 1;
        if (lin < 0 || lin >= npix) continue;
        const int r = lin / det_cols, c = lin - (lin / det_cols) * det_cols;
        rmin = min(rmin, r); rmax = max(rmax, r); cmin = min(cmin, c); cmax = max(cmax, c);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        rmin = min(rmin, __shfl_xor_sync(0xffffffffu, rmin, o));
        rmax = max(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
        cmin = min(cmin, __shfl_xor_sync(0xffffffffu, cmin, o));
        cmax = max(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
    }
    if (lane == 0) {
        s_box[0][warp] = rmin; s_box[1][warp] = rmax; s_box[2][warp] = cmin; s_box[3][warp] = cmax;
    }
    __syncthreads();
    rmin = det_rows; rmax = -1; cmin = det_cols; cmax = -1;
#pragma unroll
    for (int w = 0; w < kGbThreads / 32; ++w) {
        rmin = min(rmin, s_box[0][w]); rmax = max(rmax, s_box[1][w]);
        cmin = min(cmin, s_box[2][w]); cmax = max(cmax, s_box[3][w]);
    }
    const int c0 = cmin & ~15;
    // multiple of 16 pixels (32-byte segments), inside the detector row
    const int width = rmax >= 0 ? min(((cmax + 16) & ~15), det_cols) - c0 : 0;
    const int nr = rmax >= 0 ? rmax - rmin + 1 : 0;
    const int band_rows = width > 0 ? min(nr, kT64MaxPix / width) : 0;
    const int n_bands = band_rows > 0 ? (nr + band_rows - 1) / band_rows : 0;
    const long long n_tiles = (n_frames + kT64F - 1) / kT64F;
    if (width == 0 || (width & 15) || band_rows == 0 || n_bands > kGbMaxBands) {
        for (long long t = blockIdx.x; t < n_tiles; t += gridDim.x) {  // direct path
            const long long f0 = t * kT64F;
            const int nf = (int)min((long long)kT64F, n_frames - f0);
            for (int e = tid; e < nf * n_bf; e += kGbThreads) {
                const int f = e / n_bf, b = e - (e / n_bf) * n_bf;
                const int lin = __ldg(bf_linear + b);
                const bool ok = lin >= 0 && lin < npix;
                columns[(size_t)b * n_frames + f0 + f] =
                    ok ? __ldcs(counts + (size_t)(f0 + f) * npix + lin) : (uint16_t)0;
            }
        }
        return;
    }
    const bool sorted = s_unsorted == 0;
    if (sorted) {
        for (int k = tid; k <= n_bands; k += kGbThreads) {
            const int row = rmin + k * band_rows;
            const int key = row > rmax ? 0x7fffffff : row * det_cols;
            int lo = 0, hi = n_bf;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (__ldg(bf_linear + mid) < key) lo = mid + 1; else hi = mid;
            }
            s_band_lo[k] = lo;
        }
    }
    __syncthreads();
    const int segs_per_row = width / 16;
    const long long n_items = n_tiles * n_bands;
    const int grp = tid >> 3;  // write phase: 32 groups of 8 lanes, one BF column each
    const int sub = tid & 7;
    for (long long item = blockIdx.x; item < n_items; item += gridDim.x) {
        const long long t = item / n_bands;
        const int k = (int)(item - t * n_bands);
        const int r0 = rmin + k * band_rows;
        const int rows = min(band_rows, rmax + 1 - r0);
        const long long f0 = t * kT64F;
        const int nf = (int)min((long long)kT64F, n_frames - f0);
        // load: e -> lane pair q = e / 2 (one 32-byte segment), half h
        const int n_e = 2 * kT64F * rows * segs_per_row;
#pragma unroll 4
        for (int e = tid; e < n_e; e += kGbThreads) {
            const int h = e & 1;
            const int q = e >> 1;
            const int f = q & (kT64F - 1);
            const int seg = q >> 6;
            const int i = seg / segs_per_row;
            const int sg = seg - i * segs_per_row;
            const int px = i * width + 16 * sg + 8 * h;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (f < nf)
                v = __ldcs(reinterpret_cast<const uint4*>(
                    counts + (size_t)(f0 + f) * npix + (size_t)(r0 + i) * det_cols + c0 + 16 * sg + 8 * h));
            uint16_t* d = tile + (size_t)px * kT64P + f;
            d[0 * kT64P] = (uint16_t)(v.x & 0xffffu); d[1 * kT64P] = (uint16_t)(v.x >> 16);
            d[2 * kT64P] = (uint16_t)(v.y & 0xffffu); d[3 * kT64P] = (uint16_t)(v.y >> 16);
            d[4 * kT64P] = (uint16_t)(v.z & 0xffffu); d[5 * kT64P] = (uint16_t)(v.z >> 16);
            d[6 * kT64P] = (uint16_t)(v.w & 0xffffu); d[7 * kT64P] = (uint16_t)(v.w >> 16);
        }
        __syncthreads();
        const int b_lo = sorted && k > 0 ? s_band_lo[k] : 0;
        const int b_hi = sorted && k + 1 < n_bands ? s_band_lo[k + 1] : n_bf;
        const bool owns_invalid = sorted || k == 0;
        for (int b = b_lo + grp; b < b_hi; b += kGbThreads / 8) {
            const int lin = __ldg(bf_linear + b);
            const bool valid = lin >= 0 && lin < npix;
            const int r = valid ? lin / det_cols : -1;
            if (valid ? (r < r0 || r >= r0 + rows) : !owns_invalid) continue;
            if (8 * sub >= nf) continue;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (valid) {
                const int pos = (r - r0) * width + (lin - r * det_cols - c0);
                v = *reinterpret_cast<const uint4*>(tile + (size_t)pos * kT64P + 8 * sub);
            }
            *reinterpret_cast<uint4*>(columns + (size_t)b * n_frames + f0 + 8 * sub) = v;
        }
        __syncthreads();  // the tile is rewritten by the next item
    }
}

extern "C" int qssb_gather_bf_columns(const uint16_t* counts, int64_t n_frames, int32_t det_pixels,
                                      const int32_t* bf_linear, int32_t n_bf, uint16_t* columns,
                                      void* stream) {
    if (!counts || !bf_linear || !columns || n_frames <= 0 || det_pixels <= 0 || n_bf <= 0)
        return set_error(QSSB_ERR_INVALID, "qssb_gather_bf_columns: null pointer or empty shape");
    if (((uintptr_t)columns & 3u) != 0)
        return set_error(QSSB_ERR_INVALID, "qssb_gather_bf_columns: columns must be 4-byte aligned");
    const long long gx = (n_frames + kGatherF - 1) / kGatherF;
    const int gy = (n_bf + kGatherB - 1) / kGatherB;
    if (gx > 0x7fffffffLL || gy > 65535)
        return set_error(QSSB_ERR_INVALID, "qssb_gather_bf_columns: grid too large");
    { k_gather_columns<<<dim3((unsigned)gx, gy), 256, 0, (cudaStream_t)stream>>>(
        counts, n_frames, det_pixels, bf_linear, n_bf, columns); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}

template <int MAXPIX, int CTAS>
static int launch_gather_t64(const uint16_t* counts, int64_t n_frames, int det_rows, int det_cols,
                             const int32_t* bf_linear, int n_bf, uint16_t* columns,
                             cudaStream_t stream) {
    const long long n_tiles64 = (n_frames + kT64F - 1) / kT64F;
    long long gx = (long long)CTAS * device_sm_count();
    if (gx > n_tiles64) gx = n_tiles64;
    const int smem = (int)(sizeof(uint16_t) * kT64P * MAXPIX);
    CUDA_TRY(cudaFuncSetAttribute(k_gather_t64<MAXPIX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  smem));
    { k_gather_t64<MAXPIX><<<(unsigned)gx, kGbThreads, smem, stream>>>(
        counts, n_frames, det_rows, det_cols, bf_linear, n_bf, columns); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}

template <typename SHAPE>
static int launch_gather_bbox(const uint16_t* counts, int64_t n_frames, int det_rows, int det_cols,
                              const int32_t* bf_linear, int n_bf, uint16_t* columns,
                              cudaStream_t stream) {
    const long long n_tiles = (n_frames + SHAPE::kF - 1) / SHAPE::kF;
    long long gx = (long long)SHAPE::kCtas * device_sm_count();
    if (gx > n_tiles) gx = n_tiles;
    const int smem = (int)SHAPE::smem;
    CUDA_TRY(cudaFuncSetAttribute(k_gather_bbox<SHAPE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  smem));
    { k_gather_bbox<SHAPE><<<(unsigned)gx, kGbThreads, smem, stream>>>(
        counts, n_frames, det_rows, det_cols, bf_linear, n_bf, columns); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}

// Tile shapes the autotuner may pick (qssb_gather_bf_columns_2d_ex); all
// copy the same bits.
using GbF16 = GbShape<16, 1536>;
using GbF64 = GbShape<64, 384>;
constexpr int kGatherVariants = 7;

extern "C" int qssb_gather_bf_columns_2d_ex(const uint16_t* counts, int64_t n_frames,
                                            int32_t det_rows, int32_t det_cols,
                                            const int32_t* bf_linear, int32_t n_bf,
                                            uint16_t* columns, int32_t variant, void* stream) {
    if (!counts || !bf_linear || !columns || n_frames <= 0 || det_rows <= 0 || det_cols <= 0 ||
        n_bf <= 0)
        return set_error(QSSB_ERR_INVALID, "qssb_gather_bf_columns_2d: null pointer or empty shape");
    if ((int64_t)det_rows * det_cols > 0x7fffffff)
        return set_error(QSSB_ERR_INVALID, "qssb_gather_bf_columns_2d: detector too large");
    if (variant < 0 || variant >= kGatherVariants)
        return set_error(QSSB_ERR_INVALID, "qssb_gather_bf_columns_2d_ex: unknown variant");
    const bool vec_ok = (det_cols % 8) == 0 && ((uintptr_t)counts & 15u) == 0 &&
                        ((uintptr_t)columns & 15u) == 0;
    if (!vec_ok)  // rows not 16-byte aligned: the tile gather
        return qssb_gather_bf_columns(counts, n_frames, det_rows * det_cols, bf_linear, n_bf,
                                      columns, stream);
    cudaStream_t st = (cudaStream_t)stream;
    const bool t64_ok = (n_frames & 7) == 0;
    switch (variant) {
        case 1: return launch_gather_bbox<GbNarrow>(counts, n_frames, det_rows, det_cols, bf_linear, n_bf, columns, st);
        case 2: return launch_gather_bbox<GbF16>(counts, n_frames, det_rows, det_cols, bf_linear, n_bf, columns, st);
        case 3: return launch_gather_bbox<GbF64>(counts, n_frames, det_rows, det_cols, bf_linear, n_bf, columns, st);
        case 4: return launch_gather_bbox<GbWide>(counts, n_frames, det_rows, det_cols, bf_linear, n_bf, columns, st);
        case 5:
            if (t64_ok) return launch_gather_t64<320, 4>(counts, n_frames, det_rows, det_cols, bf_linear, n_bf, columns, st);
            break;
        case 6:
            if (t64_ok) return launch_gather_t64<704, 2>(counts, n_frames, det_rows, det_cols, bf_linear, n_bf, columns, st);
            break;
        default:
            break;
    }
    if (t64_ok && (int64_t)n_frames * n_bf * 2 > ((int64_t)64 << 20)) {
        // output larger than L2 can merge: full 128-byte column lines
        if (det_cols <= kT64SmallCols)
            return launch_gather_t64<320, 4>(counts, n_frames, det_rows, det_cols, bf_linear, n_bf,
                                             columns, (cudaStream_t)stream);
        return launch_gather_t64<704, 2>(counts, n_frames, det_rows, det_cols, bf_linear, n_bf,
                                         columns, (cudaStream_t)stream);
    }
    if (det_cols <= kGbNarrowCols)
        return launch_gather_bbox<GbNarrow>(counts, n_frames, det_rows, det_cols, bf_linear, n_bf,
                                            columns, (cudaStream_t)stream);
    return launch_gather_bbox<GbWide>(counts, n_frames, det_rows, det_cols, bf_linear, n_bf,
                                      columns, (cudaStream_t)stream);
}

extern "C" int qssb_gather_bf_columns_2d(const uint16_t* counts, int64_t n_frames,
                                         int32_t det_rows, int32_t det_cols,
                                         const int32_t* bf_linear, int32_t n_bf,
                                         uint16_t* columns, void* stream) {
    return qssb_gather_bf_columns_2d_ex(counts, n_frames, det_rows, det_cols, bf_linear, n_bf,
                                        columns, 0, stream);
}

// ------------------------------------------ 256^2 .. 1024^2 scan FFT
// The half plane (264 KB per BF image at 256^2) does not fit one CTA's
// shared memory, so the transform is two passes through G itself:
//   k_scan_rows<N>: rows 2j, 2j+1 of a BF image as one complex line (one warp
//     per pair), forward warp FFT, split into the two real rows' spectra
//     X_2j(c) = (Z(c) + conj Z(-c)) / 2, X_2j+1(c) = (Z(c) - conj Z(-c)) / 2i,
//     c = 0..N/2, written to G[b][row][c];
//   k_scan_cols<N>: T columns of G[b] staged in shared memory (odd pitch:
//     the T columns of one row land on distinct banks), forward warp FFT of
//     each column along the rows, written back in place.
template <int N>
struct ScanLines {
    static constexpr int H = N / 2 + 1;
    static constexpr int kWarps = N >= 1024 ? 4 : 8;       // row pairs per block
    static constexpr int kTile = N >= 1024 ? 8 : 16;       // columns per block
    // persistent column pass: columns per strip (one warp each) and CTAs per
    // SM. At 256 three 8-warp CTAs per SM (0.63 ms for the two scan passes of
    // 1783 BF pixels against 0.71 with one 16-warp CTA); at 512 and 1024 the
    // 16/8-warp single CTA (8-warp pairs were within 1% at 512)
    static constexpr int kTileP = N >= 1024 ? 8 : (N == 256 ? 8 : 16);
    static constexpr int kCtasP = N == 256 ? 3 : 1;
    static constexpr int kScratch = warp_fft_scratch<N>();  // >= N: also holds a line
    static constexpr int P = kScratch | 1;                  // column pitch, odd mod 16
    static constexpr size_t rows_smem = sizeof(float2) * ((size_t)kWarps * kScratch + N);
    static constexpr size_t cols_smem = sizeof(float2) * ((size_t)kTile * P + N);
};

// Rows: one warp per row pair, the line straight into registers
// (v[t] = x[32 t + lane]), warp FFT, spectrum back to the warp's shared line
// in natural order for the real-pair split.
template <int N>
__global__ void __launch_bounds__(32 * ScanLines<N>::kWarps) k_scan_rows(
    const uint16_t* __restrict__ columns, int n_bf, float2* __restrict__ g_half) {
    using L = ScanLines<N>;
    constexpr int W = L::kWarps;
    constexpr int H = L::H;
    constexpr int RPL = N / 32;
    extern __shared__ float4 scan_rows_smem[];
    float2* scr = reinterpret_cast<float2*>(scan_rows_smem);
    float2* tw = scr + W * L::kScratch;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    fill_twiddles<N>(tw, tid, 32 * W);
    __syncthreads();
    const int b = blockIdx.x;
    const int pair = blockIdx.y * W + warp;  // 0 .. N/2 - 1
    if (b >= n_bf || pair >= N / 2) return;
    const uint16_t* img = columns + (size_t)b * N * N;
    const uint16_t* r0 = img + (size_t)(2 * pair) * N;
    const uint16_t* r1 = r0 + N;
    float2 v[RPL];
#pragma unroll
    for (int t = 0; t < RPL; ++t)
        v[t] = make_float2((float)__ldcs(r0 + 32 * t + lane), (float)__ldcs(r1 + 32 * t + lane));
    float2* x = scr + warp * L::kScratch;
    warp_fft<N, -1>(v, x, tw, lane);
#pragma unroll
    for (int j = 0; j < RPL; ++j) x[warp_fft_index<N>(lane, j)] = v[j];
    __syncwarp();
    float2* g0 = g_half + ((size_t)b * N + 2 * pair) * H;
    float2* g1 = g0 + H;
    for (int c = lane; c < H; c += 32) {
        const float2 z = x[c];
        const float2 m = x[(N - c) & (N - 1)];
        g0[c] = make_float2(0.5f * (z.x + m.x), 0.5f * (z.y - m.y));
        g1[c] = make_float2(0.5f * (z.y + m.y), -0.5f * (z.x - m.x));
    }
}

// Columns: T columns of G[b] staged in shared memory, one warp FFT per
// column (the column's own line is the transpose scratch), written back.
template <int N>
__global__ void __launch_bounds__(256) k_scan_cols(int n_bf, float2* __restrict__ g_half) {
    using L = ScanLines<N>;
    constexpr int P = L::P;
    constexpr int T = L::kTile;
    constexpr int H = L::H;
    constexpr int RPL = N / 32;
    extern __shared__ float2 scan_cols_smem[];
    float2* tile = scan_cols_smem;
    float2* tw = tile + T * P;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    fill_twiddles<N>(tw, tid, 256);
    const int b = blockIdx.x;
    const int c0 = blockIdx.y * T;
    const int nc = min(T, H - c0);
    if (b >= n_bf) return;  // uniform per block: before any barrier
    float2* g = g_half + (size_t)b * N * H;
    for (int e = tid; e < N * T; e += 256) {
        const int r = e / T;
        const int c = e - r * T;
        if (c < nc) tile[c * P + r] = g[(size_t)r * H + c0 + c];
    }
    __syncthreads();
    for (int c = warp; c < nc; c += 8) {
        float2* line = tile + c * P;
        float2 v[RPL];
#pragma unroll
        for (int t = 0; t < RPL; ++t) v[t] = line[lane + 32 * t];
        __syncwarp();
        warp_fft<N, -1>(v, line, tw, lane);
#pragma unroll
        for (int j = 0; j < RPL; ++j) line[warp_fft_index<N>(lane, j)] = v[j];
        __syncwarp();
    }
    __syncthreads();
    for (int e = tid; e < N * T; e += 256) {
        const int r = e / T;
        const int c = e - r * T;
        if (c < nc) g[(size_t)r * H + c0 + c] = tile[c * P + r];
    }
}

// Persistent column pass (N >= 256): kCtasP CTAs per SM (a warp per column
// of the strip) loop over (BF pixel, column strip) items; the next strip
// arrives by cp.async into the second buffer while the current one is
// transformed (one warp per column) and stored.
__device__ __forceinline__ void scan_cp_async8(void* smem_dst, const void* gmem_src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(gmem_src) : "memory");
}

template <int N, int T = ScanLines<N>::kTileP, int CTAS = ScanLines<N>::kCtasP>
__global__ void __launch_bounds__(32 * T, CTAS) k_scan_cols_p(int n_bf, float2* __restrict__ g_half) {
    using L = ScanLines<N>;
    constexpr int P = L::P;  // T: columns per strip, one warp each; CTAS: CTAs per SM
    constexpr int NT = 32 * T;
    constexpr int H = L::H;
    constexpr int RPL = N / 32;
    constexpr int NS = (H + T - 1) / T;  // strips per BF image
    extern __shared__ float2 scan_colsp_smem[];
    float2* tiles = scan_colsp_smem;     // [2][T][P]
    float2* tw = tiles + 2 * T * P;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    fill_twiddles<N>(tw, tid, NT);
    const long long n_items = (long long)n_bf * NS;
    auto issue = [&](long long item, float2* dst) {
        const int b = (int)(item / NS);
        const int c0 = (int)(item - (long long)b * NS) * T;
        const int nc = min(T, H - c0);
        const float2* g = g_half + (size_t)b * N * H + c0;
        for (int e = tid; e < N * T; e += NT) {
            const int r = e / T;
            const int c = e - r * T;
            if (c < nc) scan_cp_async8(dst + c * P + r, g + (size_t)r * H + c);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
    int buf = 0;
    if (blockIdx.x < n_items) issue(blockIdx.x, tiles);
    for (long long item = blockIdx.x; item < n_items; item += gridDim.x) {
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        __syncthreads();  // this strip is in; the other buffer's stores are done
        if (item + gridDim.x < n_items) issue(item + gridDim.x, tiles + (buf ^ 1) * T * P);
        float2* tile = tiles + buf * T * P;
        const int b = (int)(item / NS);
        const int c0 = (int)(item - (long long)b * NS) * T;
        const int nc = min(T, H - c0);
        if (warp < nc) {
            float2* line = tile + warp * P;
            float2 v[RPL];
#pragma unroll
            for (int t = 0; t < RPL; ++t) v[t] = line[lane + 32 * t];
            __syncwarp();
            warp_fft<N, -1>(v, line, tw, lane);
#pragma unroll
            for (int j = 0; j < RPL; ++j) line[warp_fft_index<N>(lane, j)] = v[j];
        }
        __syncthreads();
        float2* g = g_half + (size_t)b * N * H + c0;
        for (int e = tid; e < N * T; e += NT) {
            const int r = e / T;
            const int c = e - r * T;
            if (c < nc) g[(size_t)r * H + c] = tile[c * P + r];
        }
        buf ^= 1;
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

template <int N, int T, int CTAS>
static int launch_scan_cols_p(int n_bf, float2* g, cudaStream_t s) {
    using L = ScanLines<N>;
    const size_t smem = sizeof(float2) * ((size_t)2 * T * L::P + N);
    CUDA_TRY(cudaFuncSetAttribute(k_scan_cols_p<N, T, CTAS>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const long long items = (long long)n_bf * ((L::H + T - 1) / T);
    const long long slots = (long long)CTAS * device_sm_count();
    const int grid = (int)(items < slots ? items : slots);
    { k_scan_cols_p<N, T, CTAS><<<grid, 32 * T, smem, s>>>(n_bf, g); note_launch(); }
    return QSSB_OK;
}

// Column-pass shapes (columns per strip = warps per CTA, CTAs per SM) the
// autotuner may pick through qssb_scan_fft_half_ex: variant 1 is the
// built-in choice, 2.. the alternatives; all give the same bits.
template <int N>
static int launch_scan_lines(const uint16_t* columns, int n_bf, float* g_half, int variant,
                             cudaStream_t s) {
    using L = ScanLines<N>;
    auto* g = reinterpret_cast<float2*>(g_half);
    CUDA_TRY(cudaFuncSetAttribute(k_scan_rows<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)L::rows_smem));
    { k_scan_rows<N><<<dim3(n_bf, (N / 2 + L::kWarps - 1) / L::kWarps), 32 * L::kWarps,
                     L::rows_smem, s>>>(columns, n_bf, g); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaFuncSetAttribute(k_scan_cols<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)L::cols_smem));
    int rc = QSSB_OK;
    if constexpr (N == 256) {
        switch (variant) {
            case 2: rc = launch_scan_cols_p<N, 16, 1>(n_bf, g, s); break;
            case 3: rc = launch_scan_cols_p<N, 8, 2>(n_bf, g, s); break;
            case 4: rc = launch_scan_cols_p<N, 16, 2>(n_bf, g, s); break;
            default: rc = launch_scan_cols_p<N, L::kTileP, L::kCtasP>(n_bf, g, s); break;
        }
    } else if constexpr (N == 512) {
        switch (variant) {
            case 2: rc = launch_scan_cols_p<N, 8, 1>(n_bf, g, s); break;
            case 3: rc = launch_scan_cols_p<N, 8, 2>(n_bf, g, s); break;
            default: rc = launch_scan_cols_p<N, L::kTileP, L::kCtasP>(n_bf, g, s); break;
        }
    } else if constexpr (N >= 1024) {
        switch (variant) {
            case 2: rc = launch_scan_cols_p<N, 4, 2>(n_bf, g, s); break;
            default: rc = launch_scan_cols_p<N, L::kTileP, L::kCtasP>(n_bf, g, s); break;
        }
    } else {
        { k_scan_cols<N><<<dim3(n_bf, (L::H + L::kTile - 1) / L::kTile), 256, L::cols_smem, s>>>(n_bf, g); note_launch(); }
    }
    if (rc) return rc;
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}

template <int N>
static int launch_scan_fft(const uint16_t* columns, int n_bf, float* g_half, cudaStream_t s) {
    const size_t smem = ScanFftSmem<N>::bytes;
    CUDA_TRY(cudaFuncSetAttribute(k_scan_fft_half<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem));
    { k_scan_fft_half<N><<<n_bf, 512, smem, s>>>(columns, n_bf, reinterpret_cast<float2*>(g_half)); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}

extern "C" int qssb_scan_fft_variants(int32_t scan_rows, int32_t* count) {
    if (!count) return set_error(QSSB_ERR_INVALID, "qssb_scan_fft_variants: null output");
    switch (scan_rows) {
        case 64: *count = 1; return QSSB_OK;
        case 128: *count = 2; return QSSB_OK;
        case 256: *count = 4; return QSSB_OK;
        case 512: *count = 3; return QSSB_OK;
        case 1024: *count = 2; return QSSB_OK;
        default:
            return set_error(QSSB_ERR_UNSUPPORTED,
                             "qssb_scan_fft_variants: scan size must be 64, 128, 256, 512 or 1024");
    }
}

extern "C" int qssb_scan_fft_half_ex(const uint16_t* columns, int32_t n_bf, int32_t scan_rows,
                                     int32_t scan_cols, float* g_half, int32_t variant,
                                     void* stream) {
    if (!columns || !g_half || n_bf <= 0)
        return set_error(QSSB_ERR_INVALID, "qssb_scan_fft_half: null pointer or empty shape");
    int32_t n_var = 0;
    if (scan_rows == scan_cols && qssb_scan_fft_variants(scan_rows, &n_var) == QSSB_OK &&
        (variant < 0 || variant > n_var))
        return set_error(QSSB_ERR_INVALID, "qssb_scan_fft_half_ex: unknown variant");
    if (scan_rows != scan_cols)
        return set_error(QSSB_ERR_UNSUPPORTED, "qssb_scan_fft_half: square scans only");
    if (((uintptr_t)columns & 15u) != 0)
        return set_error(QSSB_ERR_INVALID, "qssb_scan_fft_half: columns must be 16-byte aligned");
    if (n_bf > 0x7fffffff)
        return set_error(QSSB_ERR_INVALID, "qssb_scan_fft_half: too many BF pixels");
    cudaStream_t s = (cudaStream_t)stream;
    switch (scan_rows) {
        case 64: return launch_scan_fft<64>(columns, n_bf, g_half, s);
        case 128: {
            // persistent CTAs: two per SM (variant 1, the default), or one (variant 2)
            const size_t smem = ScanFft128PSmem::bytes;
            CUDA_TRY(cudaFuncSetAttribute(k_scan_fft128p, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
            const int slots = (variant == 2 ? 1 : 2) * device_sm_count();
            const int grid = n_bf < slots ? n_bf : slots;
            { k_scan_fft128p<<<grid, 256, smem, s>>>(columns, n_bf, reinterpret_cast<float2*>(g_half),
                                                   nullptr, n_bf); note_launch(); }
            CUDA_TRY(cudaGetLastError());
            return QSSB_OK;
        }
        case 256: return launch_scan_lines<256>(columns, n_bf, g_half, variant, s);
        case 512: return launch_scan_lines<512>(columns, n_bf, g_half, variant, s);
        case 1024: return launch_scan_lines<1024>(columns, n_bf, g_half, variant, s);
        default:
            return set_error(QSSB_ERR_UNSUPPORTED,
                             "qssb_scan_fft_half: scan size must be 64, 128, 256, 512 or 1024");
    }
}

extern "C" int qssb_scan_fft_half(const uint16_t* columns, int32_t n_bf, int32_t scan_rows,
                                  int32_t scan_cols, float* g_half, void* stream) {
    return qssb_scan_fft_half_ex(columns, n_bf, scan_rows, scan_cols, g_half, 0, stream);
}

extern "C" int qssb_scan_fft_half_mapped(const uint16_t* columns, int64_t n_cols,
                                         const int32_t* map, int32_t n_bf, int32_t scan_rows,
                                         int32_t scan_cols, float* g_half, void* stream) {
    if (!columns || !map || !g_half || n_bf <= 0 || n_cols <= 0)
        return set_error(QSSB_ERR_INVALID, "qssb_scan_fft_half_mapped: null pointer or empty shape");
    if (scan_rows != 128 || scan_cols != 128)
        return set_error(QSSB_ERR_UNSUPPORTED, "qssb_scan_fft_half_mapped: 128x128 scans only");
    if (((uintptr_t)columns & 15u) != 0)
        return set_error(QSSB_ERR_INVALID, "qssb_scan_fft_half_mapped: columns must be 16-byte aligned");
    if (n_cols > 0x7fffffff)
        return set_error(QSSB_ERR_INVALID, "qssb_scan_fft_half_mapped: too many columns");
    cudaStream_t s = (cudaStream_t)stream;
    const size_t smem = ScanFft128PSmem::bytes;
    CUDA_TRY(cudaFuncSetAttribute(k_scan_fft128p, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem));
    const int slots = 2 * device_sm_count();
    const int grid = n_bf < slots ? n_bf : slots;
    { k_scan_fft128p<<<grid, 256, smem, s>>>(columns, n_bf, reinterpret_cast<float2*>(g_half), map,
                                           (int)n_cols); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}
