// qssb_export.cu - the exact bright-field companion file: the selected BF
// detector pixels of every frame written BF-major ([bf][scan], u8 or u16),
// the browser transport the reference writes next to a reconstruction
// (ssb/compute/cuda/engine.py:577-701).
//
// Two kernels:
//  * k_count_max: the largest count of the whole loaded block (the reference
//    narrows u16 to u8 only when the entire block fits, engine.py:603-604).
//    16-byte streaming loads, per-lane packed max (__vmaxu2 / __vmaxu4), a
//    warp max and one atomicMax per warp. HBM-bound: one read of the block.
//  * k_export_bf: a gather-transpose of 32 BF pixels x 64 frames per CTA:
//    each warp reads one frame's 32 BF counts, the tile is staged in shared
//    memory, and each BF row of 64 frames leaves as one coalesced run.
#include "qssb_internal.h"

using namespace qssb;

namespace {

__device__ __forceinline__ uint32_t packed_max(uint32_t a, uint32_t b, int elem_bytes) {
    return elem_bytes == 1 ? __vmaxu4(a, b) : __vmaxu2(a, b);
}

__device__ __forceinline__ uint32_t unpack_max(uint32_t w, int elem_bytes) {
    if (elem_bytes == 2) return max(w & 0xffffu, w >> 16);
    uint32_t m = max(w & 0xffu, (w >> 8) & 0xffu);
    m = max(m, (w >> 16) & 0xffu);
    return max(m, w >> 24);
}

// Largest element of n_bytes / elem_bytes unsigned counts. `vec` is the
// 16-byte-aligned body (n_vec words), `head` / `tail` the unaligned ends
// (n_head / n_tail elements), read as scalars.
__global__ void k_count_max(const uint4* __restrict__ vec, int64_t n_vec,
                            const unsigned char* __restrict__ head, int n_head,
                            const unsigned char* __restrict__ tail, int n_tail, int elem_bytes,
                            uint32_t* __restrict__ out) {
    uint32_t w = 0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_vec; i += stride) {
        const uint4 v = __ldcs(vec + i);
        w = packed_max(w, v.x, elem_bytes);
        w = packed_max(w, v.y, elem_bytes);
        w = packed_max(w, v.z, elem_bytes);
        w = packed_max(w, v.w, elem_bytes);
    }
    uint32_t m = unpack_max(w, elem_bytes);
    if (blockIdx.x == 0) {
        for (int i = threadIdx.x; i < n_head + n_tail; i += blockDim.x) {
            const unsigned char* p = i < n_head ? head + (int64_t)i * elem_bytes
                                                : tail + (int64_t)(i - n_head) * elem_bytes;
            const uint32_t v = elem_bytes == 1 ? (uint32_t)p[0]
                                               : (uint32_t)(*reinterpret_cast<const uint16_t*>(p));
            m = max(m, v);
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, off));
    if ((threadIdx.x & 31) == 0 && m != 0) atomicMax(out, m);
}

constexpr int kExportBf = 32;      // BF pixels per tile
constexpr int kExportFrames = 64;  // frames per tile

template <typename Tin, typename Tout>
__global__ void __launch_bounds__(256) k_export_bf(const Tin* __restrict__ counts, int64_t n_scan,
                                                   int64_t det_pixels,
                                                   const int32_t* __restrict__ bf_linear,
                                                   int n_bf, Tout* __restrict__ out) {
    __shared__ Tout tile[kExportBf][kExportFrames + 2];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t f0 = (int64_t)blockIdx.x * kExportFrames;
    const int b0 = blockIdx.y * kExportBf;
    const int b = b0 + lane;
    int64_t pix = -1;
    if (b < n_bf) {
        const int32_t p = bf_linear[b];
        if (p >= 0 && (int64_t)p < det_pixels) pix = p;
    }
    // gather: warp w reads frames w, w + 8, ... of the tile (32 BF counts each)
    for (int f = warp; f < kExportFrames; f += 8) {
        const int64_t frame = f0 + f;
        Tout v = 0;
        if (pix >= 0 && frame < n_scan) v = (Tout)__ldg(counts + frame * det_pixels + pix);
        tile[lane][f] = v;
    }
    __syncthreads();
    // store: each BF row's 64 frames as one contiguous run
    const int f = threadIdx.x & (kExportFrames - 1);
    const int64_t frame = f0 + f;
    if (frame >= n_scan) return;
    for (int r = threadIdx.x / kExportFrames; r < kExportBf; r += 256 / kExportFrames) {
        if (b0 + r < n_bf) out[(int64_t)(b0 + r) * n_scan + frame] = tile[r][f];
    }
}

template <typename Tin, typename Tout>
cudaError_t launch_export(const void* counts, int64_t n_scan, int64_t det_pixels,
                          const int32_t* bf_linear, int n_bf, void* out, cudaStream_t st) {
    const dim3 grid((unsigned)((n_scan + kExportFrames - 1) / kExportFrames),
                    (unsigned)((n_bf + kExportBf - 1) / kExportBf));
    { k_export_bf<Tin, Tout><<<grid, 256, 0, st>>>(static_cast<const Tin*>(counts), n_scan,
                                                 det_pixels, bf_linear, n_bf,
                                                 static_cast<Tout*>(out)); note_launch(); }
    return cudaGetLastError();
}

}  // namespace

extern "C" int qssb_count_max(const void* counts, int32_t elem_bytes, int64_t n,
                              uint32_t* max_out, void* stream) {
    if (elem_bytes != 1 && elem_bytes != 2)
        return set_error(QSSB_ERR_INVALID, "qssb_count_max: elem_bytes must be 1 (u8) or 2 (u16)");
    if (n < 0 || (n > 0 && counts == nullptr) || max_out == nullptr)
        return set_error(QSSB_ERR_INVALID, "qssb_count_max: null pointer or negative size");
    const uintptr_t base = reinterpret_cast<uintptr_t>(counts);
    if (elem_bytes == 2 && (base & 1))
        return set_error(QSSB_ERR_INVALID, "qssb_count_max: u16 counts must be 2-byte aligned");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    CUDA_TRY(cudaMemsetAsync(max_out, 0, sizeof(uint32_t), st));
    if (n == 0) return QSSB_OK;
    const int64_t bytes = n * elem_bytes;
    // unaligned head up to the first 16-byte boundary (counts are whole elements,
    // and a u16 pointer is 2-byte aligned, so the boundary falls between elements)
    int64_t head_bytes = (int64_t)((16 - (base & 15)) & 15);
    if (head_bytes > bytes) head_bytes = bytes;
    const int64_t n_vec = (bytes - head_bytes) / 16;
    const int64_t tail_bytes = bytes - head_bytes - n_vec * 16;
    const auto* bytes_p = static_cast<const unsigned char*>(counts);
    const int sms = device_sm_count();
    int64_t blocks = (n_vec + 255) / 256;
    if (blocks > (int64_t)sms * 8) blocks = (int64_t)sms * 8;
    if (blocks < 1) blocks = 1;
    { k_count_max<<<(unsigned)blocks, 256, 0, st>>>(
        reinterpret_cast<const uint4*>(bytes_p + head_bytes), n_vec, bytes_p,
        (int)(head_bytes / elem_bytes), bytes_p + head_bytes + n_vec * 16,
        (int)(tail_bytes / elem_bytes), elem_bytes, max_out); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}

extern "C" int qssb_export_bf_columns(const void* counts, int32_t in_bytes, int64_t n_scan,
                                      int64_t det_pixels, const int32_t* bf_linear,
                                      int32_t n_bf, void* out, int32_t out_bytes, void* stream) {
    if ((in_bytes != 1 && in_bytes != 2) || (out_bytes != 1 && out_bytes != 2))
        return set_error(QSSB_ERR_INVALID,
                         "qssb_export_bf_columns: element sizes must be 1 (u8) or 2 (u16)");
    if (n_scan < 0 || det_pixels <= 0 || n_bf < 0 || det_pixels > INT32_MAX)
        return set_error(QSSB_ERR_INVALID, "qssb_export_bf_columns: invalid sizes");
    if (n_scan == 0 || n_bf == 0) return QSSB_OK;
    if (!counts || !bf_linear || !out)
        return set_error(QSSB_ERR_INVALID, "qssb_export_bf_columns: null pointer");
    if ((n_bf + kExportBf - 1) / kExportBf > 65535 ||
        (n_scan + kExportFrames - 1) / kExportFrames > (int64_t)INT32_MAX)
        return set_error(QSSB_ERR_UNSUPPORTED, "qssb_export_bf_columns: too many BF pixels or frames");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t err;
    if (in_bytes == 2 && out_bytes == 2)
        err = launch_export<uint16_t, uint16_t>(counts, n_scan, det_pixels, bf_linear, n_bf, out, st);
    else if (in_bytes == 2)
        err = launch_export<uint16_t, uint8_t>(counts, n_scan, det_pixels, bf_linear, n_bf, out, st);
    else if (out_bytes == 2)
        err = launch_export<uint8_t, uint16_t>(counts, n_scan, det_pixels, bf_linear, n_bf, out, st);
    else
        err = launch_export<uint8_t, uint8_t>(counts, n_scan, det_pixels, bf_linear, n_bf, out, st);
    CUDA_TRY(err);
    return QSSB_OK;
}
