// qssb_decode.cu - HDF5 bitshuffle + LZ4 chunks of u16 detector frames <-> device frames.
//
// The step before the SSB path: the reference reads 4D-STEM acquisitions as
// HDF5 chunks (one detector frame each) compressed by the bitshuffle filter
// with LZ4 (io/load.py:3271-3320, io/backends/cuda/decoder.py:258-403 of
// bobleesj/quantem.gpu) and writes them the same way (io/save.py,
// decoder.py:496-1003). Chunk format: big-endian uint64 uncompressed bytes,
// big-endian uint32 block bytes (8192), then per block a big-endian uint32
// compressed size and an LZ4 block of the bit-shuffled elements (bit plane b
// = bit b of every element, byte k of a plane = elements 8k..8k+7, element
// 8k+j in bit j); the last block holds the rest rounded down to 8 elements;
// the remaining < 8 elements follow raw.
//
// Decode: one CTA per chunk. Thread 0 walks the block chain (every offset
// checked against the chunk's end); each warp decodes a block's LZ4
// sequences into shared memory (every lane parses the token stream through
// L1, all lanes copy literals and matches - a match byte j reads
// out[op - off + j mod off], so overlapping matches need no serial copy) and
// bit-unshuffles the block with 8x8 bit transposes straight into the u16
// frame (16-byte stores). A malformed chunk sets status[c] (the block is
// zero-filled); nothing traps.
// Encode: the same transposes forward, a greedy LZ4 compressor per block
// (lane 0, a 4096-entry hash table in shared memory) into fixed-stride
// slots, then a pack kernel that lays out the chunks at caller offsets.
#include "qssb_internal.h"

namespace qssb {

constexpr int kDecWarps = 4;
constexpr int kBlockBytes = 8192;                         // bytes per shuffled block
constexpr int kBlockElems = kBlockBytes / 2;
constexpr int kLz4Bound = kBlockBytes + kBlockBytes / 255 + 16;  // LZ4 worst case
constexpr int kMaxBlocks = 512;                           // 4 MB frames
constexpr int kEncHash = 4096;

// Status codes written per chunk.
constexpr int kStOk = 0;
constexpr int kStHeader = 1;    // header size / block size / chunk too short
constexpr int kStChain = 2;     // a block extends past the chunk's end
constexpr int kStLz4 = 3;       // malformed LZ4 sequence or wrong decoded size

__device__ __forceinline__ uint32_t be32(const uint8_t* p) {
    return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | (uint32_t)p[3];
}

// 8x8 bit transpose (byte i = row i, bit j = column j), three delta swaps.
__device__ __forceinline__ uint64_t transpose8(uint64_t x) {
    uint64_t t = (x ^ (x >> 7)) & 0x00AA00AA00AA00AAull;
    x = x ^ t ^ (t << 7);
    t = (x ^ (x >> 14)) & 0x0000CCCC0000CCCCull;
    x = x ^ t ^ (t << 14);
    t = (x ^ (x >> 28)) & 0x00000000F0F0F0F0ull;
    x = x ^ t ^ (t << 28);
    return x;
}

// Decode one LZ4 block from in[0, csz) (global memory, read through L1) into
// out[0, cap) (shared memory) by the whole warp. Every lane parses the token
// stream itself (the same bytes: broadcast reads, uniform control flow, no
// shuffles); literal and match bytes are copied lane-parallel. Returns true
// when the stream is well formed and fills exactly cap bytes.
__device__ bool lz4_block_warp(const uint8_t* __restrict__ in, int csz, uint8_t* out, int cap,
                               int lane) {
    int ip = 0, op = 0;
    for (int guard = 0; guard < kBlockBytes + 1; ++guard) {
        if (ip >= csz) return false;
        const int token = __ldg(in + ip++);
        int lit = token >> 4;
        if (lit == 15) {
            int b;
            do {
                if (ip >= csz) return false;
                b = __ldg(in + ip++);
                lit += b;
            } while (b == 255 && lit <= cap);
        }
        if (lit > cap - op || lit > csz - ip) return false;
        for (int j = lane; j < lit; j += 32) out[op + j] = __ldg(in + ip + j);
        ip += lit;
        op += lit;
        if (ip == csz) {
            __syncwarp();
            return op == cap;
        }
        if (ip + 2 > csz) return false;
        const int off = __ldg(in + ip) | (__ldg(in + ip + 1) << 8);
        ip += 2;
        int ml = (token & 15) + 4;
        if ((token & 15) == 15) {
            int b;
            do {
                if (ip >= csz) return false;
                b = __ldg(in + ip++);
                ml += b;
            } while (b == 255 && ml <= cap);
        }
        if (off == 0 || off > op || ml > cap - op) return false;
        __syncwarp();  // literals (and earlier matches) visible to the match reads
        if (off >= ml) {  // no self-overlap: a plain copy
            for (int j = lane; j < ml; j += 32) out[op + j] = out[op - off + j];
        } else {
            // out[op + j] = out[op - off + (j mod off)]: reads only bytes before op
            int r = lane % off;
            const int step = 32 % off;
            for (int j = lane; j < ml; j += 32) {
                out[op + j] = out[op - off + r];
                r += step;
                if (r >= off) r -= off;
            }
        }
        op += ml;
        __syncwarp();
    }
    return false;
}

// Bit-unshuffle cnt (a multiple of 8) elements from a block's planes into dst.
__device__ __forceinline__ void unshuffle_store(const uint8_t* planes, int cnt, uint16_t* dst,
                                                bool vec, int lane) {
    const int P = cnt / 8;
    for (int p = lane; p < P; p += 32) {
        uint64_t lo = 0, hi = 0;
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            lo |= (uint64_t)planes[b * P + p] << (8 * b);
            hi |= (uint64_t)planes[(8 + b) * P + p] << (8 * b);
        }
        lo = transpose8(lo);  // byte j: bits 0..7 of element 8p + j
        hi = transpose8(hi);  // byte j: bits 8..15
        uint32_t w[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const uint32_t e0 = (uint32_t)((lo >> (16 * q)) & 0xff) | ((uint32_t)((hi >> (16 * q)) & 0xff) << 8);
            const uint32_t e1 = (uint32_t)((lo >> (16 * q + 8)) & 0xff) | ((uint32_t)((hi >> (16 * q + 8)) & 0xff) << 8);
            w[q] = e0 | (e1 << 16);
        }
        uint16_t* o = dst + 8 * p;
        if (vec) {
            *reinterpret_cast<uint4*>(o) = make_uint4(w[0], w[1], w[2], w[3]);
        } else {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                o[2 * q] = (uint16_t)(w[q] & 0xffff);
                o[2 * q + 1] = (uint16_t)(w[q] >> 16);
            }
        }
    }
}

struct DecSmem {
    int start[kMaxBlocks];  // block's LZ4 data offset within the chunk
    int size[kMaxBlocks];
    int tail_at;            // raw leftover elements' offset
    int status;
};

__global__ void __launch_bounds__(32 * kDecWarps) k_decode_bslz4_u16(
    const uint8_t* __restrict__ comp, long long comp_bytes, const long long* __restrict__ offsets,
    int n_chunks, long long chunk_bytes, uint16_t* __restrict__ out, int* __restrict__ status) {
    extern __shared__ uint4 dec_smem4[];
    uint8_t* wbuf = reinterpret_cast<uint8_t*>(dec_smem4);  // per warp: one decoded block
    __shared__ DecSmem sh;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int c = blockIdx.x;
    const long long n_elem = chunk_bytes / 2;
    const long long n8 = n_elem & ~7LL;
    const int n_blocks = (int)((n8 + kBlockElems - 1) / kBlockElems);
    const long long c0 = offsets[c];
    const long long c1 = c + 1 < n_chunks ? offsets[c + 1] : comp_bytes;
    const uint8_t* ch = comp + c0;
    const long long len = c1 - c0;
    if (c0 >= 0 && c1 <= comp_bytes) {
        // the chunk's bytes into L1 (one prefetch per 128-byte line) before the
        // serial block-chain walk and the parses read them
        for (long long i = (long long)tid * 128; i < len; i += 128LL * 32 * kDecWarps)
            asm volatile("prefetch.global.L1 [%0];" ::"l"(ch + i));
    }
    __syncthreads();
    if (tid == 0) {
        int st = kStOk;
        if (c0 < 0 || c1 > comp_bytes || len < 12) {
            st = kStHeader;
        } else {
            unsigned long long total = 0;
            for (int i = 0; i < 8; ++i) total = (total << 8) | ch[i];
            if ((long long)total != chunk_bytes || be32(ch + 8) != (uint32_t)kBlockBytes) st = kStHeader;
        }
        long long pos = 12;
        for (int i = 0; i < n_blocks && st == kStOk; ++i) {
            if (pos + 4 > len) { st = kStChain; break; }
            const long long csz = be32(ch + pos);
            if (csz > kLz4Bound || pos + 4 + csz > len) { st = kStChain; break; }
            sh.start[i] = (int)(pos + 4);
            sh.size[i] = (int)csz;
            pos += 4 + csz;
        }
        if (st == kStOk && pos + (n_elem - n8) * 2 > len) st = kStChain;
        sh.tail_at = (int)pos;
        sh.status = st;
        if (status) status[c] = st;  // blocks that fail raise it below
    }
    __syncthreads();
    uint16_t* frame = out + (size_t)c * n_elem;
    const bool vec = (n_elem & 7) == 0 && ((uintptr_t)out & 15u) == 0;
    if (sh.status != kStOk) {
        for (long long i = tid; i < n_elem; i += 32 * kDecWarps) frame[i] = 0;
        return;
    }
    uint8_t* out_buf = wbuf + (size_t)warp * kBlockBytes;
    for (int i = warp; i < n_blocks; i += kDecWarps) {
        const long long e0 = (long long)i * kBlockElems;
        const int cnt = (int)min((long long)kBlockElems, n8 - e0);
        const bool good = lz4_block_warp(ch + sh.start[i], sh.size[i], out_buf, 2 * cnt, lane);
        if (good) {
            unshuffle_store(out_buf, cnt, frame + e0, vec, lane);
        } else {
            for (int j = lane; j < cnt; j += 32) frame[e0 + j] = 0;
            if (lane == 0 && status) atomicMax(status + c, kStLz4);
        }
        __syncwarp();
    }
    if (warp == 0) {  // raw leftover elements
        const uint8_t* raw = ch + sh.tail_at;
        for (long long j = n8 + lane; j < n_elem; j += 32) {
            const long long b = (j - n8) * 2;
            frame[j] = (uint16_t)(raw[b] | (raw[b + 1] << 8));
        }
    }
}

// ------------------------------------------------------------------ encode
// Scratch layout: per (chunk, block) a slot of kEncSlot bytes holding the
// big-endian compressed size followed by the LZ4 block.
constexpr int kEncSlot = (4 + kLz4Bound + 15) & ~15;

__device__ __forceinline__ uint32_t rd32(const uint8_t* p) {
    return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}

__global__ void __launch_bounds__(32 * kDecWarps) k_encode_bslz4_u16(
    const uint16_t* __restrict__ frames, int n_chunks, long long chunk_bytes,
    uint8_t* __restrict__ scratch) {
    extern __shared__ uint4 enc_smem4[];
    uint8_t* base = reinterpret_cast<uint8_t*>(enc_smem4);
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int c = blockIdx.x;
    const long long n_elem = chunk_bytes / 2;
    const long long n8 = n_elem & ~7LL;
    const int n_blocks = (int)((n8 + kBlockElems - 1) / kBlockElems);
    uint8_t* planes = base + (size_t)warp * (kBlockBytes + 2 * kEncHash);
    uint16_t* table = reinterpret_cast<uint16_t*>(planes + kBlockBytes);
    const uint16_t* frame = frames + (size_t)c * n_elem;
    for (int i = warp; i < n_blocks; i += kDecWarps) {
        const long long e0 = (long long)i * kBlockElems;
        const int cnt = (int)min((long long)kBlockElems, n8 - e0);
        const int P = cnt / 8;
        for (int p = lane; p < P; p += 32) {  // forward bit shuffle
            uint64_t lo = 0, hi = 0;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const uint16_t v = frame[e0 + 8 * p + j];
                lo |= (uint64_t)(v & 0xff) << (8 * j);
                hi |= (uint64_t)(v >> 8) << (8 * j);
            }
            lo = transpose8(lo);
            hi = transpose8(hi);
#pragma unroll
            for (int b = 0; b < 8; ++b) {
                planes[b * P + p] = (uint8_t)(lo >> (8 * b));
                planes[(8 + b) * P + p] = (uint8_t)(hi >> (8 * b));
            }
        }
        for (int h = lane; h < kEncHash; h += 32) table[h] = 0xffff;
        __syncwarp();
        if (lane == 0) {  // greedy LZ4 (last 5 bytes literal, no match in the last 12)
            const int n = 2 * cnt;
            uint8_t* slot = scratch + ((size_t)c * n_blocks + i) * kEncSlot;
            uint8_t* o = slot + 4;
            int op = 0, anchor = 0, ip = 0;
            auto put_len = [&](int x) {
                while (x >= 255) { o[op++] = 255; x -= 255; }
                o[op++] = (uint8_t)x;
            };
            while (ip < n - 12) {
                const uint32_t v = rd32(planes + ip);
                const uint32_t h = (v * 2654435761u) >> 20;
                const int cand = table[h];
                table[h] = (uint16_t)ip;
                if (cand != 0xffff && rd32(planes + cand) == v) {
                    int m = 4;
                    while (ip + m < n - 5 && planes[cand + m] == planes[ip + m]) ++m;
                    const int lit = ip - anchor;
                    o[op++] = (uint8_t)((min(lit, 15) << 4) | min(m - 4, 15));
                    if (lit >= 15) put_len(lit - 15);
                    for (int k = 0; k < lit; ++k) o[op++] = planes[anchor + k];
                    const int off = ip - cand;
                    o[op++] = (uint8_t)(off & 0xff);
                    o[op++] = (uint8_t)(off >> 8);
                    if (m - 4 >= 15) put_len(m - 4 - 15);
                    ip += m;
                    anchor = ip;
                } else {
                    ++ip;
                }
            }
            const int lit = n - anchor;
            o[op++] = (uint8_t)(min(lit, 15) << 4);
            if (lit >= 15) put_len(lit - 15);
            for (int k = 0; k < lit; ++k) o[op++] = planes[anchor + k];
            slot[0] = (uint8_t)(op >> 24);
            slot[1] = (uint8_t)(op >> 16);
            slot[2] = (uint8_t)(op >> 8);
            slot[3] = (uint8_t)op;
        }
        __syncwarp();
    }
}

// sizes[c] = bytes of chunk c: header, the blocks with their size words, raw leftovers.
__global__ void k_bslz4_chunk_sizes(const uint8_t* __restrict__ scratch, int n_chunks,
                                    long long chunk_bytes, long long* __restrict__ sizes) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_chunks) return;
    const long long n_elem = chunk_bytes / 2;
    const long long n8 = n_elem & ~7LL;
    const int n_blocks = (int)((n8 + kBlockElems - 1) / kBlockElems);
    long long total = 12 + (n_elem - n8) * 2;
    for (int i = 0; i < n_blocks; ++i) total += 4 + be32(scratch + ((size_t)c * n_blocks + i) * kEncSlot);
    sizes[c] = total;
}

__global__ void __launch_bounds__(256) k_bslz4_pack(const uint8_t* __restrict__ scratch,
                                                    const uint16_t* __restrict__ frames,
                                                    int n_chunks, long long chunk_bytes,
                                                    const long long* __restrict__ offsets,
                                                    uint8_t* __restrict__ packed) {
    const int c = blockIdx.x;
    const int tid = threadIdx.x;
    const long long n_elem = chunk_bytes / 2;
    const long long n8 = n_elem & ~7LL;
    const int n_blocks = (int)((n8 + kBlockElems - 1) / kBlockElems);
    uint8_t* dst = packed + offsets[c];
    if (tid < 12) {
        dst[tid] = tid < 8 ? (uint8_t)((unsigned long long)chunk_bytes >> (8 * (7 - tid)))
                           : (uint8_t)((uint32_t)kBlockBytes >> (8 * (11 - tid)));
    }
    long long pos = 12;
    for (int i = 0; i < n_blocks; ++i) {
        const uint8_t* slot = scratch + ((size_t)c * n_blocks + i) * kEncSlot;
        const int len = 4 + (int)be32(slot);
        for (int j = tid; j < len; j += 256) dst[pos + j] = slot[j];
        pos += len;
    }
    const uint16_t* frame = frames + (size_t)c * n_elem;
    for (long long j = n8 + tid; j < n_elem; j += 256) {
        const uint16_t v = frame[j];
        dst[pos + 2 * (j - n8)] = (uint8_t)(v & 0xff);
        dst[pos + 2 * (j - n8) + 1] = (uint8_t)(v >> 8);
    }
}

static int check_chunk_bytes(long long chunk_bytes, const char* who) {
    if (chunk_bytes < 2 || (chunk_bytes & 1) || chunk_bytes / 2 / kBlockElems >= kMaxBlocks)
        return set_error(QSSB_ERR_INVALID, who);
    return QSSB_OK;
}

}  // namespace qssb

using namespace qssb;

extern "C" int qssb_decode_bslz4_u16(const uint8_t* compressed, int64_t compressed_bytes,
                                     const int64_t* chunk_offsets, int32_t n_chunks,
                                     int64_t chunk_bytes, uint16_t* out, int32_t* status,
                                     void* stream) {
    if (!compressed || !chunk_offsets || !out || n_chunks <= 0 || compressed_bytes <= 0)
        return set_error(QSSB_ERR_INVALID, "qssb_decode_bslz4_u16: null pointer or empty input");
    int rc = check_chunk_bytes(chunk_bytes, "qssb_decode_bslz4_u16: chunk_bytes must be even, "
                                            "at most 4 MB");
    if (rc) return rc;
    const size_t smem = (size_t)kDecWarps * kBlockBytes;
    CUDA_TRY(cudaFuncSetAttribute(k_decode_bslz4_u16, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem));
    { k_decode_bslz4_u16<<<n_chunks, 32 * kDecWarps, smem, (cudaStream_t)stream>>>(
        compressed, compressed_bytes, reinterpret_cast<const long long*>(chunk_offsets), n_chunks,
        chunk_bytes, out, status); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}

extern "C" int qssb_encode_bslz4_scratch_bytes(int32_t n_chunks, int64_t chunk_bytes,
                                               size_t* bytes) {
    if (!bytes || n_chunks <= 0)
        return set_error(QSSB_ERR_INVALID, "qssb_encode_bslz4_scratch_bytes: bad arguments");
    int rc = check_chunk_bytes(chunk_bytes, "qssb_encode_bslz4_scratch_bytes: chunk_bytes must be "
                                            "even, at most 4 MB");
    if (rc) return rc;
    const long long n8 = (chunk_bytes / 2) & ~7LL;
    const long long n_blocks = (n8 + kBlockElems - 1) / kBlockElems;
    *bytes = (size_t)n_chunks * (size_t)n_blocks * kEncSlot;
    return QSSB_OK;
}

extern "C" int qssb_encode_bslz4_u16(const uint16_t* frames, int32_t n_chunks, int64_t chunk_bytes,
                                     uint8_t* scratch, int64_t* chunk_sizes, void* stream) {
    if (!frames || !scratch || !chunk_sizes || n_chunks <= 0)
        return set_error(QSSB_ERR_INVALID, "qssb_encode_bslz4_u16: null pointer or empty input");
    int rc = check_chunk_bytes(chunk_bytes, "qssb_encode_bslz4_u16: chunk_bytes must be even, "
                                            "at most 4 MB");
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t smem = (size_t)kDecWarps * (kBlockBytes + 2 * kEncHash);
    CUDA_TRY(cudaFuncSetAttribute(k_encode_bslz4_u16, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem));
    { k_encode_bslz4_u16<<<n_chunks, 32 * kDecWarps, smem, s>>>(frames, n_chunks, chunk_bytes, scratch); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    { k_bslz4_chunk_sizes<<<(n_chunks + 255) / 256, 256, 0, s>>>(
        scratch, n_chunks, chunk_bytes, reinterpret_cast<long long*>(chunk_sizes)); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}

extern "C" int qssb_pack_bslz4(const uint8_t* scratch, const uint16_t* frames, int32_t n_chunks,
                               int64_t chunk_bytes, const int64_t* chunk_offsets, uint8_t* packed,
                               void* stream) {
    if (!scratch || !frames || !chunk_offsets || !packed || n_chunks <= 0)
        return set_error(QSSB_ERR_INVALID, "qssb_pack_bslz4: null pointer or empty input");
    int rc = check_chunk_bytes(chunk_bytes, "qssb_pack_bslz4: chunk_bytes must be even, at most 4 MB");
    if (rc) return rc;
    { k_bslz4_pack<<<n_chunks, 256, 0, (cudaStream_t)stream>>>(
        scratch, frames, n_chunks, chunk_bytes, reinterpret_cast<const long long*>(chunk_offsets),
        packed); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}
