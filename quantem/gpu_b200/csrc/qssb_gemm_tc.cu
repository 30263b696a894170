// qssb_gemm_tc.cu - the proposer MLP's large GEMMs on the 5th-generation
// tensor cores (tcgen05): C[M][N] (+)= op(A)[M][K] op(B)[K][N], BF16 operands,
// FP32 accumulation in tensor memory. No counterpart in the reference.
//
// One CTA (4 warps, two CTAs per SM) per 128 x 128 output tile and K range
// (split K): the tile's operands are staged in shared memory 64 K-elements at
// a time by cp.async in a three-stage ring, in the no-swizzle canonical
// layouts of the MMA's shared-memory descriptors (8 x 16-byte core matrices;
// a K-major operand keeps 8 consecutive k of a row in one 16-byte unit, an
// MN-major one 8 consecutive rows of one k). Each thread's copies are
// ordered so that a quarter-warp writes eight different 16-byte bank groups.
// One thread issues the four 128 x 128 x 16 MMAs of a stage (tcgen05.mma
// kind::f16) and commits them to the stage's mbarrier; a stage is refilled
// once that barrier shows its MMAs done, so loads of the next two k-tiles
// overlap the MMAs of the current one. The accumulator lives in 128 TMEM
// columns; the epilogue reads it with tcgen05.ld (each warp its 32 lanes =
// rows). Without split K it applies bias / accumulate / GELU and writes C
// directly; with it, FP32 partial tiles [split][M][N] go to the workspace and
// k_gemm_tc_reduce adds the splits in a fixed order and applies them. Every
// mbarrier wait is bounded; a wait that runs out sets *status and the CTA
// skips its epilogue.
#include <cuda_bf16.h>
#include <math.h>

#include "qssb_internal.h"

namespace qssb {

namespace tc {

constexpr int BM = 128, BN = 128, BK = 64, STAGES = 3, THREADS = 128;
constexpr int TILE_BYTES = BM * BK * 2;          // 16 KB per operand per stage (BM == BN)
constexpr int SMEM_BYTES = STAGES * 2 * TILE_BYTES;
constexpr long long kWaitLimit = 1LL << 26;      // try_wait polls before giving up

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor, no swizzle: start >> 4 in bits 0..13,
// leading byte offset >> 4 in 16..29, stride byte offset >> 4 in 32..45,
// version 1 in bits 46..47, layout type 0 (no swizzle) in 61..63.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator (bits 4..5 = 1),
// BF16 A and B (bits 7..9, 10..12 = 1), A / B major (bit 15 / 16: 0 K-major,
// 1 MN-major), N >> 3 in bits 17..22, M >> 4 in bits 24..28.
__host__ __device__ constexpr uint32_t instr_desc(int a_mn_major, int b_mn_major) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn_major << 15) |
           ((uint32_t)b_mn_major << 16) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (long long it = 0; it < kWaitLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Offset in bytes of element (mn, k) of a BM x BK stage tile.
//  K-major:  (k / 8) * (BM / 8 * 128) + (mn / 8) * 128 + (mn % 8) * 16 + (k % 8) * 2
//            LBO (next 8 k) = BM / 8 * 128, SBO (next 8 rows) = 128
//  MN-major: (k / 8) * (BM / 8 * 128) + (mn / 8) * 128 + (k % 8) * 16 + (mn % 8) * 2
//            LBO (next 8 k) = BM / 8 * 128, SBO (next 8 rows) = 128
constexpr uint32_t kLbo = BM / 8 * 128;
constexpr uint32_t kSbo = 128;

// Stage one operand tile by cp.async: rows [r0, r0 + 128) of op(X) (M or N
// side), k in [k0, k0 + 64). X is row-major with leading dimension ld;
// kmajor: X[row][k] (k contiguous), else X[k][row] (rows contiguous). Unit u
// of the 1024 16-byte units goes to shared offset 16 u in both layouts'
// orders (conflict-free stores): K-major u = kg * 128 + row (a thread walks
// one row's eight 16-byte pieces over its eight units, so the L1-allocating
// copies reuse each line), MN-major u = kg * 128 + rowgroup * 8 + k % 8.
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" :: "r"(dst), "l"(src) : "memory");
}

__device__ __forceinline__ void stage_tile_async(uint32_t dst, const __nv_bfloat16* __restrict__ X,
                                                 int ld, bool kmajor, int r0, int k0, int tid) {
#pragma unroll
    for (int it = 0; it < (BM * BK / 8) / THREADS; ++it) {
        const int u = tid + it * THREADS;  // 16-byte unit, in shared-memory order
        const int kg = u >> 7;             // which 8 k
        const __nv_bfloat16* src;
        if (kmajor) {
            const int row = u & 127;
            src = X + (size_t)(r0 + row) * ld + (k0 + kg * 8);
        } else {
            const int rg = (u >> 3) & 15;  // which 8 rows
            const int kk = kg * 8 + (u & 7);
            src = X + (size_t)(k0 + kk) * ld + (r0 + rg * 8);
        }
        cp_async16(dst + 16u * (uint32_t)u, src);
    }
}

__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;" ::: "memory");
}

template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" :: "n"(N) : "memory");
}

__device__ __forceinline__ float gelu_tc(float x) {
    const float s = 0.7978845608028654f;
    const float u = s * fmaf(0.044715f * x * x, x, x);
    return 0.5f * x * (1.0f + tanhf(u));
}

template <bool TA, bool TB>
__global__ void __launch_bounds__(THREADS, 2) k_gemm_tc(
    const __nv_bfloat16* __restrict__ A, int lda, const __nv_bfloat16* __restrict__ B, int ldb,
    int M, int N, int k_per_split, float* __restrict__ part, int* __restrict__ status,
    const float* __restrict__ bias, int accumulate, float* __restrict__ C, int ldc,
    __nv_bfloat16* __restrict__ act, int ld_act) {
    extern __shared__ __align__(128) char smem[];
    __shared__ __align__(8) uint64_t bars[STAGES];
    __shared__ uint32_t s_tmem;
    __shared__ int s_fail;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int n0 = blockIdx.x * BN, m0 = blockIdx.y * BM, split = blockIdx.z;
    const int kbeg = split * k_per_split;
    const int ktiles = k_per_split / BK;
    // A K-major when not transposed; B K-major when transposed (stored [N][K])
    constexpr bool a_kmajor = !TA, b_kmajor = TB;
    constexpr uint32_t idesc = instr_desc(a_kmajor ? 0 : 1, b_kmajor ? 0 : 1);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(&s_tmem)), "r"(BN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        s_fail = 0;
        for (int s = 0; s < STAGES; ++s)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&bars[s])));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    const uint32_t smem_base = smem_u32(smem);
    auto load_tile = [&](int kt) {
        const uint32_t a_addr = smem_base + (kt % STAGES) * 2 * TILE_BYTES;
        const int k0 = kbeg + kt * BK;
        stage_tile_async(a_addr, A, lda, a_kmajor, m0, k0, tid);
        stage_tile_async(a_addr + TILE_BYTES, B, ldb, b_kmajor, n0, k0, tid);
    };
    // prologue: the first STAGES - 1 tiles in flight (one commit group each)
#pragma unroll
    for (int kt = 0; kt < STAGES - 1; ++kt) {
        if (kt < ktiles) load_tile(kt);
        cp_async_commit();
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = s_tmem;
    for (int kt = 0; kt < ktiles; ++kt) {
        const int st = kt % STAGES;
        cp_async_wait<STAGES - 2>();  // this thread's copies of tile kt have landed
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // -> the tensor core
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
        if (s_fail) break;
        asm volatile("tcgen05.fence::after_thread_sync;");
        if (tid == 0) {
            const uint32_t a_addr = smem_base + st * 2 * TILE_BYTES;
            const uint32_t b_addr = a_addr + TILE_BYTES;
#pragma unroll
            for (int ks = 0; ks < BK / 16; ++ks) {  // 16 k per MMA = two 8-k core columns
                const uint64_t ad = smem_desc(a_addr + ks * 2 * kLbo, kLbo, kSbo);
                const uint64_t bd = smem_desc(b_addr + ks * 2 * kLbo, kLbo, kSbo);
                const uint32_t acc = (kt > 0 || ks > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}"
                    :: "r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0u));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         :: "r"(smem_u32(&bars[st])) : "memory");
        }
        // refill: tile kt + STAGES - 1 goes to the stage tile kt - 1 used, once
        // the MMAs that read it are done
        const int nt = kt + STAGES - 1;
        if (nt < ktiles) {
            if (kt >= 1 && !mbar_wait(smem_u32(&bars[(kt - 1) % STAGES]), ((kt - 1) / STAGES) & 1))
                s_fail = 1;
            else
                load_tile(nt);
        }
        cp_async_commit();
    }
    cp_async_wait<0>();
    // the last commit covers every MMA issued before it
    if (!s_fail && ktiles > 0) {
        const int last = ktiles - 1;
        if (!mbar_wait(smem_u32(&bars[last % STAGES]), (last / STAGES) & 1)) s_fail = 1;
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (!s_fail) {
        // warp w reads TMEM lanes 32 w .. 32 w + 31 (rows), 32 columns at a time
        const int row = m0 + warp * 32 + (tid & 31);
        const bool direct = gridDim.z == 1;
        float* out = part + ((size_t)split * M + row) * N + n0;
#pragma unroll 1
        for (int c = 0; c < BN; c += 32) {
            uint32_t r[32];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
                "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                  "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                  "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]),
                  "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
                  "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
                  "=r"(r[30]), "=r"(r[31])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (direct) {
                const int col0 = n0 + c;
#pragma unroll
                for (int j = 0; j < 32; j += 4) {
                    float v[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        v[q] = __uint_as_float(r[j + q]) + (bias ? bias[col0 + j + q] : 0.0f);
                    if (C) {
                        float4* pc = reinterpret_cast<float4*>(C + (size_t)row * ldc + col0 + j);
                        if (accumulate) {
                            const float4 o = *pc;
                            v[0] += o.x; v[1] += o.y; v[2] += o.z; v[3] += o.w;
                        }
                        *pc = make_float4(v[0], v[1], v[2], v[3]);
                    }
                    if (act) {
#pragma unroll
                        for (int q = 0; q < 4; ++q)
                            act[(size_t)row * ld_act + col0 + j + q] = __float2bfloat16_rn(gelu_tc(v[q]));
                    }
                }
            } else {
#pragma unroll
                for (int j = 0; j < 32; j += 4)
                    *reinterpret_cast<float4*>(out + c + j) =
                        make_float4(__uint_as_float(r[j]), __uint_as_float(r[j + 1]),
                                    __uint_as_float(r[j + 2]), __uint_as_float(r[j + 3]));
            }
        }
    } else if (tid == 0 && status) {
        atomicExch(status, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(BN));
}

}  // namespace tc

using tc::gelu_tc;

// Sum of the split partials in split order, then bias / accumulate / GELU.
__global__ void k_gemm_tc_reduce(const float* __restrict__ part, int splits, int M, int N,
                                 const float* __restrict__ bias, int accumulate,
                                 float* __restrict__ C, int ldc, __nv_bfloat16* __restrict__ act,
                                 int ld_act) {
    const long long total = (long long)M * N;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        float v = 0.0f;
        for (int s = 0; s < splits; ++s) v += part[(size_t)s * total + i];
        const int r = (int)(i / N), c = (int)(i - (long long)r * N);
        if (bias) v += bias[c];
        if (C) {
            float* pc = C + (size_t)r * ldc + c;
            *pc = accumulate ? *pc + v : v;
        }
        if (act) act[(size_t)r * ld_act + c] = __float2bfloat16_rn(gelu_tc(v));
    }
}

}  // namespace qssb

using namespace qssb;

extern "C" int qssb_gemm_tc_workspace_bytes(int32_t M, int32_t N, int32_t K, int32_t splits,
                                            size_t* bytes) {
    if (!bytes || M <= 0 || N <= 0 || K <= 0 || splits <= 0)
        return set_error(QSSB_ERR_INVALID, "qssb_gemm_tc_workspace_bytes: invalid sizes");
    *bytes = (splits > 1 ? sizeof(float) * (size_t)splits * M * N : 0) + 256;
    return QSSB_OK;
}

extern "C" int qssb_gemm_bf16_tc(const void* A, int32_t lda, int32_t trans_a, const void* B,
                                 int32_t ldb, int32_t trans_b, int32_t M, int32_t N, int32_t K,
                                 int32_t splits, const float* bias, int32_t accumulate, float* C,
                                 int32_t ldc, void* act_bf16, int32_t ld_act, void* workspace,
                                 size_t workspace_bytes, void* stream) {
    using namespace qssb::tc;
    if (!A || !B || !workspace || (!C && !act_bf16))
        return set_error(QSSB_ERR_INVALID, "qssb_gemm_bf16_tc: null operand, workspace or output");
    if (M <= 0 || N <= 0 || K <= 0 || M % BM || N % BN || splits <= 0 || K % (BK * splits))
        return set_error(QSSB_ERR_UNSUPPORTED,
                         "qssb_gemm_bf16_tc: M and N must be multiples of 128 and K of 64 x splits");
    const int cols_a = trans_a ? M : K, cols_b = trans_b ? K : N;
    if (lda < cols_a || ldb < cols_b || (lda % 8) || (ldb % 8) || (C && ldc < N) ||
        (act_bf16 && ld_act < N))
        return set_error(QSSB_ERR_INVALID, "qssb_gemm_bf16_tc: leading dimensions");
    if (((uintptr_t)A & 15u) || ((uintptr_t)B & 15u) || ((uintptr_t)workspace & 255u))
        return set_error(QSSB_ERR_INVALID, "qssb_gemm_bf16_tc: A, B 16-byte and workspace 256-byte aligned");
    if (splits == 1 && C && (((uintptr_t)C & 15u) || (ldc % 4)))
        return set_error(QSSB_ERR_INVALID,
                         "qssb_gemm_bf16_tc: without split K, C 16-byte aligned and ldc a multiple of 4");
    size_t need = 0;
    int rc = qssb_gemm_tc_workspace_bytes(M, N, K, splits, &need);
    if (rc) return rc;
    if (workspace_bytes < need)
        return set_error(QSSB_ERR_WORKSPACE, "qssb_gemm_bf16_tc: workspace too small");
    if ((long long)(M / BM) > 65535 || splits > 65535)
        return set_error(QSSB_ERR_UNSUPPORTED, "qssb_gemm_bf16_tc: grid too large");
    cudaStream_t s = (cudaStream_t)stream;
    float* part = static_cast<float*>(workspace);
    // the last 256 bytes: an int the kernel sets to 1 if an mbarrier wait ran out
    int* status = reinterpret_cast<int*>(static_cast<char*>(workspace) + need - 256);
    CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(int), s));
    const auto* a = static_cast<const __nv_bfloat16*>(A);
    const auto* b = static_cast<const __nv_bfloat16*>(B);
    const dim3 grid(N / BN, M / BM, splits);
    const int kps = K / splits;
    auto launch = [&](auto kern) -> int {
        CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
        { kern<<<grid, THREADS, SMEM_BYTES, s>>>(a, lda, b, ldb, M, N, kps, part, status, bias,
                                               accumulate, C, ldc,
                                               static_cast<__nv_bfloat16*>(act_bf16), ld_act); note_launch(); }
        CUDA_TRY(cudaGetLastError());
        return QSSB_OK;
    };
    if (trans_a) {
        rc = trans_b ? launch(k_gemm_tc<true, true>) : launch(k_gemm_tc<true, false>);
    } else {
        rc = trans_b ? launch(k_gemm_tc<false, true>) : launch(k_gemm_tc<false, false>);
    }
    if (rc) return rc;
    if (splits == 1) return QSSB_OK;  // the MMA kernel wrote C / act itself
    const long long total = (long long)M * N;
    long long blocks = (total + 255) / 256;
    const long long cap = 8LL * device_sm_count();
    if (blocks > cap) blocks = cap;
    { k_gemm_tc_reduce<<<(unsigned)blocks, 256, 0, s>>>(part, splits, M, N, bias, accumulate, C, ldc,
                                                     static_cast<__nv_bfloat16*>(act_bf16), ld_act); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}
