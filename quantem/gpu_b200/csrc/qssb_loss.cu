// qssb_loss.cu - SSB phase-variance loss for a batch of aberration candidates.
//
// L(theta) = mean_R[(1/B) sum_b phi_b^2 - ((1/B) sum_b phi_b)^2],
// phi_b = atan2(ifft2(C_b)) (docs/kernels/ssb.md:256-266 of the reference;
// engine.py:1464-1514 and 2120-2295). Unlike the object, this needs one
// inverse FFT per (candidate, BF pixel).
//
// k_loss_moments: grid (BF chunks, candidates), one CTA per SM (the N x N+1
// complex plane lives in shared memory). Per BF pixel the CTA
//   A) evaluates C_b on the +-q half set and mirrors it (C(-q) = -conj C(q),
//      see qssb_object.cu), DC := dc;
//   B) inverse-FFTs all rows, then all columns, in shared memory;
//   C) takes atan2 of its owned pixels and accumulates sum / sum of squares
//      in registers.
// Partial moment planes per chunk are folded in a fixed order in FP64
// (k_loss_reduce), and the per-pixel variance is averaged (k_loss_final):
// repeated calls give identical bits.
#include <limits.h>
#include <math.h>

#include "qssb_internal.h"

namespace qssb {

constexpr int kLossThreads = 512;
constexpr int kLossWarps = kLossThreads / 32;

template <int N>
struct LossSmem {
    static constexpr int P = N + 1;  // odd pitch: conflict-free column access
    static constexpr size_t bytes = sizeof(float2) * ((size_t)N * P + N);
};

// e^{-i Q(q)} for every scan frequency of every candidate (quadratic chi).
template <int N>
__global__ void k_eq_table(const qssb_aberrations_t* __restrict__ cands, qssb_calibration_t cal,
                           float2* __restrict__ eq) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    const int cand = blockIdx.y;
    if (idx >= N * N) return;
    const qssb_aberrations_t ab = cands[cand];
    const Probe p = make_probe_common(cal, ab.C10, ab.C12, ab.phi12, ab.C30);
    eq[(size_t)cand * N * N + idx] = eq_value(idx / N, idx % N, p);
}

template <int N, bool SYM, bool CHI64, bool QUAD>
__global__ void __launch_bounds__(kLossThreads, 1) k_loss_moments(
    const float2* __restrict__ g, int n_bf, const float* __restrict__ geom,
    const float* __restrict__ q_row, const float* __restrict__ q_col,
    const qssb_aberrations_t* __restrict__ cands, qssb_calibration_t cal,
    const float2* __restrict__ eq_table, int bf_per_chunk, int n_chunks, float* __restrict__ part) {
    constexpr int H = N / 2 + 1;
    constexpr int P = LossSmem<N>::P;
    constexpr int CPW = N / kLossWarps;  // columns owned per warp
    constexpr int RPL = N / 32;          // rows owned per lane
    constexpr int NEVAL = SYM ? (N / 2 + 1) * N + (N / 2 - 1) : N * N;
    extern __shared__ float2 smem[];
    __shared__ Probe sp;
    float2* plane = smem;
    float2* tw = smem + N * P;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int chunk = blockIdx.x;
    const int cand = blockIdx.y;
    if (tid == 0) {
        const qssb_aberrations_t ab = cands[cand];
        sp = make_probe_common(cal, ab.C10, ab.C12, ab.phi12, ab.C30);
    }
    fill_twiddles<N>(tw, tid, kLossThreads);
    __syncthreads();
    const Probe& p = sp;
    const float2* eqc = eq_table + (size_t)cand * N * N;
    float as[CPW][RPL], aq[CPW][RPL];
#pragma unroll
    for (int i = 0; i < CPW; ++i)
#pragma unroll
        for (int t = 0; t < RPL; ++t) as[i][t] = aq[i][t] = 0.0f;
    const int b0 = chunk * bf_per_chunk;
    int nb = n_bf - b0;
    if (nb > bf_per_chunk) nb = bf_per_chunk;
    const float2 dc = make_float2((float)cal.dc_re, (float)cal.dc_im);
    for (int i = 0; i < nb; ++i) {
        const int b = b0 + i;
        const BFQuad kq = bf_quad(geom, n_bf, b, p);
        float2 pk = make_float2(0.0f, 0.0f);
        if constexpr (!QUAD)
            pk = probe_at_bf<CHI64>(__ldg(geom + 2 * n_bf + b), __ldg(geom + 3 * n_bf + b),
                                    __ldg(geom + 4 * n_bf + b), __ldg(geom + 5 * n_bf + b), p);
        const float2* gb = g + (size_t)b * N * H;
        // A) corrected spectrum into shared memory
        for (int e = tid; e < NEVAL; e += kLossThreads) {
            int r, c;
            bool mirror = false;
            if (!SYM || e < (N / 2 + 1) * N) {
                r = e / N;
                c = e - r * N;
                mirror = SYM && r >= 1 && r < N / 2 && c != N / 2;
            } else {
                r = N / 2 + 1 + (e - (N / 2 + 1) * N);
                c = N / 2;
            }
            float2 gv;
            if (c <= N / 2) {
                gv = __ldg(gb + r * H + c);
            } else {
                gv = cconj(__ldg(gb + ((N - r) & (N - 1)) * H + (N - c)));
            }
            float2 v;
            if constexpr (QUAD) {
                v = corrected_quad<CHI64>(__ldg(q_row + r), __ldg(q_col + c), r, c,
                                          __ldg(eqc + r * N + c), kq, gv, p);
            } else {
                v = corrected<CHI64>(__ldg(q_row + r), __ldg(q_col + c), r, c, kq.kx, kq.ky, kq.kx_lo,
                                     kq.ky_lo, pk, gv, p);
            }
            if (r == 0 && c == 0) v = dc;
            plane[r * P + c] = v;
            if (mirror) plane[(N - r) * P + ((N - c) & (N - 1))] = cneg_conj(v);
        }
        __syncthreads();
        // B) rows, then columns (inverse, unnormalised: atan2 is scale-free)
        for (int row = warp; row < N; row += kLossWarps) line_fft<N, +1>(plane + row * P, 1, tw, lane);
        __syncthreads();
#pragma unroll
        for (int ci = 0; ci < CPW; ++ci) {
            const int col = warp + ci * kLossWarps;
            line_fft<N, +1>(plane + col, P, tw, lane);
            // C) phase moments of the owned pixels
#pragma unroll
            for (int t = 0; t < RPL; ++t) {
                const float2 v = plane[(lane + 32 * t) * P + col];
                const float ph = phase_atan2(v.y, v.x);
                as[ci][t] += ph;
                aq[ci][t] = fmaf(ph, ph, aq[ci][t]);
            }
        }
        __syncthreads();
    }
    // column-major partial planes: part[((cand * n_chunks + chunk) * 2 + m) * N * N + col * N + row]
    float* ps = part + ((size_t)(cand * n_chunks + chunk) * 2) * N * N;
    float* pq = ps + (size_t)N * N;
#pragma unroll
    for (int ci = 0; ci < CPW; ++ci) {
        const int col = warp + ci * kLossWarps;
#pragma unroll
        for (int t = 0; t < RPL; ++t) {
            ps[col * N + lane + 32 * t] = as[ci][t];
            pq[col * N + lane + 32 * t] = aq[ci][t];
        }
    }
}

// ------------------------------------------------------------ N = 128 path
// One CTA (16 warps = 64 groups of 8 lanes) per (BF chunk, candidate). Per BF:
//  A) C_b on rows 0..64 (all columns) into Hp, C_b(-r, 64) for r = 1..63;
//     then delta_r = conj(C(r,64)) + C(-r,64), the Nyquist-column deviation
//     from C(-q) = -conj(C(q));
//  B) row IFFTs of rows 0..64 only: after them row -r is
//     -conj(row r) + delta_r (-1)^x, so the lower half is never stored;
//  C) column IFFTs of all 128 columns, reading rows 65..127 through that
//     relation; atan2 of each output, sum in registers, sum of squares in
//     shared memory (each pixel owned by one lane for the whole launch).
// Row/column -> group maps keep the two groups of a half-warp 8 apart mod 16
// in bank space (conflict-free 8-byte accesses) and the four groups of a
// warp 8 apart mod 32 (conflict-free 4-byte accesses to the squares).
constexpr int kL128P = 129;  // Hp and squares pitch
struct Loss128Smem {
    static constexpr size_t hp = sizeof(float2) * 65 * kL128P;
    static constexpr size_t t = sizeof(float2) * 64 * kG8Scratch;
    static constexpr size_t sq = sizeof(float) * 128 * kL128P;
    static constexpr size_t misc = sizeof(float2) * (128 + 64 + 64);  // tw, cneg, delta
    static constexpr size_t bytes = hp + t + sq + misc;
};

template <bool CHI64, bool QUAD>
__global__ void __launch_bounds__(512, 1) k_loss_moments128(
    const float2* __restrict__ g, int n_bf, const float* __restrict__ geom,
    const float* __restrict__ q_row, const float* __restrict__ q_col,
    const qssb_aberrations_t* __restrict__ cands, qssb_calibration_t cal,
    const float2* __restrict__ eq_table, int bf_per_chunk, int n_chunks, float* __restrict__ part) {
    constexpr int N = 128;
    constexpr int H = N / 2 + 1;
    extern __shared__ float4 smem4[];
    char* base = reinterpret_cast<char*>(smem4);
    float2* Hp = reinterpret_cast<float2*>(base);
    float2* T = reinterpret_cast<float2*>(base + Loss128Smem::hp);
    float* sq = reinterpret_cast<float*>(base + Loss128Smem::hp + Loss128Smem::t);
    float2* tw = reinterpret_cast<float2*>(base + Loss128Smem::hp + Loss128Smem::t + Loss128Smem::sq);
    float2* cneg = tw + 128;
    float2* delta = cneg + 64;
    __shared__ Probe sp;
    // FP32-chi path: theta = 2 (q_row u + q_col v) is separable, so
    // e^{i theta} = s_phr[r] * s_phc[c] from 256 sincos per BF pixel
    constexpr bool kSep = QUAD && !CHI64;
    __shared__ float2 s_phr[kSep ? 128 : 1];
    __shared__ float2 s_phc[kSep ? 128 : 1];
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int grp = lane >> 3;
    const int s = lane & 7;
    float2* Tg = T + (warp * 4 + grp) * kG8Scratch;
    const int chunk = blockIdx.x;
    const int cand = blockIdx.y;
    if (tid == 0) {
        const qssb_aberrations_t ab = cands[cand];
        sp = make_probe_common(cal, ab.C10, ab.C12, ab.phi12, ab.C30);
    }
    fill_twiddles<N>(tw, tid, 512);
    for (int i = tid; i < 128 * kL128P; i += 512) sq[i] = 0.0f;
    __syncthreads();
    const Probe& p = sp;
    const float2* eqc = eq_table + (size_t)cand * N * N;
    // e^{i 2 q_row(r) u}, e^{i 2 q_col(c) v} of BF pixel b, (u, v) = M k
    auto fill_phase = [&](int b) {
        if (tid < 256) {
            const float kx = __ldg(geom + b);
            const float ky = __ldg(geom + n_bf + b);
            float sn, cs;
            if (tid < 128) {
                sincosf(2.0f * __ldg(q_row + tid) * fmaf(p.mxx, kx, p.mxy * ky), &sn, &cs);
                s_phr[tid] = make_float2(cs, sn);
            } else {
                sincosf(2.0f * __ldg(q_col + tid - 128) * fmaf(p.mxy, kx, p.myy * ky), &sn, &cs);
                s_phc[tid - 128] = make_float2(cs, sn);
            }
        }
    };
    // the line (row or column) of this group within a round of 64
    const int line = (warp & 7) + 8 * grp + 32 * (warp >> 3);
    float acc[2][16];
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int t = 0; t < 16; ++t) acc[r][t] = 0.0f;
    const int b0 = chunk * bf_per_chunk;
    int nb = n_bf - b0;
    if (nb > bf_per_chunk) nb = bf_per_chunk;
    const float2 dc = make_float2((float)cal.dc_re, (float)cal.dc_im);
    if constexpr (kSep) {
        if (nb > 0) fill_phase(b0);
        __syncthreads();
    }
    for (int i = 0; i < nb; ++i) {
        const int b = b0 + i;
        const BFQuad kq = bf_quad(geom, n_bf, b, p);
        float2 pk = make_float2(0.0f, 0.0f);
        if constexpr (!QUAD)
            pk = probe_at_bf<CHI64>(__ldg(geom + 2 * n_bf + b), __ldg(geom + 3 * n_bf + b),
                                    __ldg(geom + 4 * n_bf + b), __ldg(geom + 5 * n_bf + b), p);
        const float2* gb = g + (size_t)b * N * H;
        // A) rows 0..64 and the lower Nyquist column; the G (and e^{iQ})
        // values of a thread's next element are loaded one element ahead
        constexpr int kNA = 65 * N + 63;
        auto elem_rc = [](int e, int& r, int& c) {
            if (e < 65 * N) {
                r = e >> 7;
                c = e & 127;
            } else {
                r = N - 1 - (e - 65 * N);  // 127 .. 65
                c = 64;
            }
        };
        auto g_at = [&](int r, int c) {
            return c <= 64 ? __ldg(gb + r * H + c)
                           : cconj(__ldg(gb + ((N - r) & (N - 1)) * H + (N - c)));
        };
        float2 g_nx = make_float2(0.f, 0.f), eq_nx = make_float2(1.f, 0.f);
        if (tid < kNA) {
            int r, c;
            elem_rc(tid, r, c);
            g_nx = g_at(r, c);
            if constexpr (QUAD) eq_nx = __ldg(eqc + r * N + c);
        }
        for (int e = tid; e < kNA; e += 512) {
            int r, c;
            elem_rc(e, r, c);
            const float2 gv = g_nx;
            const float2 eqv = eq_nx;
            if (e + 512 < kNA) {
                int rn, cn;
                elem_rc(e + 512, rn, cn);
                g_nx = g_at(rn, cn);
                if constexpr (QUAD) eq_nx = __ldg(eqc + rn * N + cn);
            }
            float2 v;
            if constexpr (kSep) {
                const float2 lo = make_float2(kq.kx_lo, kq.ky_lo);
                v = corrected_quad_e(__ldg(q_row + r), __ldg(q_col + c), r, c, eqv, kq.kx, kq.ky,
                                     kq.ak, &lo, cmul(s_phr[r], s_phc[c]), gv, p);
            } else if constexpr (QUAD) {
                v = corrected_quad<CHI64>(__ldg(q_row + r), __ldg(q_col + c), r, c, eqv, kq, gv, p);
            } else {
                v = corrected<CHI64>(__ldg(q_row + r), __ldg(q_col + c), r, c, kq.kx, kq.ky,
                                     kq.kx_lo, kq.ky_lo, pk, gv, p);
            }
            if (e < 65 * N) {
                Hp[r * kL128P + c] = (r == 0 && c == 0) ? dc : v;
            } else {
                cneg[N - r] = v;  // C(-r', 64), r' = N - r in 1..63
            }
        }
        __syncthreads();
        if (tid >= 1 && tid < 64) delta[tid] = cadd(cconj(Hp[tid * kL128P + 64]), cneg[tid]);
        // every thread is past A: the next BF pixel's phase rows can be written
        if constexpr (kSep) {
            if (i + 1 < nb) fill_phase(b + 1);
        }
        __syncthreads();
        // B) row IFFTs of rows 0..63, then row 64
        {
            float2 v[16];
            float2* rowp = Hp + line * kL128P;
#pragma unroll
            for (int n1 = 0; n1 < 16; ++n1) v[n1] = rowp[s + 8 * n1];
            fft128_g8<+1>(v, Tg, s, tw);
#pragma unroll
            for (int t = 0; t < 16; ++t) rowp[fft128_g8_index(s, t)] = v[t];
            if (warp == 0) {
                float2* r64 = Hp + 64 * kL128P;
#pragma unroll
                for (int n1 = 0; n1 < 16; ++n1) v[n1] = lane < 8 ? r64[s + 8 * n1] : make_float2(0.f, 0.f);
                fft128_g8<+1>(v, Tg, s, tw);
                if (lane < 8) {
#pragma unroll
                    for (int t = 0; t < 16; ++t) r64[fft128_g8_index(s, t)] = v[t];
                }
            }
        }
        __syncthreads();
        // C) column IFFTs, two rounds of 64 columns
#pragma unroll
        for (int round = 0; round < 2; ++round) {
            const int x = line + 64 * round;
            const float sign = (x & 1) ? -1.0f : 1.0f;
            float2 v[16];
#pragma unroll
            for (int n1 = 0; n1 < 16; ++n1) {
                const int r = s + 8 * n1;
                if (r <= 64) {
                    v[n1] = Hp[r * kL128P + x];
                } else {
                    const float2 m = Hp[(N - r) * kL128P + x];
                    const float2 d = delta[N - r];
                    v[n1] = make_float2(fmaf(sign, d.x, -m.x), fmaf(sign, d.y, m.y));
                }
            }
            fft128_g8<+1>(v, Tg, s, tw);
#pragma unroll
            for (int t = 0; t < 16; ++t) {
                const int y = fft128_g8_index(s, t);
                const float ph = phase_atan2(v[t].y, v[t].x);
                acc[round][t] += ph;
                float* q2 = sq + y * kL128P + x;
                *q2 = fmaf(ph, ph, *q2);
            }
        }
        __syncthreads();
    }
    // row-major partial planes: part[((cand * n_chunks + chunk) * 2 + m) * N * N + y * N + x]
    float* ps = part + ((size_t)(cand * n_chunks + chunk) * 2) * N * N;
    float* pq = ps + (size_t)N * N;
#pragma unroll
    for (int round = 0; round < 2; ++round) {
        const int x = line + 64 * round;
#pragma unroll
        for (int t = 0; t < 16; ++t) ps[fft128_g8_index(s, t) * N + x] = acc[round][t];
    }
    for (int i = tid; i < N * N; i += 512) pq[i] = sq[(i >> 7) * kL128P + (i & 127)];
}

// Per pixel: fold the partial planes in FP64, write the mean phase, and sum
// the variance over this block's 32 pixels: block_var[cand][blockIdx.x]. The
// eight warps of a block take every 8th partial plane of the same 32 pixels
// (four planes' loads in flight before their in-order adds), then warp 0
// adds the eight slices in order - a fixed order for a given plan. N^2 is a
// multiple of 32 for every size.
constexpr int kReducePix = 32;
constexpr int kReduceSlices = 8;

template <int N>
__global__ void __launch_bounds__(kReducePix * kReduceSlices) k_loss_reduce(
    const float* __restrict__ part, int n_chunks, int n_bf, double* __restrict__ block_var,
    float* __restrict__ mean_phase, int row_major) {
    __shared__ double r1[kReduceSlices][kReducePix];
    __shared__ double r2[kReduceSlices][kReducePix];
    __shared__ double rv[kReducePix];
    const int px = threadIdx.x & (kReducePix - 1);
    const int sl = threadIdx.x / kReducePix;
    const int j = blockIdx.x * kReducePix + px;  // col * N + row, or row * N + col
    const int cand = blockIdx.y;
    constexpr size_t NN = (size_t)N * N;
    const float* cbase = part + (size_t)cand * n_chunks * 2 * NN + j;
    double s1 = 0.0, s2 = 0.0;
    int k = sl;
    for (; k + 3 * kReduceSlices < n_chunks; k += 4 * kReduceSlices) {
        float a[4], b[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const float* base = cbase + (size_t)(k + u * kReduceSlices) * 2 * NN;
            a[u] = __ldg(base);
            b[u] = __ldg(base + NN);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            s1 += (double)a[u];
            s2 += (double)b[u];
        }
    }
    for (; k < n_chunks; k += kReduceSlices) {
        const float* base = cbase + (size_t)k * 2 * NN;
        s1 += (double)__ldg(base);
        s2 += (double)__ldg(base + NN);
    }
    r1[sl][px] = s1;
    r2[sl][px] = s2;
    __syncthreads();
    if (sl == 0) {
        double t1 = 0.0, t2 = 0.0;
#pragma unroll
        for (int w = 0; w < kReduceSlices; ++w) {
            t1 += r1[w][px];
            t2 += r2[w][px];
        }
        const double inv_b = 1.0 / (double)n_bf;
        const double mean = t1 * inv_b;
        rv[px] = t2 * inv_b - mean * mean;
        if (mean_phase) {
            const int hi = j / N;
            const int lo = j - hi * N;
            mean_phase[(size_t)cand * NN + (row_major ? j : lo * N + hi)] = (float)mean;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double acc = 0.0;
#pragma unroll
        for (int i = 0; i < kReducePix; ++i) acc += rv[i];
        block_var[(size_t)cand * (NN / kReducePix) + blockIdx.x] = acc;
    }
}

// L = (sum of the block sums, fixed order) / N^2; NaN when status (the
// persistent loss's abort word, or null) is set.
__global__ void __launch_bounds__(256) k_loss_final(const double* __restrict__ block_var,
                                                    int n_blocks, int npos,
                                                    float* __restrict__ losses,
                                                    const int* __restrict__ status = nullptr) {
    __shared__ double red[256];
    const int cand = blockIdx.x;
    const double* v = block_var + (size_t)cand * n_blocks;
    double acc = 0.0;
    for (int i = threadIdx.x; i < n_blocks; i += 256) acc += v[i];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        losses[cand] = (status && *status != 0) ? __int_as_float(0x7fc00000)
                                                : (float)(red[0] / (double)npos);
}

// ---------------------------------------- N = 128 with the overlap table
// The registered cancel flag (qssb_set_cancel): a device int the table
// kernel polls once per BF pixel pair; nonzero stops every CTA at its next
// pair and makes the losses NaN.
static const int* g_cancel_flag = nullptr;
static const int* cancel_flag() { return g_cancel_flag; }
constexpr int kFusedFoldChunks = 32;

// For quadratic chi the overlap factorises (corrected_quad in
// qssb_device.cuh): C_b(q) = G_b(q) e^{-i theta} (d cos Q + i s sin Q) / |.|,
// where theta = 2 q^T M k_b and Q(q) depend on the candidate but the
// aperture pair (A(q - k_b), A(q + k_b)) does not. k_overlap_table128
// evaluates the pair once per dataset on the evaluated half set (rows
// 0..64 x 128 columns, then (127 - j, 64), j < 63), with the kernels'
// aperture arithmetic and FP64 tie rule, so a candidate costs a table read,
// a separable phase product and one reciprocal square root per element.
constexpr int kNE128 = 65 * 128 + 63;

__device__ __forceinline__ void elem_rc128(int e, int& r, int& c) {
    if (e < 65 * 128) {
        r = e >> 7;
        c = e & 127;
    } else {
        r = 127 - (e - 65 * 128);  // 127 .. 65
        c = 64;
    }
}

// (A(q - k_b), A(q + k_b)) at scan frequency (r, c) for BF pixel b: the fast
// float32 aperture, recomputed in FP64 where the pair ties in the soft edge
// (corrected_quad_e's rule and arithmetic).
__device__ __forceinline__ float2 aperture_pair(const float* __restrict__ geom, int n_bf, int b,
                                                const float* __restrict__ q_row,
                                                const float* __restrict__ q_col, int r, int c,
                                                const Probe& p) {
    const float kx = __ldg(geom + b);
    const float ky = __ldg(geom + n_bf + b);
    const float qx = __ldg(q_row + r);
    const float qy = __ldg(q_col + c);
    const float dxm = qx - kx, dym = qy - ky;
    const float dxp = qx + kx, dyp = qy + ky;
    const float r2m = fmaf(dxm, dxm, dym * dym);
    const float r2p = fmaf(dxp, dxp, dyp * dyp);
    float am = soft_aperture_fast(dxm, dym, r2m, p);
    float ap = soft_aperture_fast(dxp, dyp, r2p, p);
    if (fabsf(am - ap) < kApertureTie && (in_edge_band(r2m, p) || in_edge_band(r2p, p))) {
        const double qx64 = fftfreq_d(r, p.n_r, p.qval_r);
        const double qy64 = fftfreq_d(c, p.n_c, p.qval_c);
        const double kx64 = (double)kx + (double)__ldg(geom + 6 * n_bf + b);
        const double ky64 = (double)ky + (double)__ldg(geom + 7 * n_bf + b);
        am = soft_aperture_fp64(qx64 - kx64, qy64 - ky64, p.semi_d, p.lam_d, p.ang_r_d, p.ang_c_d);
        ap = soft_aperture_fp64(qx64 + kx64, qy64 + ky64, p.semi_d, p.lam_d, p.ang_r_d, p.ang_c_d);
    }
    return make_float2(am, ap);
}

__global__ void __launch_bounds__(256) k_overlap_table128(
    const float* __restrict__ geom, int n_bf, const float* __restrict__ q_row,
    const float* __restrict__ q_col, Probe p, float2* __restrict__ table) {
    const int e = blockIdx.x * 256 + threadIdx.x;
    const int b = blockIdx.y;
    if (e >= kNE128 || b >= n_bf) return;
    int r, c;
    elem_rc128(e, r, c);
    table[(size_t)b * kNE128 + e] = aperture_pair(geom, n_bf, b, q_row, q_col, r, c, p);
}

// The two-pass (256^2 .. 1024^2) table: per BF pixel the frequencies the row
// pass evaluates - rows 0 .. N/2 over all N columns, row-major - then the
// partners (N - r, N/2) of its Nyquist-column relation at index
// (N/2 + 1) N + r, r = 1 .. N/2 - 1 (index r = 0 unused).
template <int N>
__host__ __device__ constexpr size_t two_pass_table_elems() {
    return (size_t)(N / 2 + 1) * N + N / 2;
}

template <int N>
__global__ void __launch_bounds__(256) k_overlap_table_rows(
    const float* __restrict__ geom, int n_bf, const float* __restrict__ q_row,
    const float* __restrict__ q_col, Probe p, float2* __restrict__ table) {
    constexpr int kMain = (N / 2 + 1) * N;
    const int e = blockIdx.x * 256 + threadIdx.x;
    const int b = blockIdx.y;
    if (e >= (int)two_pass_table_elems<N>() || b >= n_bf) return;
    float2 v = make_float2(0.0f, 0.0f);
    if (e < kMain) {
        v = aperture_pair(geom, n_bf, b, q_row, q_col, e / N, e % N, p);
    } else if (e > kMain) {
        v = aperture_pair(geom, n_bf, b, q_row, q_col, N - (e - kMain), N / 2, p);
    }
    table[(size_t)b * two_pass_table_elems<N>() + e] = v;
}

// C = G conj(Gamma_hat) from the table entry a = (A(q - k), A(q + k)),
// e^{-i Q} = eq, e^{i theta} = e and A(k) = ak: corrected_quad_e's arithmetic.
__device__ __forceinline__ float2 corrected_table(float2 a, float2 eq, float2 e, float ak, float2 g) {
    // packed (re, im) pairs; lane by lane the scalar operations of
    // corrected_quad_e, so the bits are the same
    const float2 d = __fmul2_rn(__fadd2_rn(make_float2(a.x, a.x), make_float2(-a.y, a.y)),
                                make_float2(eq.x, -eq.y));  // (dr, di)
    float2 gg = cscale(cmul(e, d), ak);
    const float m2 = fmaf(gg.x, gg.x, gg.y * gg.y);
    const float inv = m2 > 1e-16f ? rsqrtf(m2) : 1e8f;
    gg = cscale(gg, inv);
    const float2 t = __fmul2_rn(make_float2(g.y, -g.x), make_float2(gg.y, gg.y));
    return __ffma2_rn(g, make_float2(gg.x, gg.x), t);
}

// The same from the table without the quadratic factorisation (C30 != 0):
// with m = A(k) A(q-k) and l = A(k) A(q+k),
//   Gamma = m e^{-i chi(q-k)} e^{i chi(k)} - l e^{i chi(q+k)} e^{-i chi(k)}
// (corrected with the apertures from the table); ek = e^{i chi(k)}.
template <bool CHI64>
__device__ __forceinline__ float2 corrected_table_direct(float2 a, float qx, float qy, float kx,
                                                         float ky, float ak, float2 ek, float2 g,
                                                         const Probe& p) {
    const float m = ak * a.x;
    const float l = ak * a.y;
    const Disp dm = displacement(qx - kx, qy - ky, p);
    const Disp dp = displacement(qx + kx, qy + ky, p);
    float sm, cm, sp, cp;
    __sincosf(chi_value<CHI64>(dm.alpha2, dm.cos2, dm.sin2, p), &sm, &cm);
    __sincosf(chi_value<CHI64>(dp.alpha2, dp.cos2, dp.sin2, p), &sp, &cp);
    // t1 = m (cm - i sm)(ck + i sk), t2 = l (cp + i sp)(ck - i sk)
    const float t1r = m * fmaf(cm, ek.x, sm * ek.y);
    const float t1i = m * fmaf(cm, ek.y, -sm * ek.x);
    const float t2r = l * fmaf(cp, ek.x, sp * ek.y);
    const float t2i = l * fmaf(sp, ek.x, -cp * ek.y);
    float gr = t1r - t2r;
    float gi = t1i - t2i;
    const float m2 = fmaf(gr, gr, gi * gi);
    const float inv = m2 > 1e-16f ? rsqrtf(m2) : 1e8f;
    gr *= inv;
    gi *= inv;
    return make_float2(fmaf(g.x, gr, g.y * gi), fmaf(g.y, gr, -g.x * gi));
}

// Two BF pixels per inverse 2D FFT. Split each corrected spectrum into its
// anti-Hermitian part A (C(-q) = -conj C(q): every scan frequency off the
// Nyquist row and column, where the evaluated half set defines the other
// half) and its Hermitian part E (DC and the two Nyquist lines). Then
// IFFT2(A) = i a and IFFT2(E) = e with a, e real, so O_b = e_b + i a_b and
// phi_b = atan2(a_b, e_b). The two pixels' A share one complex transform,
//   S = A_2 - i A_1,  IFFT2(S) = a_1 + i a_2,
// and E_b, nonzero on two lines only, gives
//   e_b(y, x) = Re dc + (-1)^y E^row_b(x) + (-1)^x E^col_b(y)
// from two 128-point transforms (one complex line per pixel: E^row + i E^col).
// Per pixel pair: 2 x 8383 table evaluations, 128 row and 128 column FFTs
// (the one-pixel kernel: 65 + 128 per pixel) and no shared-memory moments:
// phi^2 is summed per thread in FP64 (the loss needs only its total, since
// mean_R (1/B) sum_b phi_b^2 = (1/(N^2 B)) sum_{R,b} phi_b^2), phi per pixel
// in registers as before.
struct Pair128Smem {
    static constexpr size_t s = sizeof(float2) * 128 * kL128P;    // packed plane S
    static constexpr size_t t = sizeof(float2) * 64 * kG8Scratch;  // group transposes
    static constexpr size_t tw = sizeof(float2) * 128;
    static constexpr size_t ph = sizeof(float2) * 2 * 256;    // [bf][e^{2i q_r u} | e^{2i q_c v}]
    static constexpr size_t ny = sizeof(float2) * 2 * 256;    // [bf][row 64 | column 64]: C
    static constexpr size_t eb = sizeof(float2) * 2 * 256;    // [bf][E row | E col]
    static constexpr size_t na = sizeof(float2) * 2 * 256;    // [bf][row 64 | column 64]: A
    static constexpr size_t el = sizeof(float) * 2 * 256;     // [bf][E^row(x) | E^col(y)]
    static constexpr size_t bytes = s + t + tw + ph + ny + eb + na + el;
};

template <bool CHI64, bool QUAD>
__global__ void __launch_bounds__(512, 1) k_loss_pair128(
    const float2* __restrict__ g, int n_bf, const float* __restrict__ geom,
    const float* __restrict__ q_row, const float* __restrict__ q_col,
    const float2* __restrict__ overlap, const qssb_aberrations_t* __restrict__ cands,
    qssb_calibration_t cal, const float2* __restrict__ eq_table, int bf_per_chunk, int n_chunks,
    float* __restrict__ part, double* __restrict__ part_sq, const int* __restrict__ cancel,
    unsigned int* __restrict__ arrivals, float* __restrict__ losses, float* __restrict__ mean_phase) {
    constexpr int N = 128;
    constexpr int H = N / 2 + 1;
    constexpr int P = kL128P;
    extern __shared__ float4 smem4[];
    char* base = reinterpret_cast<char*>(smem4);
    float2* S = reinterpret_cast<float2*>(base);
    float2* T = reinterpret_cast<float2*>(base + Pair128Smem::s);
    float2* tw = reinterpret_cast<float2*>(base + Pair128Smem::s + Pair128Smem::t);
    float2* ph = tw + 128;
    float2* ny = ph + 512;
    float2* eb = ny + 512;
    float2* na = eb + 512;
    float* el = reinterpret_cast<float*>(na + 512);
    __shared__ Probe sp;
    __shared__ double s_red[16];
    __shared__ int s_stop, s_last;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int grp = lane >> 3;
    const int s = lane & 7;
    float2* Tg = T + (warp * 4 + grp) * kG8Scratch;
    const int chunk = blockIdx.x;
    const int cand = blockIdx.y;
    if (tid == 0) {
        const qssb_aberrations_t ab = cands[cand];
        sp = make_probe_common(cal, ab.C10, ab.C12, ab.phi12, ab.C30);
        s_stop = 0;
    }
    fill_twiddles<N>(tw, tid, 512);
    __syncthreads();
    const Probe& p = sp;
    const float2* eqc = eq_table + (size_t)cand * N * N;
    // the line (row or column) of this group within a round of 64
    const int line = (warp & 7) + 8 * grp + 32 * (warp >> 3);
    float acc[2][16];
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int t = 0; t < 16; ++t) acc[r][t] = 0.0f;
    double sq = 0.0;
    const int b0 = chunk * bf_per_chunk;
    int nb = n_bf - b0;
    if (nb > bf_per_chunk) nb = bf_per_chunk;
    const float2 dc = make_float2((float)cal.dc_re, (float)cal.dc_im);
    // e^{i 2 q_row(r) u_b}, e^{i 2 q_col(c) v_b} of the pair starting at pixel
    // i of the chunk, (u, v) = M k; written during the previous pair's row pass
    auto fill_phase = [&](int i) {
        const int b1 = b0 + i;
        const int b2 = i + 1 < nb ? b1 + 1 : b1;
        {
            const int bf = tid >> 8;
            const int j = tid & 255;
            const int b = bf ? b2 : b1;
            const float kx = __ldg(geom + b);
            const float ky = __ldg(geom + n_bf + b);
            float sn, cs;
            if constexpr (!QUAD) {
                // e^{i chi(k_b)} (the reference's pk without A(k), which the table holds)
                if (j == 0) {
                    __sincosf(chi_value<CHI64>(__ldg(geom + 2 * n_bf + b), __ldg(geom + 3 * n_bf + b),
                                               __ldg(geom + 4 * n_bf + b), p), &sn, &cs);
                    ph[bf * 256] = make_float2(cs, sn);
                }
                return;
            } else if constexpr (CHI64) {
                const double kx64 = (double)kx + (double)__ldg(geom + 6 * n_bf + b);
                const double ky64 = (double)ky + (double)__ldg(geom + 7 * n_bf + b);
                const double u = j < 128 ? fma(p.mxx_d, kx64, p.mxy_d * ky64)
                                         : fma(p.mxy_d, kx64, p.myy_d * ky64);
                const double q = j < 128 ? fftfreq_d(j, N, p.qval_r) : fftfreq_d(j - 128, N, p.qval_c);
                sincosf(reduce_angle(2.0 * q * u), &sn, &cs);
            } else {
                const float u = j < 128 ? fmaf(p.mxx, kx, p.mxy * ky) : fmaf(p.mxy, kx, p.myy * ky);
                const float q = j < 128 ? __ldg(q_row + j) : __ldg(q_col + j - 128);
                sincosf(2.0f * q * u, &sn, &cs);
            }
            ph[tid] = make_float2(cs, sn);
        }
    };
    if (nb > 0) fill_phase(0);
    __syncthreads();
    for (int i = 0; i < nb; i += 2) {
        const bool two = i + 1 < nb;
        const int b1 = b0 + i;
        const int b2 = two ? b1 + 1 : b1;
        // A) both pixels' corrected spectra on the evaluated set, packed into S
        {
            const float2* g1 = g + (size_t)b1 * N * H;
            const float2* g2 = g + (size_t)b2 * N * H;
            const float2* t1 = overlap + (size_t)b1 * kNE128;
            const float2* t2 = overlap + (size_t)b2 * kNE128;
            // the next element's five loads are issued before this one's math
            auto gofs = [](int r, int c) {
                return c <= 64 ? r * H + c : ((N - r) & (N - 1)) * H + (N - c);
            };
            float2 ng1, ng2, nt1, nt2, neq = make_float2(1.0f, 0.0f);
            {
                int r, c;
                elem_rc128(tid, r, c);  // tid < 512 < kNE128
                const int go = gofs(r, c);
                ng1 = __ldg(g1 + go);
                ng2 = __ldg(g2 + go);
                nt1 = __ldg(t1 + tid);
                nt2 = __ldg(t2 + tid);
                if constexpr (QUAD) neq = __ldg(eqc + r * N + c);
            }
            const float ak1 = __ldg(geom + 5 * n_bf + b1);
            const float ak2 = __ldg(geom + 5 * n_bf + b2);
            float k1x = 0.f, k1y = 0.f, k2x = 0.f, k2y = 0.f;
            if constexpr (!QUAD) {
                k1x = __ldg(geom + b1);
                k1y = __ldg(geom + n_bf + b1);
                k2x = __ldg(geom + b2);
                k2y = __ldg(geom + n_bf + b2);
            }
            for (int e = tid; e < kNE128; e += 512) {
                int r, c;
                elem_rc128(e, r, c);
                float2 gv1 = ng1, gv2 = ng2;
                const float2 d1 = nt1, d2 = nt2, eqv = neq;
                if (e + 512 < kNE128) {
                    int rn, cn;
                    elem_rc128(e + 512, rn, cn);
                    const int go = gofs(rn, cn);
                    ng1 = __ldg(g1 + go);
                    ng2 = __ldg(g2 + go);
                    nt1 = __ldg(t1 + e + 512);
                    nt2 = __ldg(t2 + e + 512);
                    if constexpr (QUAD) neq = __ldg(eqc + rn * N + cn);
                }
                if (c > 64) {
                    gv1.y = -gv1.y;
                    gv2.y = -gv2.y;
                }
                float2 v1, v2;
                if constexpr (QUAD) {
                    v1 = corrected_table(d1, eqv, cmul(ph[r], ph[128 + c]), ak1, gv1);
                    v2 = corrected_table(d2, eqv, cmul(ph[256 + r], ph[384 + c]), ak2, gv2);
                } else {
                    const float qx = __ldg(q_row + r);
                    const float qy = __ldg(q_col + c);
                    v1 = corrected_table_direct<CHI64>(d1, qx, qy, k1x, k1y, ak1, ph[0], gv1, p);
                    v2 = corrected_table_direct<CHI64>(d2, qx, qy, k2x, k2y, ak2, ph[256], gv2, p);
                }
                if (!two) v2 = make_float2(0.0f, 0.0f);
                if (r == 64 || c == 64) {
                    if (r == 64) {
                        ny[c] = v1;
                        ny[256 + c] = v2;
                    }
                    if (c == 64) {
                        ny[128 + r] = v1;
                        ny[384 + r] = v2;
                    }
                } else if (r == 0 && c == 0) {
                    // DC := dc; its anti-Hermitian part is i Im(dc)
                    const float a2 = two ? dc.y : 0.0f;
                    S[0] = make_float2(dc.y, a2);
                } else {
                    S[r * P + c] = make_float2(v2.x + v1.y, v2.y - v1.x);
                    if (r != 0)
                        S[(N - r) * P + ((N - c) & (N - 1))] = make_float2(v1.y - v2.x, v1.x + v2.y);
                }
            }
        }
        __syncthreads();
        // A') the Nyquist lines: A into S, E transformed (thread: pixel, line, index)
        {
            const int bf = tid >> 8;
            const int ln = (tid >> 7) & 1;
            const int j = tid & 127;
            const float2* cl = ny + bf * 256 + ln * 128;
            const float2 c0 = cl[j];
            const float2 c1 = cl[(N - j) & (N - 1)];
            float2 a = make_float2(0.5f * (c0.x - c1.x), 0.5f * (c0.y + c1.y));
            float2 ev = make_float2(0.5f * (c0.x + c1.x), 0.5f * (c0.y - c1.y));
            if (ln == 1 && j == 64) a = ev = make_float2(0.0f, 0.0f);  // (64, 64): row line
            na[tid] = a;
            eb[tid] = ev;
        }
        __syncthreads();
        if (tid < 256) {
            const int ln = tid >> 7;
            const int j = tid & 127;
            const float2 a1 = na[ln * 128 + j];
            const float2 a2 = na[256 + ln * 128 + j];
            const float2 v = make_float2(a2.x + a1.y, a2.y - a1.x);
            if (ln == 0)
                S[64 * P + j] = v;
            else if (j != 64)
                S[j * P + 64] = v;
        } else if (tid < 320) {
            // warps 8 and 9: E_row + i E_col of one pixel, inverse transform;
            // real part = row line's E^row(x), imaginary = column line's E^col(y)
            const int bf = warp - 8;
            float2* x = eb + bf * 256;
            for (int j = lane; j < 128; j += 32) {
                const float2 er = x[j];
                const float2 ec = x[128 + j];
                x[j] = make_float2(er.x - ec.y, er.y + ec.x);
            }
            __syncwarp();
            line_fft<N, +1>(x, 1, tw, lane);
            for (int j = lane; j < 128; j += 32) {
                el[bf * 256 + j] = x[j].x;
                el[bf * 256 + 128 + j] = x[j].y;
            }
        }
        __syncthreads();
        // B) row IFFTs of S, two rounds of 64 rows
#pragma unroll
        for (int round = 0; round < 2; ++round) {
            float2* rowp = S + (line + 64 * round) * P;
            float2 v[16];
#pragma unroll
            for (int n1 = 0; n1 < 16; ++n1) v[n1] = rowp[s + 8 * n1];
            fft128_g8<+1>(v, Tg, s, tw);
#pragma unroll
            for (int t = 0; t < 16; ++t) rowp[fft128_g8_index(s, t)] = v[t];
        }
        // A of this pair is done with ph: the next pair's phase rows go in now
        if (i + 2 < nb) fill_phase(i + 2);
        __syncthreads();
        // C) column IFFTs: a_1 + i a_2 at (y, x); phases against e_b(y, x)
#pragma unroll
        for (int round = 0; round < 2; ++round) {
            const int x = line + 64 * round;
            const float sx = (x & 1) ? -1.0f : 1.0f;
            const float er1 = el[x];
            const float er2 = el[256 + x];
            float2 v[16];
#pragma unroll
            for (int n1 = 0; n1 < 16; ++n1) v[n1] = S[(s + 8 * n1) * P + x];
            fft128_g8<+1>(v, Tg, s, tw);
#pragma unroll
            for (int t = 0; t < 16; ++t) {
                const int y = fft128_g8_index(s, t);
                const float sy = (y & 1) ? -1.0f : 1.0f;
                const float e1 = fmaf(sx, el[128 + y], fmaf(sy, er1, dc.x));
                const float p1 = phase_atan2(v[t].x, e1);
                float a = p1;
                sq = fma((double)p1, (double)p1, sq);
                if (two) {
                    const float e2 = fmaf(sx, el[384 + y], fmaf(sy, er2, dc.x));
                    const float p2 = phase_atan2(v[t].y, e2);
                    a += p2;
                    sq = fma((double)p2, (double)p2, sq);
                }
                acc[round][t] += a;
            }
        }
        // the cancel flag, read by one thread so the whole CTA stops together
        if (tid == 0 && cancel && *reinterpret_cast<const volatile int*>(cancel) != 0) s_stop = 1;
        __syncthreads();
        if (s_stop) break;
    }
    if (s_stop) sq = __longlong_as_double(0x7ff8000000000000LL);  // NaN: the loss reports it
    // row-major partial sum planes part[(cand * n_chunks + chunk) * N * N + y * N + x]
    float* ps = part + (size_t)(cand * n_chunks + chunk) * N * N;
#pragma unroll
    for (int round = 0; round < 2; ++round) {
        const int x = line + 64 * round;
#pragma unroll
        for (int t = 0; t < 16; ++t) ps[fft128_g8_index(s, t) * N + x] = acc[round][t];
    }
    // the CTA's sum of phi^2: lanes, then the 16 warps in order
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, off);
    if (lane == 0) s_red[warp] = sq;
    __syncthreads();
    if (tid == 0) {
        double t = 0.0;
#pragma unroll
        for (int w = 0; w < 16; ++w) t += s_red[w];
        part_sq[cand * n_chunks + chunk] = t;
    }
    if (!arrivals) return;  // the fold runs as its own kernels
    // In-kernel fold: the last of the candidate's chunks to finish folds them
    // all (no CTA waits for another). Writers make their partials visible
    // before counting in; the counter is left at 0 for the next launch.
    __threadfence();
    __syncthreads();
    if (tid == 0) s_last = atomicAdd(arrivals + cand, 1u) == (unsigned)(n_chunks - 1);
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    constexpr int NN = N * N;
    const float* pc = part + (size_t)cand * n_chunks * NN;
    double neg = 0.0;
    for (int j = tid; j < NN; j += 512) {
        double t = 0.0;
        for (int k = 0; k < n_chunks; ++k) t += (double)__ldcg(pc + (size_t)k * NN + j);
        const double mean = t / (double)n_bf;
        if (mean_phase) mean_phase[(size_t)cand * NN + j] = (float)mean;
        neg -= mean * mean;
    }
    double* red = reinterpret_cast<double*>(S);  // S is free now
    red[tid] = neg;
    __syncthreads();
    for (int w = 256; w > 0; w >>= 1) {
        if (tid < w) red[tid] += red[tid + w];
        __syncthreads();
    }
    if (tid == 0) {
        double q = 0.0;
        for (int k = 0; k < n_chunks; ++k) q += __ldcg(part_sq + (size_t)cand * n_chunks + k);
        losses[cand] = (float)((red[0] + q / (double)n_bf) / (double)NN);
        arrivals[cand] = 0u;
    }
}

// The pair kernel's fold: per pixel the FP64 sum of the chunks' phi planes,
// the mean phase, and -mean^2 summed over the block's 32 pixels (the sum of
// squares arrives as one FP64 number per chunk, added in k_loss_final_sq).
template <int N>
__global__ void __launch_bounds__(kReducePix * kReduceSlices) k_loss_reduce_sum(
    const float* __restrict__ part, int n_chunks, int n_bf, double* __restrict__ block_var,
    float* __restrict__ mean_phase) {
    __shared__ double r1[kReduceSlices][kReducePix];
    __shared__ double rv[kReducePix];
    const int px = threadIdx.x & (kReducePix - 1);
    const int sl = threadIdx.x / kReducePix;
    const int j = blockIdx.x * kReducePix + px;  // y * N + x
    const int cand = blockIdx.y;
    constexpr size_t NN = (size_t)N * N;
    const float* cbase = part + (size_t)cand * n_chunks * NN + j;
    double s1 = 0.0;
    int k = sl;
    for (; k + 3 * kReduceSlices < n_chunks; k += 4 * kReduceSlices) {
        float a[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) a[u] = __ldg(cbase + (size_t)(k + u * kReduceSlices) * NN);
#pragma unroll
        for (int u = 0; u < 4; ++u) s1 += (double)a[u];
    }
    for (; k < n_chunks; k += kReduceSlices) s1 += (double)__ldg(cbase + (size_t)k * NN);
    r1[sl][px] = s1;
    __syncthreads();
    if (sl == 0) {
        double t1 = 0.0;
#pragma unroll
        for (int w = 0; w < kReduceSlices; ++w) t1 += r1[w][px];
        const double mean = t1 / (double)n_bf;
        rv[px] = -mean * mean;
        if (mean_phase) mean_phase[(size_t)cand * NN + j] = (float)mean;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double acc = 0.0;
#pragma unroll
        for (int i = 0; i < kReducePix; ++i) acc += rv[i];
        block_var[(size_t)cand * (NN / kReducePix) + blockIdx.x] = acc;
    }
}

// L = (sum of the blocks' -mean^2 + (sum of phi^2) / B) / N^2, fixed order.
__global__ void __launch_bounds__(256) k_loss_final_sq(const double* __restrict__ block_var,
                                                       int n_blocks, const double* __restrict__ part_sq,
                                                       int n_chunks, int n_bf, int npos,
                                                       float* __restrict__ losses) {
    __shared__ double red[256];
    const int cand = blockIdx.x;
    const double* v = block_var + (size_t)cand * n_blocks;
    double acc = 0.0;
    for (int i = threadIdx.x; i < n_blocks; i += 256) acc += v[i];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double q = 0.0;
        for (int k = 0; k < n_chunks; ++k) q += part_sq[(size_t)cand * n_chunks + k];
        losses[cand] = (float)((red[0] + q / (double)n_bf) / (double)npos);
    }
}


// ---------------------------------------------- N >= 256: two passes
// A 256^2 .. 1024^2 plane does not fit one CTA's shared memory. The BF pixels
// are taken in chunks whose row-transformed planes stay in L2 (about 48 MB
// for all candidates of the call):
//   k_loss_rows: one warp per row of C_b (rows 0..N/2 on the +-q half set, all
//     N rows for the 14-term chi): evaluate, inverse-FFT, store the row in the
//     chunk's staging planes; the half-set path also stores
//     delta_r = conj C(r, N/2) + C(-r, N/2), r = 1..N/2-1, the Nyquist-column
//     deviation from C(-q) = -conj C(q) (row(-r) = -conj row(r) + (-1)^x delta_r
//     after the row transforms);
//   k_loss_cols: a CTA owns a strip of 16 columns (8 at 1024) and every n_sub-th BF pixel
//     of the chunk: it loads the strip (coalesced 128-byte rows), rebuilds the
//     lower half rows, inverse-FFTs one column per warp and keeps phi and phi^2
//     of its pixels in registers; at the end of the chunk it adds them to its
//     own partial planes (column-major), so every element has one writer.
constexpr int kL256 = 256;
constexpr size_t kStageBudget = 32u << 20;
// The persistent one-launch loss (k_loss_queue, QSSB_FLAG_PERSISTENT): 256^2,
// half set, float32 chi, at most this many candidate groups (27 candidates each).
constexpr int kQueueN = 256;
constexpr int kQueueSlots = 3;  // staging slots of the persistent loss
constexpr int kQueueMaxGroups = 16;
// Queue words: the ticket, the abort word, then per chunk the completed row
// and column items.
__host__ __device__ constexpr int queue_words(int K) { return 2 + 2 * K; }
constexpr int kQueueAbortWord = 1;

static bool loss_queue_requested(int n, int flags) {
    return n == kQueueN && (flags & QSSB_FLAG_PERSISTENT) &&
           !(flags & (QSSB_FLAG_CHI_FP64 | QSSB_FLAG_FULL_PLANE));
}

// Rows per CTA of the row pass and columns per CTA of the column pass (one
// warp each): 16, or 8 at 1024 where a lane holds 32 values of its line.
// Row pass shape: warps per CTA, CTAs per SM asked of the compiler, and the
// elements whose loads are issued before their math. At 256^2 three 8-warp
// CTAs per SM (80 registers) hide more latency than one 16-warp CTA at 128.
__host__ __device__ constexpr int row_warps(int n) { return n >= 1024 ? 8 : (n == 256 ? 8 : 16); }
__host__ __device__ constexpr int row_min_ctas(int n) { return n == 256 ? 3 : 1; }
__host__ __device__ constexpr int row_load_batch(int n) { return n == 256 ? 4 : 8; }
__host__ __device__ constexpr int col_tile(int n) { return n >= 1024 ? 8 : 16; }

template <int N, bool FULL>
struct TwoPass {
    static constexpr int rows = FULL ? N : N / 2 + 1;
    static constexpr int rwarps = row_warps(N);
    // at 256^2 the half set's Nyquist row N/2 is taken by warp 0 of the first
    // CTA after its row 0, so the rows 0 .. N/2 - 1 fill whole CTAs (17 CTAs
    // of 8 warps would leave one CTA a single row)
    static constexpr bool fold_nyquist = !FULL && N == 256;
    static constexpr int row_ctas = fold_nyquist ? N / 2 / rwarps : (rows + rwarps - 1) / rwarps;
    static constexpr int tile = col_tile(N);
    static constexpr int scratch = warp_fft_scratch<N>();
    // column line pitch: odd mod 16 (conflict-free strip loads), and room for
    // the warp FFT's transpose once the line is in registers
    static constexpr int pitch = (scratch > N ? scratch : N) | 1;
    static constexpr size_t row_smem = sizeof(float2) * ((size_t)rwarps * scratch + N);
    static constexpr size_t col_smem = sizeof(float2) * ((size_t)2 * tile * pitch + N);
    // half set at 256^2 and 512^2: column pairs (k_loss_cols_pair), a warp
    // per pair of the strip's columns, staged as one float4 per row (the two
    // columns' values side by side); a pair's lines hold one warp FFT's scratch
    static constexpr bool pair_cols = !FULL && (N == 256 || N == 512);
    static constexpr int pair_warps = tile / 2;
    static constexpr int pair_pitch = (rows > (scratch + 1) / 2 ? rows : (scratch + 1) / 2) | 1;
    // + two buffers of the BF pixel's N/2 Nyquist-column deviations
    static constexpr size_t col_pair_smem = sizeof(float4) * (size_t)2 * pair_warps * pair_pitch +
                                            sizeof(float2) * N + sizeof(float) * (size_t)pair_warps * N +
                                            sizeof(float2) * (size_t)N;
    // CTAs per SM of the column pass, for the plan's wave arithmetic
    static constexpr int col_ctas_per_sm = pair_cols && N == 256 ? 3 : 2;
};

struct TwoPassPlan {
    int group;     // candidates per launch sequence
    int chunk_bf;  // BF pixels per (rows, columns) launch pair
    int n_sub;     // column-pass interleave = partial planes per candidate
};

// Candidates go through the passes in groups whose column pass fills one wave
// of its CTA slots (64 candidates at 256^2: 27, 27 and 10; 16 at 512^2: 9 and
// 7), so that a chunk of the staging budget holds several BF pixels per
// candidate and each column CTA folds them into its moments before one
// read-modify-write of its partial planes (a whole 64-candidate batch at once
// leaves one pixel per chunk). Full waves beat equal groups: 27/27/10 takes
// 1.14 ms per candidate at 256^2 against 1.24 for 22/22/20.
static TwoPassPlan plan_two_pass(int n, bool full, int n_bf, int n_cand, int chunks_req) {
    TwoPassPlan tp;
    const int strips = n / col_tile(n);
    // column-pass CTA slots of the B200 (148 SMs); groups of equal size
    const int slots = 148 * ((!full && n == 256) ? TwoPass<256, false>::col_ctas_per_sm : 2);
    int group = slots / strips;
    if (group < 1) group = 1;
    if (group > n_cand) group = n_cand;
    tp.group = group;
    const size_t per_bf = sizeof(float2) * (size_t)(full ? n : n / 2 + 1) * n;
    long long c = (long long)(kStageBudget / (per_bf * (size_t)group));
    if (c < 1) c = 1;
    if (c > n_bf) c = n_bf;
    tp.chunk_bf = (int)c;
    // whole waves of the column pass's CTA slots, not a last partial wave
    int sub = chunks_req > 0 ? chunks_req : slots / (strips * group);
    if (sub < 1) sub = 1;
    if (sub > tp.chunk_bf) sub = tp.chunk_bf;
    tp.n_sub = sub;
    return tp;
}

// One row-pass work item: rows rowblock * RW .. + RW - 1 of BF pixel b0 + bi
// for candidate cand0 + zc. scr: RW warp FFT scratches; tw: the twiddles
// (filled before the item's first barrier).
template <int N, bool CHI64, bool QUAD, bool FULL>
__device__ __forceinline__ void loss_rows_item(
    const float2* __restrict__ g, int n_bf, const float* __restrict__ geom,
    const float* __restrict__ q_row, const float* __restrict__ q_col, const void* __restrict__ cands,
    const qssb_calibration_t& cal, const Probe* __restrict__ probes,
    const float2* __restrict__ eq_table, int cand0, int b0, int nb_chunk,
    float2* __restrict__ stage, float2* __restrict__ delta, const float2* __restrict__ overlap,
    int rowblock, int bi, int zc, float2* scr, const float2* tw) {
    using TP = TwoPass<N, FULL>;
    constexpr int H = N / 2 + 1;
    constexpr int RW = TP::rwarps;
    constexpr int RPL = N / 32;
    constexpr bool kSep = !FULL && QUAD && !CHI64;
    __shared__ Probe sp;
    __shared__ FullChi sf;
    __shared__ FullChi64 sd;
    __shared__ float2 s_phc[kSep ? N : 1];
    __shared__ float2 s_phr[kSep ? RW : 1];
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int b = b0 + bi;
    const int cand = cand0 + zc;
    const int r0 = rowblock * RW;
    {  // the candidate's probe, from k_two_pass_setup
        const auto* src = reinterpret_cast<const unsigned int*>(probes + cand);
        auto* dst = reinterpret_cast<unsigned int*>(&sp);
        for (int i = tid; i < (int)(sizeof(Probe) / 4); i += 32 * RW) dst[i] = __ldg(src + i);
    }
    if constexpr (FULL) {
        if (tid == 0) {
            const auto* fc = static_cast<const qssb_full_aberrations_t*>(cands) + cand;
            make_full_chi(fc->magnitude, fc->angle_rad, cal.wavelength_A, sf, sd);
        }
    }
    __syncthreads();
    const Probe& p = sp;
    const BFQuad kq = bf_quad(geom, n_bf, b, p);
    float2 pk = make_float2(0.0f, 0.0f);
    if constexpr (FULL) {
        pk = probe_full_at_bf((double)kq.kx + (double)kq.kx_lo, (double)kq.ky + (double)kq.ky_lo,
                              kq.ak, sd);
    } else if constexpr (!QUAD) {
        pk = probe_at_bf<CHI64>(__ldg(geom + 2 * n_bf + b), __ldg(geom + 3 * n_bf + b),
                                __ldg(geom + 4 * n_bf + b), __ldg(geom + 5 * n_bf + b), p);
    }
    if constexpr (kSep) {  // e^{i 2 q_col(c) v} for all columns, e^{i 2 q_row(r) u} for this CTA's rows
        for (int i = tid; i < N + RW; i += 32 * RW) {
            float sn, cs;
            if (i < N) {
                sincosf(2.0f * __ldg(q_col + i) * kq.v, &sn, &cs);
                s_phc[i] = make_float2(cs, sn);
            } else if (r0 + i - N < N) {
                sincosf(2.0f * __ldg(q_row + r0 + i - N) * kq.u, &sn, &cs);
                s_phr[i - N] = make_float2(cs, sn);
            }
        }
        __syncthreads();
    }
    const float2* gb = g + (size_t)b * N * H;
    const float2* eqc = eq_table + (size_t)cand * N * N;
    const float2 dc = make_float2((float)cal.dc_re, (float)cal.dc_im);
    // G is read once per candidate: streaming loads keep the chunk's staged
    // rows in L2 for the column pass
    auto load_g = [&](int rr, int c) -> float2 {
        return c <= N / 2 ? __ldcs(gb + rr * H + c)
                          : cconj(__ldcs(gb + ((N - rr) & (N - 1)) * H + (N - c)));
    };
    // with the per-geometry table the apertures are read, not evaluated
    // (float32 quadratic chi, and the general chi with C30)
    constexpr bool kTab = kSep || (!FULL && !QUAD);
    const bool tab = kTab && overlap != nullptr;
    const float2* ovb = tab ? overlap + (size_t)b * two_pass_table_elems<N>() : nullptr;
    auto eval = [&](int rr, int c, float qx, float qy, float2 gv, float2 eq, float2 e_row,
                    float2 ov) -> float2 {
        if constexpr (FULL) {
            return corrected_full<CHI64>(qx, qy, rr, c, kq.kx, kq.ky, kq.kx_lo, kq.ky_lo, pk, gv, p,
                                         sf, sd);
        } else if constexpr (kSep) {
            if (tab) return corrected_table(ov, eq, cmul(e_row, s_phc[c]), kq.ak, gv);
            const float2 lo = make_float2(kq.kx_lo, kq.ky_lo);
            return corrected_quad_e(qx, qy, rr, c, eq, kq.kx, kq.ky, kq.ak, &lo,
                                    cmul(e_row, s_phc[c]), gv, p);
        } else if constexpr (QUAD) {
            return corrected_quad<CHI64>(qx, qy, rr, c, eq, kq, gv, p);
        } else {
            if (tab) {
                const Disp dm = displacement(qx - kq.kx, qy - kq.ky, p);
                const Disp dp = displacement(qx + kq.kx, qy + kq.ky, p);
                return corrected_from_apertures<CHI64>(dm, dp, ov.x, ov.y, pk, gv, p);
            }
            return corrected<CHI64>(qx, qy, rr, c, kq.kx, kq.ky, kq.kx_lo, kq.ky_lo, pk, gv, p);
        }
    };
    // one row per warp (e_row: the row's separable phase factor)
    auto row = [&](const int r, const float2 e_row) {
        const float qx = __ldg(q_row + r);
        float2 v[RPL];
        constexpr int kBatch = row_load_batch(N);  // loads issued before their math
#pragma unroll
        for (int t0 = 0; t0 < RPL; t0 += kBatch) {
            float2 gv[kBatch], eq[kBatch], ov[kBatch];
            float qy[kBatch];
#pragma unroll
            for (int u = 0; u < kBatch; ++u) {
                const int c = lane + 32 * (t0 + u);
                gv[u] = load_g(r, c);
                qy[u] = __ldg(q_col + c);
                eq[u] = QUAD && !FULL ? __ldg(eqc + r * N + c) : make_float2(1.0f, 0.0f);
                ov[u] = tab ? __ldg(ovb + r * N + c) : make_float2(0.0f, 0.0f);
            }
#pragma unroll
            for (int u = 0; u < kBatch; ++u) {
                const int t = t0 + u;
                const int c = lane + 32 * t;
                v[t] = (r == 0 && c == 0) ? dc : eval(r, c, qx, qy[u], gv[u], eq[u], e_row, ov[u]);
                if (!FULL && t == N / 64 && lane == 0 && r >= 1 && r < N / 2) {  // c == N/2
                    float2 e_neg = make_float2(1.0f, 0.0f);
                    if constexpr (kSep) {
                        float sn, cs;
                        sincosf(2.0f * __ldg(q_row + N - r) * kq.u, &sn, &cs);
                        e_neg = make_float2(cs, sn);
                    }
                    const float2 eqn = QUAD && !FULL ? __ldg(eqc + (N - r) * N + N / 2)
                                                     : make_float2(1.0f, 0.0f);
                    const float2 ovn =
                        tab ? __ldg(ovb + (N / 2 + 1) * N + r) : make_float2(0.0f, 0.0f);
                    const float2 partner = eval(N - r, N / 2, __ldg(q_row + N - r), qy[u],
                                                load_g(N - r, N / 2), eqn, e_neg, ovn);
                    delta[((size_t)zc * nb_chunk + bi) * (N / 2) + r] =
                        cadd(cconj(v[t]), partner);
                }
            }
        }
        warp_fft<N, +1>(v, scr + warp * TP::scratch, tw, lane);
        float2* out = stage + (((size_t)zc * nb_chunk + bi) * TP::rows + r) * N;
#pragma unroll
        for (int j = 0; j < RPL; ++j) out[warp_fft_index<N>(lane, j)] = v[j];
    };
    const int r = r0 + warp;
    if (r < TP::rows) row(r, kSep ? s_phr[warp] : make_float2(1.0f, 0.0f));
    if constexpr (TP::fold_nyquist) {
        static_assert(TP::row_ctas * RW == N / 2, "whole CTAs of rows");
        if (rowblock == 0 && warp == 0) {
            __syncwarp();  // the FFT scratch is reused by the Nyquist row
            float2 e_row = make_float2(1.0f, 0.0f);
            if constexpr (kSep) {
                float sn, cs;
                sincosf(2.0f * __ldg(q_row + N / 2) * kq.u, &sn, &cs);
                e_row = make_float2(cs, sn);
            }
            row(N / 2, e_row);
        }
    }
}

template <int N, bool CHI64, bool QUAD, bool FULL>
__global__ void __launch_bounds__(32 * row_warps(N), row_min_ctas(N)) k_loss_rows(
    const float2* __restrict__ g, int n_bf, const float* __restrict__ geom,
    const float* __restrict__ q_row, const float* __restrict__ q_col, const void* __restrict__ cands,
    qssb_calibration_t cal, const Probe* __restrict__ probes, const float2* __restrict__ twg,
    const float2* __restrict__ eq_table, int cand0, int b0, int nb_chunk,
    float2* __restrict__ stage, float2* __restrict__ delta, const float2* __restrict__ overlap) {
    using TP = TwoPass<N, FULL>;
    extern __shared__ float4 smem4[];
    float2* scr = reinterpret_cast<float2*>(smem4);
    float2* tw = scr + TP::rwarps * TP::scratch;
    for (int i = threadIdx.x; i < N; i += 32 * TP::rwarps) tw[i] = __ldg(twg + i);
    loss_rows_item<N, CHI64, QUAD, FULL>(g, n_bf, geom, q_row, q_col, cands, cal, probes,
                                         eq_table, cand0, b0, nb_chunk, stage, delta, overlap,
                                         blockIdx.x, blockIdx.y, blockIdx.z, scr, tw);
}

__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gmem_src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(gmem_src) : "memory");
}

template <int N, bool FULL>
__global__ void __launch_bounds__(32 * col_tile(N)) k_loss_cols(
    const float2* __restrict__ stage, const float2* __restrict__ delta,
    const float2* __restrict__ twg, int cand0, int nb_chunk, int n_sub, int first,
    float* __restrict__ part) {
    using TP = TwoPass<N, FULL>;
    constexpr int P = TP::pitch;
    constexpr int RPL = N / 32;
    constexpr int kColTile = TP::tile;
    constexpr int NT = 32 * kColTile;
    extern __shared__ float4 smem4[];
    float2* tiles = reinterpret_cast<float2*>(smem4);  // two strips: the next one arrives by cp.async
    float2* tw = tiles + 2 * kColTile * P;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int x0 = blockIdx.x * kColTile;
    const int sub = blockIdx.y;
    const int zc = blockIdx.z;  // the candidate within the group (staging index)
    const int cand = cand0 + zc;
    const int x = x0 + warp;
    const float sign = (x & 1) ? -1.0f : 1.0f;
    for (int i = tid; i < N; i += NT) tw[i] = __ldg(twg + i);
    auto issue = [&](int bi, float2* dst) {
        const float2* S = stage + ((size_t)zc * nb_chunk + bi) * TP::rows * N + x0;
        for (int e = tid; e < TP::rows * kColTile; e += NT) {
            const int rr = e / kColTile;
            const int c = e - rr * kColTile;
            cp_async8(dst + c * P + rr, S + (size_t)rr * N + c);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
    float as[RPL], aq[RPL];
#pragma unroll
    for (int t = 0; t < RPL; ++t) as[t] = aq[t] = 0.0f;
    int buf = 0;
    if (sub < nb_chunk) issue(sub, tiles);
    for (int bi = sub; bi < nb_chunk; bi += n_sub) {
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        // this strip has arrived everywhere; every warp is done with the other
        // buffer (and tw is filled)
        __syncthreads();
        if (bi + n_sub < nb_chunk) issue(bi + n_sub, tiles + (buf ^ 1) * kColTile * P);
        float2* line = tiles + buf * kColTile * P + warp * P;
        if constexpr (!FULL) {
            const float2* d = delta + ((size_t)zc * nb_chunk + bi) * (N / 2);
#pragma unroll
            for (int t = 0; t < RPL; ++t) {
                const int rr = lane + 32 * t;
                if (rr > N / 2) {
                    const float2 m = line[N - rr];
                    const float2 dd = __ldg(d + N - rr);
                    line[rr] = make_float2(fmaf(sign, dd.x, -m.x), fmaf(sign, dd.y, m.y));
                }
            }
            __syncwarp();
        }
        float2 v[RPL];
#pragma unroll
        for (int t = 0; t < RPL; ++t) v[t] = line[lane + 32 * t];
        __syncwarp();  // the line becomes the FFT's transpose scratch
        warp_fft<N, +1>(v, line, tw, lane);
#pragma unroll
        for (int j = 0; j < RPL; ++j) {
            const float ph = phase_atan2(v[j].y, v[j].x);
            as[j] += ph;
            aq[j] = fmaf(ph, ph, aq[j]);
        }
        buf ^= 1;
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    float* ps = part + ((size_t)(cand * n_sub + sub) * 2) * N * N + (size_t)x * N;
    float* pq = ps + (size_t)N * N;
#pragma unroll
    for (int j = 0; j < RPL; ++j) {
        const int y = warp_fft_index<N>(lane, j);
        if (first) {
            ps[y] = as[j];
            pq[y] = aq[j];
        } else {
            ps[y] += as[j];
            pq[y] += aq[j];
        }
    }
}

// 16-byte cp.async: through L2 only (L2ONLY, for data written earlier in the
// same launch by other SMs) or allocating in L1 as well
template <bool L2ONLY>
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    if constexpr (L2ONLY)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem_src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem_src) : "memory");
}

// The column pass of the half set two columns at a time (256^2, 512^2). A
// column line L of the row-transformed half plane, completed by the +-q
// relation L[N - r] = -conj(L[r]) + s delta_r (s = (-1)^x, delta_r the
// Nyquist-column deviation of row r), splits into an anti-Hermitian part
//   AL[r] = L[r] - (s/2) conj(delta_r), AL[N - r] = -conj(AL[r]),
//   AL[0] = i Im L[0], AL[N/2] = i Im L[N/2],
// whose transform is purely imaginary, and a Hermitian part whose transform
// is real: Re L[0] + (-1)^y Re L[N/2] + s Dhat(y), with
// Dhat(y) = Re sum_r delta_r w^{-r y} the same for every column of the BF
// pixel. So one complex FFT of AL_a + i AL_b gives both columns' imaginary
// parts (i Y_a - Y_b), and one FFT per BF pixel gives Dhat: about half the
// column FFTs of k_loss_cols. Dhat is computed W pixels ahead, one per warp,
// with the idle strip buffer as scratch. L2ONLY (the persistent queue kernel,
// whose producers write in the same launch): staged rows, deviations and
// partial planes are read through L2 only (cp.async.cg, ld.global.cg).
template <int N, bool L2ONLY>
__device__ __forceinline__ void loss_cols_pair_item(
    const float2* __restrict__ stage, const float2* __restrict__ delta, int cand0, int nb_chunk,
    int n_sub, int first, float* __restrict__ part, int strip, int sub, int zc, float4* tiles,
    const float2* tw, float* dh, float2* dsm) {
    using TP = TwoPass<N, false>;
    constexpr int P = TP::pair_pitch;
    constexpr int RPL = N / 32;
    constexpr int kColTile = TP::tile;
    constexpr int W = TP::pair_warps;
    constexpr int NT = 32 * W;
    static_assert(TP::pair_cols && 2 * P >= TP::scratch, "a pair's lines hold the FFT scratch");
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int x0 = strip * kColTile;
    const int cand = cand0 + zc;
    const int xa = x0 + 2 * warp;  // even: s = +1 for column xa, -1 for xa + 1
    // the strip of BF pixel bi and its deviations (dsm: two buffers of N/2)
    auto issue = [&](int bi, int into) {
        float4* dst = tiles + into * W * P;
        const float2* S = stage + ((size_t)zc * nb_chunk + bi) * TP::rows * N + x0;
        for (int e = tid; e < TP::rows * W; e += NT) {
            const int rr = e / W;
            const int pp = e - rr * W;
            cp_async16<L2ONLY>(dst + pp * P + rr, S + (size_t)rr * N + 2 * pp);
        }
        if constexpr (L2ONLY) {  // else read from global through L1
            const float2* D = delta + ((size_t)zc * nb_chunk + bi) * (N / 2);
            for (int e = tid; e < N / 4; e += NT)
                cp_async16<true>(dsm + into * (N / 2) + 2 * e, D + 2 * e);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
    float asa[RPL], aqa[RPL], asb[RPL], aqb[RPL];
#pragma unroll
    for (int t = 0; t < RPL; ++t) asa[t] = aqa[t] = asb[t] = aqb[t] = 0.0f;
    int buf = 0;
    if (sub < nb_chunk) issue(sub, 0);
    int step = 0;
    for (int bi = sub; bi < nb_chunk; bi += n_sub, ++step) {
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        // this strip has arrived everywhere; every warp is done with the other
        // buffer (and tw is filled)
        __syncthreads();
        const int slot = step % W;
        if (slot == 0) {  // CTA-uniform
            const int bj = bi + warp * n_sub;
            if (bj < nb_chunk) {
                const float2* d = delta + ((size_t)zc * nb_chunk + bj) * (N / 2);
                float2 v[RPL];
#pragma unroll
                for (int t = 0; t < RPL; ++t) {
                    const int rr = lane + 32 * t;
                    v[t] = rr > N / 2 ? (L2ONLY ? __ldcg(d + N - rr) : __ldg(d + N - rr))
                                      : make_float2(0.0f, 0.0f);
                }
                warp_fft<N, +1>(v, reinterpret_cast<float2*>(tiles + ((buf ^ 1) * W + warp) * P),
                                tw, lane);
#pragma unroll
                for (int j = 0; j < RPL; ++j) dh[warp * N + warp_fft_index<N>(lane, j)] = v[j].x;
            }
            __syncthreads();
        }
        if (bi + n_sub < nb_chunk) issue(bi + n_sub, buf ^ 1);
        float4* pr = tiles + (buf * W + warp) * P;
        const float2* d =
            L2ONLY ? dsm + buf * (N / 2) : delta + ((size_t)zc * nb_chunk + bi) * (N / 2);
        float2 v[RPL];
#pragma unroll
        for (int t = 0; t < RPL; ++t) {
            const int rr = lane + 32 * t;
            if (rr == 0 || rr == N / 2) {
                const float4 q = pr[rr];
                v[t] = make_float2(-q.w, q.y);
            } else {
                const int rp = rr < N / 2 ? rr : N - rr;
                const float2 dd = L2ONLY ? d[rp] : __ldg(d + rp);
                const float4 q = pr[rp];
                const float ax = fmaf(-0.5f, dd.x, q.x), ay = fmaf(0.5f, dd.y, q.y);
                const float bx = fmaf(0.5f, dd.x, q.z), by = fmaf(-0.5f, dd.y, q.w);
                v[t] = rr < N / 2 ? make_float2(ax - by, ay + bx) : make_float2(-ax - by, ay - bx);
            }
        }
        const float4 h0 = pr[0], hN = pr[N / 2];
        __syncwarp();  // the pair's lines become the FFT's transpose scratch
        warp_fft<N, +1>(v, reinterpret_cast<float2*>(pr), tw, lane);
        const float* dhs = dh + slot * N;
#pragma unroll
        for (int j = 0; j < RPL; ++j) {
            const int y = warp_fft_index<N>(lane, j);
            const float sy = (y & 1) ? -1.0f : 1.0f;
            const float dv = dhs[y];
            const float pa = phase_atan2(v[j].y, fmaf(sy, hN.x, h0.x) + dv);
            const float pb = phase_atan2(-v[j].x, fmaf(sy, hN.z, h0.z) - dv);
            asa[j] += pa;
            aqa[j] = fmaf(pa, pa, aqa[j]);
            asb[j] += pb;
            aqb[j] = fmaf(pb, pb, aqb[j]);
        }
        buf ^= 1;
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    float* ps = part + ((size_t)(cand * n_sub + sub) * 2) * N * N + (size_t)xa * N;
    float* pq = ps + (size_t)N * N;
#pragma unroll
    for (int j = 0; j < RPL; ++j) {
        const int y = warp_fft_index<N>(lane, j);
        if (first) {
            ps[y] = asa[j];
            pq[y] = aqa[j];
            ps[N + y] = asb[j];
            pq[N + y] = aqb[j];
        } else if constexpr (L2ONLY) {
            ps[y] = __ldcg(ps + y) + asa[j];
            pq[y] = __ldcg(pq + y) + aqa[j];
            ps[N + y] = __ldcg(ps + N + y) + asb[j];
            pq[N + y] = __ldcg(pq + N + y) + aqb[j];
        } else {
            ps[y] += asa[j];
            pq[y] += aqa[j];
            ps[N + y] += asb[j];
            pq[N + y] += aqb[j];
        }
    }
}

template <int N>
__global__ void __launch_bounds__(16 * col_tile(N), TwoPass<N, false>::col_ctas_per_sm)
    k_loss_cols_pair(const float2* __restrict__ stage, const float2* __restrict__ delta,
                     const float2* __restrict__ twg, int cand0, int nb_chunk, int n_sub,
                     int first, float* __restrict__ part) {
    using TP = TwoPass<N, false>;
    extern __shared__ float4 smem4[];
    float4* tiles = smem4;  // two strips: the next one arrives by cp.async
    float2* tw = reinterpret_cast<float2*>(tiles + 2 * TP::pair_warps * TP::pair_pitch);
    float* dh = reinterpret_cast<float*>(tw + N);  // [W][N]: Dhat of the next W pixels
    float2* dsm = reinterpret_cast<float2*>(dh + TP::pair_warps * N);
    for (int i = threadIdx.x; i < N; i += 32 * TP::pair_warps) tw[i] = __ldg(twg + i);
    loss_cols_pair_item<N, false>(stage, delta, cand0, nb_chunk, n_sub, first, part, blockIdx.x,
                           blockIdx.y, blockIdx.z, tiles, tw, dh, dsm);
}

struct LossPlan {
    int bf_per_chunk;
    int n_chunks;      // partial planes per candidate
    int chunk_bf;      // N >= 256: BF pixels per row/column launch pair
    int group;         // N >= 256: candidates per row/column launch pair
    size_t part_bytes;
    size_t var_bytes;
    size_t eq_bytes;
    size_t stage_bytes;  // N >= 256: row-transformed planes of one chunk
    size_t delta_bytes;  // N >= 256, half set: Nyquist-column deviations
    size_t setup_bytes;  // N >= 256: per-candidate probes and the N twiddles
    bool queue;          // 256^2 half set: one persistent launch (k_loss_queue)
    int n_groups;        // queue: candidate groups
    int n_phase_chunks;  // queue: BF chunks over all groups
    size_t queue_bytes;  // queue: ticket, abort word and per-chunk completion counts
};

// Deterministic: about 296 CTAs in total (two per B200 SM), at least one BF
// pixel each. N >= 256: the two-pass plan (n_chunks = its column interleave).
static LossPlan plan_loss(int n, int n_bf, int n_cand, int chunks_req = 0, bool full = false,
                          bool queue = false) {
    LossPlan pl;
    pl.queue = false;
    pl.n_groups = 0;
    pl.n_phase_chunks = 0;
    pl.queue_bytes = 0;
    if (n >= kL256) {
        const TwoPassPlan tp = plan_two_pass(n, full, n_bf, n_cand, chunks_req);
        pl.chunk_bf = tp.chunk_bf;
        pl.n_chunks = tp.n_sub;
        pl.bf_per_chunk = 0;
        const size_t rows = full ? (size_t)n : (size_t)(n / 2 + 1);
        pl.group = tp.group;
        pl.stage_bytes = sizeof(float2) * rows * n * (size_t)tp.chunk_bf * tp.group;
        pl.delta_bytes = full ? 0 : sizeof(float2) * (size_t)(n / 2) * tp.chunk_bf * tp.group;
        pl.delta_bytes = (pl.delta_bytes + 255) & ~(size_t)255;
        pl.setup_bytes = ((sizeof(Probe) * (size_t)n_cand + 255) & ~(size_t)255) +
                         sizeof(float2) * (size_t)n;
        const int n_groups = (n_cand + tp.group - 1) / tp.group;
        if (queue && !full && n == kQueueN && n_groups <= kQueueMaxGroups) {
            // kQueueSlots staging slots (rows of later chunks while columns of chunk k)
            pl.queue = true;
            pl.n_groups = n_groups;
            int k = 0;
            for (int g = 0; g < n_groups; ++g) {
                const int nc = n_cand - g * tp.group < tp.group ? n_cand - g * tp.group : tp.group;
                int chunk = tp.chunk_bf * tp.group / nc;
                if (chunk > n_bf) chunk = n_bf;
                k += (n_bf + chunk - 1) / chunk;
            }
            pl.n_phase_chunks = k;
            pl.stage_bytes = kQueueSlots * ((pl.stage_bytes + 255) & ~(size_t)255);
            pl.delta_bytes = kQueueSlots * pl.delta_bytes;
            pl.queue_bytes = (sizeof(int) * (size_t)queue_words(k) + 255) & ~(size_t)255;
        }
    } else if (n == 128 && chunks_req <= 0) {
        // one 512-thread CTA per SM: pick the chunking whose waves are
        // fullest - minimise waves x (pairs per CTA + one pair's worth of
        // per-CTA cost: set-up and its 64 KB partial plane), with an even BF
        // count per chunk (the table kernel takes pixels in pairs), at most
        // 4096 partial planes, fewest chunks on a tie. A fixed function of the
        // problem (the B200's 148 SMs as a constant), so the bits do not
        // depend on the device.
        constexpr long kPlanSms = 148;
        long best = -1;
        int best_bpc = n_bf + (n_bf & 1);
        const int cmax = n_bf < 8192 ? n_bf : 8192;
        for (int c = 1; c <= cmax; ++c) {
            int bpc = (n_bf + c - 1) / c;
            bpc += bpc & 1;
            const long chunks = (n_bf + bpc - 1) / bpc;
            if (c > 1 && (long)n_cand * chunks > 4096) continue;
            const long waves = ((long)n_cand * chunks + kPlanSms - 1) / kPlanSms;
            const long cost = waves * (bpc / 2 + 1);
            if (best < 0 || cost < best) {
                best = cost;
                best_bpc = bpc;
            }
        }
        pl.bf_per_chunk = best_bpc;
        pl.n_chunks = (n_bf + best_bpc - 1) / best_bpc;
        pl.chunk_bf = 0;
        pl.group = 0;
        pl.stage_bytes = 0;
        pl.delta_bytes = 0;
        pl.setup_bytes = 0;
    } else {
        int chunks = chunks_req > 0 ? chunks_req : (296 + n_cand - 1) / n_cand;
        if (chunks < 1) chunks = 1;
        if (chunks > n_bf) chunks = n_bf;
        pl.bf_per_chunk = (n_bf + chunks - 1) / chunks;
        pl.n_chunks = (n_bf + pl.bf_per_chunk - 1) / pl.bf_per_chunk;
        pl.chunk_bf = 0;
        pl.group = 0;
        pl.stage_bytes = 0;
        pl.delta_bytes = 0;
        pl.setup_bytes = 0;
    }
    pl.part_bytes = sizeof(float) * 2 * (size_t)n * n * pl.n_chunks * n_cand;
    pl.part_bytes = (pl.part_bytes + 255) & ~(size_t)255;
    pl.var_bytes = sizeof(double) * (size_t)n * n * n_cand;
    pl.eq_bytes = full ? 0 : sizeof(float2) * (size_t)n * n * n_cand;
    pl.stage_bytes = (pl.stage_bytes + 255) & ~(size_t)255;
    return pl;
}

static size_t loss_workspace(const LossPlan& pl) {
    return pl.part_bytes + pl.var_bytes + pl.eq_bytes + pl.stage_bytes + pl.delta_bytes +
           pl.setup_bytes + pl.queue_bytes;
}

// ------------------------------------- the persistent one-launch loss (256^2)
// With QSSB_FLAG_PERSISTENT one launch runs every row and column item of the
// batch (all candidate groups, all BF chunks) from a global ticket, in the
// order
//   R(0), R(1), C(0), R(2), C(1), ..., R(K-1), C(K-2), C(K-1)
// (R(k): the row items of chunk k, C(k): its column items), with three
// staging slots. An item waits (thread 0, bounded) only for items with
// smaller tickets: C(k) for R(k) and, within a candidate group, for C(k - 1)
// (the partial planes' read-modify-write order); R(k) for C(k - 3) (its slot).
// A waiting CTA holds a ticket taken after the ones it waits on, and every
// ticket taken is held by a running CTA, so the batch drains whatever the
// number of resident CTAs. Producers write through L2 and fence before their
// counts; consumers read staged rows, deviations and partial planes through
// L2 only. The chunking is the launch sequence's, and so are the bits on the
// quadratic path (the general-chi arithmetic, inlined into another kernel,
// may contract differently: float32 rounding). A wait that runs out, or a set
// cancel flag, sets the abort word: later items only count themselves and
// k_loss_final writes NaN losses. CTAs that wait hold their slots; with two
// staging slots that cost 16% against the launch sequence, with three (96 MB
// of L2-resident staging at 27 candidates per group) it is 3% faster with C30
// and 2.5% slower with quadratic chi.
struct QueuePlan {
    int K;       // BF chunks over all candidate groups
    int SR, SC;  // items of one row phase, of one column phase
    int n_sub;
    int n_groups;
    int kstart[kQueueMaxGroups + 1];
    int c0[kQueueMaxGroups];
    int nc[kQueueMaxGroups];
    int chunk[kQueueMaxGroups];
    size_t stage_slot;  // float2 elements per staging slot
    size_t delta_slot;
};

constexpr long long kQueueSpinLimit = 1ll << 22;  // polls 128 ns apart: over half a second

__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Thread 0 of an item: wait until *count reaches target. Nonzero: the batch
// is aborted (the cancel flag is set, this wait ran out, or another did).
__device__ int queue_wait(const int* count, int target, int* abort_word, const int* cancel) {
    for (long long it = 0;; ++it) {
        if (ld_acquire_gpu(count) >= target) return 0;
        if (*reinterpret_cast<volatile int*>(abort_word) != 0) return 1;
        if (cancel && *reinterpret_cast<const volatile int*>(cancel) != 0) {
            atomicCAS(abort_word, 0, 1);
            return 1;
        }
        if (it >= kQueueSpinLimit) {
            atomicCAS(abort_word, 0, 2);
            return 1;
        }
        __nanosleep(128);
    }
}

template <int N, bool QUAD>
__global__ void __launch_bounds__(32 * TwoPass<N, false>::rwarps, 3) k_loss_queue(
    const float2* __restrict__ g, int n_bf, const float* __restrict__ geom,
    const float* __restrict__ q_row, const float* __restrict__ q_col, const void* __restrict__ cands,
    qssb_calibration_t cal, const Probe* __restrict__ probes, const float2* __restrict__ twg,
    const float2* __restrict__ eq_table, float2* __restrict__ stage, float2* __restrict__ delta,
    const float2* __restrict__ overlap, float* __restrict__ part, QueuePlan qp,
    int* __restrict__ queue, const int* __restrict__ cancel) {
    using TP = TwoPass<N, false>;
    static_assert(TP::pair_cols && TP::rwarps == TP::pair_warps, "one CTA shape for both items");
    constexpr int NT = 32 * TP::rwarps;
    constexpr int kStrips = N / TP::tile;
    extern __shared__ float4 smem4[];
    float2* tw = reinterpret_cast<float2*>(smem4);
    float4* area = smem4 + N / 2;  // row items: warp FFT scratches; column items: strips, Dhat
    float2* scr = reinterpret_cast<float2*>(area);
    float4* tiles = area;
    float* dh = reinterpret_cast<float*>(tiles + 2 * TP::pair_warps * TP::pair_pitch);
    float2* dsm = reinterpret_cast<float2*>(dh + TP::pair_warps * N);
    __shared__ int s_item;
    __shared__ int s_skip;
    int* ticket = queue;
    int* abort_word = queue + kQueueAbortWord;
    int* done_r = queue + 2;
    int* done_c = done_r + qp.K;
    for (int i = threadIdx.x; i < N; i += NT) tw[i] = __ldg(twg + i);
    const int total = qp.K * (qp.SR + qp.SC);
    for (;;) {
        __syncthreads();  // the previous item is done with shared memory
        if (threadIdx.x == 0) s_item = atomicAdd(ticket, 1);
        __syncthreads();
        const int t = s_item;
        if (t >= total) break;
        bool row;
        int k, w;
        if (t < qp.SR) {
            row = true;
            k = 0;
            w = t;
        } else {
            const int tp = t - qp.SR;
            const int q = 1 + tp / (qp.SR + qp.SC);
            w = tp - (q - 1) * (qp.SR + qp.SC);
            if (q < qp.K && w < qp.SR) {
                row = true;
                k = q;
            } else {
                row = false;
                k = q - 1;
                if (q < qp.K) w -= qp.SR;
            }
        }
        int gi = 0;
        while (gi + 1 < qp.n_groups && k >= qp.kstart[gi + 1]) ++gi;
        const int kg = k - qp.kstart[gi];
        const int ch = qp.chunk[gi];
        const int b0 = kg * ch;
        const int nb = n_bf - b0 < ch ? n_bf - b0 : ch;
        float2* st = stage + (size_t)(k % kQueueSlots) * qp.stage_slot;
        float2* dl = delta + (size_t)(k % kQueueSlots) * qp.delta_slot;
        if (threadIdx.x == 0) {
            if (cancel && *reinterpret_cast<const volatile int*>(cancel) != 0)
                atomicCAS(abort_word, 0, 1);
            int skip = 0;
            if (row) {
                if (k >= kQueueSlots)
                    skip = queue_wait(done_c + k - kQueueSlots, qp.SC, abort_word, cancel);
            } else {
                skip = queue_wait(done_r + k, qp.SR, abort_word, cancel);
                if (!skip && kg >= 1) skip = queue_wait(done_c + k - 1, qp.SC, abort_word, cancel);
            }
            s_skip = skip | (*reinterpret_cast<volatile int*>(abort_word) != 0);
        }
        __syncthreads();
        if (!s_skip) {  // CTA-uniform, as is every branch below
            if (row) {
                const int rb = w % TP::row_ctas;
                const int pl = w / TP::row_ctas;
                const int zc = pl / ch;
                const int bi = pl - zc * ch;
                if (zc < qp.nc[gi] && bi < nb)
                    loss_rows_item<N, false, QUAD, false>(g, n_bf, geom, q_row, q_col, cands, cal,
                                                          probes, eq_table, qp.c0[gi], b0, nb, st,
                                                          dl, overlap, rb, bi, zc, scr, tw);
            } else {
                const int strip = w % kStrips;
                const int rest = w / kStrips;
                const int sub = rest % qp.n_sub;
                const int zc = rest / qp.n_sub;
                if (zc < qp.nc[gi])
                    loss_cols_pair_item<N, true>(st, dl, qp.c0[gi], nb, qp.n_sub, kg == 0 ? 1 : 0,
                                                 part, strip, sub, zc, tiles, tw, dh, dsm);
            }
        }
        __threadfence();  // this thread's writes of the item, before its count
        __syncthreads();
        if (threadIdx.x == 0) atomicAdd(row ? done_r + k : done_c + k, 1);
    }
}

template <int N>
struct QueueSmem {
    using TP = TwoPass<N, false>;
    static constexpr size_t scr = sizeof(float2) * (size_t)TP::rwarps * TP::scratch;
    static constexpr size_t cols = sizeof(float4) * (size_t)2 * TP::pair_warps * TP::pair_pitch +
                                   sizeof(float) * (size_t)TP::pair_warps * N +
                                   sizeof(float2) * (size_t)N;
    static constexpr size_t bytes = sizeof(float2) * N + (scr > cols ? scr : cols);
};

// Once per batch: every candidate's probe parameters (FP64 divisions and the
// FP64 cos/sin of 2 phi12) and the N FFT twiddles, so that the row and column
// CTAs start by copying them instead of evaluating them in a serial prologue.
template <int N, bool FULL>
__global__ void __launch_bounds__(128) k_two_pass_setup(const void* __restrict__ cands,
                                                         qssb_calibration_t cal, int n_cand,
                                                         Probe* __restrict__ probes,
                                                         float2* __restrict__ tw,
                                                         int* __restrict__ queue, int n_queue) {
    const int i = blockIdx.x * 128 + threadIdx.x;
    if (i < n_queue) queue[i] = 0;  // the queue kernel's ticket, abort word and counts
    if (i < n_cand) {
        if constexpr (FULL) {
            probes[i] = make_probe_common(cal, 0.0f, 0.0f, 0.0f, 0.0f);
        } else {
            const qssb_aberrations_t ab = static_cast<const qssb_aberrations_t*>(cands)[i];
            probes[i] = make_probe_common(cal, ab.C10, ab.C12, ab.phi12, ab.C30);
        }
    }
    fill_twiddles<N>(tw, i, (int)(gridDim.x * 128));
}

// The N >= 256 launch sequence after the eq table: row and column passes per
// BF chunk; the partial planes then go through k_loss_reduce.
template <int N, bool CHI64, bool QUAD, bool FULL>
static int launch_two_pass(const float* g_half, const float* geom, const float* q_row,
                           const float* q_col, const qssb_calibration_t& cal, const void* cands,
                           int n_cand, const LossPlan& pl, const float2* eq, float* part,
                           char* stage_base, cudaStream_t s, const float2* overlap = nullptr) {
    using TP = TwoPass<N, FULL>;
    float2* stage = reinterpret_cast<float2*>(stage_base);
    float2* delta = reinterpret_cast<float2*>(stage_base + pl.stage_bytes);
    Probe* probes = reinterpret_cast<Probe*>(stage_base + pl.stage_bytes + pl.delta_bytes);
    float2* twg = reinterpret_cast<float2*>(stage_base + pl.stage_bytes + pl.delta_bytes +
                                            pl.setup_bytes - sizeof(float2) * N);
    CUDA_TRY(cudaFuncSetAttribute(k_loss_rows<N, CHI64, QUAD, FULL>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TP::row_smem));
    CUDA_TRY(cudaFuncSetAttribute(k_loss_cols<N, FULL>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TP::col_smem));
    if constexpr (TP::pair_cols) {
        CUDA_TRY(cudaFuncSetAttribute(k_loss_cols_pair<N>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)TP::col_pair_smem));
        CUDA_TRY(cudaFuncSetAttribute(k_loss_cols_pair<N>,
                                      cudaFuncAttributePreferredSharedMemoryCarveout,
                                      (int)cudaSharedmemCarveoutMaxShared));
    }
    CUDA_TRY(cudaFuncSetAttribute(k_loss_rows<N, CHI64, QUAD, FULL>,
                                  cudaFuncAttributePreferredSharedMemoryCarveout,
                                  (int)cudaSharedmemCarveoutMaxShared));
    CUDA_TRY(cudaFuncSetAttribute(k_loss_cols<N, FULL>,
                                  cudaFuncAttributePreferredSharedMemoryCarveout,
                                  (int)cudaSharedmemCarveoutMaxShared));
    const auto* g = reinterpret_cast<const float2*>(g_half);
    int* queue = reinterpret_cast<int*>(stage_base + pl.stage_bytes + pl.delta_bytes +
                                        pl.setup_bytes);
    const int n_queue = pl.queue ? queue_words(pl.n_phase_chunks) : 0;
    {
        int n = n_cand > N ? n_cand : N;
        if (n_queue > n) n = n_queue;
        { k_two_pass_setup<N, FULL><<<(n + 127) / 128, 128, 0, s>>>(cands, cal, n_cand, probes, twg,
                                                                   queue, n_queue); note_launch(); }
        CUDA_TRY(cudaGetLastError());
    }
    if constexpr (N == kQueueN && !FULL && !CHI64) {
        if (pl.queue) {
            QueuePlan qp = {};
            qp.n_sub = pl.n_chunks;
            qp.n_groups = pl.n_groups;
            qp.SR = TP::row_ctas * pl.chunk_bf * pl.group;
            qp.SC = (N / TP::tile) * pl.n_chunks * pl.group;
            int k = 0;
            for (int gi = 0; gi < pl.n_groups; ++gi) {
                const int c0 = gi * pl.group;
                const int nc = n_cand - c0 < pl.group ? n_cand - c0 : pl.group;
                int chunk = pl.chunk_bf * pl.group / nc;
                if (chunk > cal.n_bf) chunk = cal.n_bf;
                qp.kstart[gi] = k;
                qp.c0[gi] = c0;
                qp.nc[gi] = nc;
                qp.chunk[gi] = chunk;
                k += (cal.n_bf + chunk - 1) / chunk;
            }
            qp.kstart[pl.n_groups] = k;
            qp.K = k;
            qp.stage_slot = pl.stage_bytes / kQueueSlots / sizeof(float2);
            qp.delta_slot = pl.delta_bytes / kQueueSlots / sizeof(float2);
            if (k != pl.n_phase_chunks || (long long)k * (qp.SR + qp.SC) > INT_MAX)
                return set_error(QSSB_ERR_UNSUPPORTED, "qssb_loss_batch: queue plan mismatch");
            const size_t smem = QueueSmem<N>::bytes;
            CUDA_TRY(cudaFuncSetAttribute(k_loss_queue<N, QUAD>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            CUDA_TRY(cudaFuncSetAttribute(k_loss_queue<N, QUAD>,
                                          cudaFuncAttributePreferredSharedMemoryCarveout,
                                          (int)cudaSharedmemCarveoutMaxShared));
            int per_sm = 0;
            CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &per_sm, k_loss_queue<N, QUAD>, 32 * TP::rwarps, smem));
            if (per_sm < 1) per_sm = 1;
            { k_loss_queue<N, QUAD><<<device_sm_count() * per_sm, 32 * TP::rwarps, smem, s>>>(
                g, cal.n_bf, geom, q_row, q_col, cands, cal, probes, twg, eq, stage, delta, overlap,
                part, qp, queue, cancel_flag()); note_launch(); }
            CUDA_TRY(cudaGetLastError());
            return QSSB_OK;
        }
    }
    for (int c0 = 0; c0 < n_cand; c0 += pl.group) {
        const int nc = n_cand - c0 < pl.group ? n_cand - c0 : pl.group;
        // a smaller last group takes more BF pixels per chunk in the same staging
        int chunk = pl.chunk_bf * pl.group / nc;
        if (chunk > cal.n_bf) chunk = cal.n_bf;
        for (int b0 = 0; b0 < cal.n_bf; b0 += chunk) {
            const int nb = cal.n_bf - b0 < chunk ? cal.n_bf - b0 : chunk;
            { k_loss_rows<N, CHI64, QUAD, FULL>
                <<<dim3(TP::row_ctas, nb, nc), 32 * TP::rwarps, TP::row_smem, s>>>(
                    g, cal.n_bf, geom, q_row, q_col, cands, cal, probes, twg, eq, c0, b0, nb,
                    stage, delta, overlap); note_launch(); }
            CUDA_TRY(cudaGetLastError());
            if constexpr (TP::pair_cols) {
                { k_loss_cols_pair<N><<<dim3(N / TP::tile, pl.n_chunks, nc), 32 * TP::pair_warps,
                                        TP::col_pair_smem, s>>>(stage, delta, twg, c0, nb,
                                                                pl.n_chunks, b0 == 0 ? 1 : 0,
                                                                part); note_launch(); }
            } else {
                { k_loss_cols<N, FULL><<<dim3(N / TP::tile, pl.n_chunks, nc), 32 * TP::tile,
                                       TP::col_smem, s>>>(stage, delta, twg, c0, nb, pl.n_chunks,
                                                          b0 == 0 ? 1 : 0, part); note_launch(); }
            }
            CUDA_TRY(cudaGetLastError());
        }
    }
    return QSSB_OK;
}

template <int N, bool SYM, bool CHI64, bool QUAD>
static int launch_loss(const float* g_half, const float* geom, const float* q_row,
                       const float* q_col, const qssb_calibration_t& cal,
                       const qssb_aberrations_t* cands, int n_cand, int flags, char* ws,
                       float* losses, float* mean_phase, const float2* overlap, cudaStream_t s) {
    const LossPlan pl = plan_loss(N, cal.n_bf, n_cand, flag_chunks(flags), false,
                                  loss_queue_requested(N, flags));
    float* part = reinterpret_cast<float*>(ws);
    double* var = reinterpret_cast<double*>(ws + pl.part_bytes);
    float2* eq = reinterpret_cast<float2*>(ws + pl.part_bytes + pl.var_bytes);
    if (QUAD) {
        { k_eq_table<N><<<dim3((N * N + 255) / 256, n_cand), 256, 0, s>>>(cands, cal, eq); note_launch(); }
        CUDA_TRY(cudaGetLastError());
    }
    if constexpr (N == 128 && SYM) {
        if (overlap) {
            // the pair kernel: sum planes (one per chunk) then one double per chunk
            double* part_sq = reinterpret_cast<double*>(part + (size_t)n_cand * pl.n_chunks * N * N);
            // a candidate's chunks folded by its last CTA when they are few
            // (one launch); many chunks fold faster in the parallel kernels
            const bool fused = pl.n_chunks <= kFusedFoldChunks;
            unsigned int* arrivals = reinterpret_cast<unsigned int*>(part_sq + (size_t)n_cand * pl.n_chunks);
            if (fused) CUDA_TRY(cudaMemsetAsync(arrivals, 0, sizeof(unsigned int) * n_cand, s));
            const size_t smem = Pair128Smem::bytes;
            CUDA_TRY(cudaFuncSetAttribute(k_loss_pair128<CHI64, QUAD>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            { k_loss_pair128<CHI64, QUAD><<<dim3(pl.n_chunks, n_cand), 512, smem, s>>>(
                reinterpret_cast<const float2*>(g_half), cal.n_bf, geom, q_row, q_col, overlap,
                cands, cal, eq, pl.bf_per_chunk, pl.n_chunks, part, part_sq, cancel_flag(),
                fused ? arrivals : nullptr, losses, mean_phase); note_launch(); }
            CUDA_TRY(cudaGetLastError());
            if (fused) return QSSB_OK;
            { k_loss_reduce_sum<N><<<dim3(N * N / kReducePix, n_cand), kReducePix * kReduceSlices, 0, s>>>(
                part, pl.n_chunks, cal.n_bf, var, mean_phase); note_launch(); }
            CUDA_TRY(cudaGetLastError());
            { k_loss_final_sq<<<n_cand, 256, 0, s>>>(var, N * N / kReducePix, part_sq, pl.n_chunks,
                                                   cal.n_bf, N * N, losses); note_launch(); }
            CUDA_TRY(cudaGetLastError());
            return QSSB_OK;
        }
    }
    if constexpr (N >= kL256) {
        static_assert(SYM, "the two-pass loss evaluates the half set");
        const int rc = launch_two_pass<N, CHI64, QUAD, false>(
            g_half, geom, q_row, q_col, cal, cands, n_cand, pl, eq, part,
            ws + pl.part_bytes + pl.var_bytes + pl.eq_bytes, s, overlap);
        if (rc) return rc;
    } else if constexpr (N == 128) {
        const size_t smem = Loss128Smem::bytes;
        CUDA_TRY(cudaFuncSetAttribute(k_loss_moments128<CHI64, QUAD>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        { k_loss_moments128<CHI64, QUAD><<<dim3(pl.n_chunks, n_cand), 512, smem, s>>>(
            reinterpret_cast<const float2*>(g_half), cal.n_bf, geom, q_row, q_col, cands, cal, eq,
            pl.bf_per_chunk, pl.n_chunks, part); note_launch(); }
    } else {
        const size_t smem = LossSmem<N>::bytes;
        CUDA_TRY(cudaFuncSetAttribute(k_loss_moments<N, SYM, CHI64, QUAD>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        { k_loss_moments<N, SYM, CHI64, QUAD><<<dim3(pl.n_chunks, n_cand), kLossThreads, smem, s>>>(
            reinterpret_cast<const float2*>(g_half), cal.n_bf, geom, q_row, q_col, cands, cal, eq,
            pl.bf_per_chunk, pl.n_chunks, part); note_launch(); }
    }
    CUDA_TRY(cudaGetLastError());
    { k_loss_reduce<N><<<dim3(N * N / kReducePix, n_cand), kReducePix * kReduceSlices, 0, s>>>(
        part, pl.n_chunks, cal.n_bf, var, mean_phase, N == 128 ? 1 : 0); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    // the persistent loss's abort word (cancel or a wait that ran out): NaN losses
    const int* status = nullptr;
    if (pl.queue)
        status = reinterpret_cast<const int*>(ws + pl.part_bytes + pl.var_bytes + pl.eq_bytes +
                                              pl.stage_bytes + pl.delta_bytes + pl.setup_bytes) +
                 kQueueAbortWord;
    { k_loss_final<<<n_cand, 256, 0, s>>>(var, N * N / kReducePix, N * N, losses, status); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}

template <int N, bool QUAD>
static int dispatch_loss_q(bool sym, bool chi64, const float* g_half, const float* geom,
                           const float* q_row, const float* q_col, const qssb_calibration_t& cal,
                           const qssb_aberrations_t* cands, int n_cand, int flags, char* ws,
                           float* losses, float* mean_phase, const float2* ov, cudaStream_t s) {
    if constexpr (N >= kL256) {
        if (!sym)
            return set_error(QSSB_ERR_UNSUPPORTED,
                             "qssb_loss_batch: QSSB_FLAG_FULL_PLANE is offered up to 128^2");
        return chi64 ? launch_loss<N, true, true, QUAD>(g_half, geom, q_row, q_col, cal, cands, n_cand, flags, ws, losses, mean_phase, ov, s)
                     : launch_loss<N, true, false, QUAD>(g_half, geom, q_row, q_col, cal, cands, n_cand, flags, ws, losses, mean_phase, ov, s);
    } else {
        if (sym)
            return chi64 ? launch_loss<N, true, true, QUAD>(g_half, geom, q_row, q_col, cal, cands, n_cand, flags, ws, losses, mean_phase, ov, s)
                         : launch_loss<N, true, false, QUAD>(g_half, geom, q_row, q_col, cal, cands, n_cand, flags, ws, losses, mean_phase, ov, s);
        return chi64 ? launch_loss<N, false, true, QUAD>(g_half, geom, q_row, q_col, cal, cands, n_cand, flags, ws, losses, mean_phase, ov, s)
                     : launch_loss<N, false, false, QUAD>(g_half, geom, q_row, q_col, cal, cands, n_cand, flags, ws, losses, mean_phase, ov, s);
    }
}

// Candidates live on the device, so the path is chosen by a flag: the
// general (C30) path unless QSSB_FLAG_QUADRATIC promises C30 == 0 for all.
template <int N>
static int dispatch_loss(bool sym, bool chi64, bool quad, const float* g_half, const float* geom,
                         const float* q_row, const float* q_col, const qssb_calibration_t& cal,
                         const qssb_aberrations_t* cands, int n_cand, int flags, char* ws,
                         float* losses, float* mean_phase, const float2* ov, cudaStream_t s) {
    if (quad)
        return dispatch_loss_q<N, true>(sym, chi64, g_half, geom, q_row, q_col, cal, cands, n_cand, flags, ws, losses, mean_phase, ov, s);
    return dispatch_loss_q<N, false>(sym, chi64, g_half, geom, q_row, q_col, cal, cands, n_cand, flags, ws, losses, mean_phase, ov, s);
}

// ------------------------------------------------------ 14-term chi
// Odd-m terms (C21, C23, C41, C43, C45) make chi odd in part, which breaks
// C(-q) = -conj C(q): every scan frequency is evaluated. N <= 128: the whole
// N x (N+1) plane in shared memory (k_loss_moments without the mirror).
// N >= 256: each warp evaluates, inverse-FFTs and stages full rows in the
// CTA's global plane, then rebuilds its columns from it (k_loss_staged
// without the row(-r) reconstruction). Partial planes are column-major.
struct FullConsts {
    Probe p;
    FullChi f;
    FullChi64 d;
};

__device__ __forceinline__ void load_full_consts(FullConsts& sh, const qssb_full_aberrations_t* cands,
                                                 int cand, const qssb_calibration_t& cal) {
    sh.p = make_probe_common(cal, 0.0f, 0.0f, 0.0f, 0.0f);
    make_full_chi(cands[cand].magnitude, cands[cand].angle_rad, cal.wavelength_A, sh.f, sh.d);
}

template <int N, bool CHI64>
__global__ void __launch_bounds__(kLossThreads, 1) k_loss_full(
    const float2* __restrict__ g, int n_bf, const float* __restrict__ geom,
    const float* __restrict__ q_row, const float* __restrict__ q_col,
    const qssb_full_aberrations_t* __restrict__ cands, qssb_calibration_t cal, int bf_per_chunk,
    int n_chunks, float* __restrict__ part) {
    constexpr int H = N / 2 + 1;
    constexpr int P = LossSmem<N>::P;
    constexpr int CPW = N / kLossWarps;
    constexpr int RPL = N / 32;
    extern __shared__ float2 smem[];
    __shared__ FullConsts sh;
    float2* plane = smem;
    float2* tw = smem + N * P;
    float* sq = reinterpret_cast<float*>(tw + N);  // [col][row] sums of squares
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int chunk = blockIdx.x;
    const int cand = blockIdx.y;
    if (tid == 0) load_full_consts(sh, cands, cand, cal);
    fill_twiddles<N>(tw, tid, kLossThreads);
    for (int i = tid; i < N * N; i += kLossThreads) sq[i] = 0.0f;
    __syncthreads();
    float as[CPW][RPL];
#pragma unroll
    for (int i = 0; i < CPW; ++i)
#pragma unroll
        for (int t = 0; t < RPL; ++t) as[i][t] = 0.0f;
    const int b0 = chunk * bf_per_chunk;
    int nb = n_bf - b0;
    if (nb > bf_per_chunk) nb = bf_per_chunk;
    const float2 dc = make_float2((float)cal.dc_re, (float)cal.dc_im);
    for (int i = 0; i < nb; ++i) {
        const int b = b0 + i;
        const float kx = __ldg(geom + b);
        const float ky = __ldg(geom + n_bf + b);
        const float kx_lo = __ldg(geom + 6 * n_bf + b);
        const float ky_lo = __ldg(geom + 7 * n_bf + b);
        const float2 pk = probe_full_at_bf((double)kx + (double)kx_lo, (double)ky + (double)ky_lo,
                                           __ldg(geom + 5 * n_bf + b), sh.d);
        const float2* gb = g + (size_t)b * N * H;
        for (int e = tid; e < N * N; e += kLossThreads) {
            const int r = e / N;
            const int c = e - r * N;
            const float2 gv = c <= N / 2 ? __ldg(gb + r * H + c)
                                         : cconj(__ldg(gb + ((N - r) & (N - 1)) * H + (N - c)));
            float2 v = corrected_full<CHI64>(__ldg(q_row + r), __ldg(q_col + c), r, c, kx, ky, kx_lo,
                                             ky_lo, pk, gv, sh.p, sh.f, sh.d);
            if (e == 0) v = dc;
            plane[r * P + c] = v;
        }
        __syncthreads();
        for (int row = warp; row < N; row += kLossWarps) line_fft<N, +1>(plane + row * P, 1, tw, lane);
        __syncthreads();
#pragma unroll
        for (int ci = 0; ci < CPW; ++ci) {
            const int col = warp + ci * kLossWarps;
            line_fft<N, +1>(plane + col, P, tw, lane);
#pragma unroll
            for (int t = 0; t < RPL; ++t) {
                const float2 v = plane[(lane + 32 * t) * P + col];
                const float ph = phase_atan2(v.y, v.x);
                as[ci][t] += ph;
                float* q2 = sq + col * N + lane + 32 * t;
                *q2 = fmaf(ph, ph, *q2);
            }
        }
        __syncthreads();
    }
    float* ps = part + ((size_t)(cand * n_chunks + chunk) * 2) * N * N;
    float* pq = ps + (size_t)N * N;
#pragma unroll
    for (int ci = 0; ci < CPW; ++ci) {
        const int col = warp + ci * kLossWarps;
#pragma unroll
        for (int t = 0; t < RPL; ++t) ps[col * N + lane + 32 * t] = as[ci][t];
    }
    for (int i = tid; i < N * N; i += kLossThreads) pq[i] = sq[i];
}

template <int N, bool CHI64>
static int launch_loss_full(const float* g_half, const float* geom, const float* q_row,
                            const float* q_col, const qssb_calibration_t& cal,
                            const qssb_full_aberrations_t* cands, int n_cand, int chunks, char* ws,
                            float* losses, float* mean_phase, cudaStream_t s) {
    const LossPlan pl = plan_loss(N, cal.n_bf, n_cand, chunks, true);
    float* part = reinterpret_cast<float*>(ws);
    double* var = reinterpret_cast<double*>(ws + pl.part_bytes);
    if constexpr (N >= kL256) {
        const int rc = launch_two_pass<N, CHI64, false, true>(
            g_half, geom, q_row, q_col, cal, cands, n_cand, pl, nullptr, part,
            ws + pl.part_bytes + pl.var_bytes, s);
        if (rc) return rc;
    } else {
        const size_t smem = LossSmem<N>::bytes + sizeof(float) * N * N;
        CUDA_TRY(cudaFuncSetAttribute(k_loss_full<N, CHI64>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        { k_loss_full<N, CHI64><<<dim3(pl.n_chunks, n_cand), kLossThreads, smem, s>>>(
            reinterpret_cast<const float2*>(g_half), cal.n_bf, geom, q_row, q_col, cands, cal,
            pl.bf_per_chunk, pl.n_chunks, part); note_launch(); }
        CUDA_TRY(cudaGetLastError());
    }
    { k_loss_reduce<N><<<dim3(N * N / kReducePix, n_cand), kReducePix * kReduceSlices, 0, s>>>(
        part, pl.n_chunks, cal.n_bf, var, mean_phase, 0); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    { k_loss_final<<<n_cand, 256, 0, s>>>(var, N * N / kReducePix, N * N, losses); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}

template <int N>
static int dispatch_loss_full(bool chi64, const float* g_half, const float* geom,
                              const float* q_row, const float* q_col, const qssb_calibration_t& cal,
                              const qssb_full_aberrations_t* cands, int n_cand, int chunks, char* ws,
                              float* losses, float* mean_phase, cudaStream_t s) {
    return chi64 ? launch_loss_full<N, true>(g_half, geom, q_row, q_col, cal, cands, n_cand, chunks, ws, losses, mean_phase, s)
                 : launch_loss_full<N, false>(g_half, geom, q_row, q_col, cal, cands, n_cand, chunks, ws, losses, mean_phase, s);
}

}  // namespace qssb

using namespace qssb;

extern "C" int qssb_loss_workspace_bytes(const qssb_calibration_t* cal, int32_t n_cand,
                                         int32_t flags, size_t* bytes) {
    int rc = validate_calibration(cal, "qssb_loss_workspace_bytes: null calibration");
    if (rc) return rc;
    if (!bytes || n_cand <= 0 || n_cand > 65535)
        return set_error(QSSB_ERR_INVALID, "qssb_loss_workspace_bytes: n_cand must be in [1, 65535]");
    const int n = cal->scan_rows;
    if (n != 64 && n != 128 && n != 256 && n != 512 && n != 1024)
        return set_error(QSSB_ERR_UNSUPPORTED,
                         "qssb_loss_batch: scan size must be 64, 128, 256, 512 or 1024");
    const LossPlan pl =
        plan_loss(n, cal->n_bf, n_cand, flag_chunks(flags), false, loss_queue_requested(n, flags));
    *bytes = loss_workspace(pl);
    return QSSB_OK;
}

extern "C" int qssb_loss_batch(const float* g_half, const float* bf_geom, const float* q_row,
                               const float* q_col, const qssb_calibration_t* cal,
                               const qssb_aberrations_t* candidates, int32_t n_cand, int32_t flags,
                               void* workspace, size_t workspace_bytes, float* losses,
                               float* mean_phase, void* stream) {
    return qssb_loss_batch_ex(g_half, bf_geom, q_row, q_col, cal, candidates, n_cand, flags,
                              nullptr, workspace, workspace_bytes, losses, mean_phase, stream);
}

static size_t overlap_table_elems(int n) {
    switch (n) {
        case 128: return (size_t)kNE128;
        case 256: return two_pass_table_elems<256>();
        case 512: return two_pass_table_elems<512>();
        case 1024: return two_pass_table_elems<1024>();
        default: return 0;
    }
}

extern "C" int qssb_overlap_table_bytes(const qssb_calibration_t* cal, size_t* bytes) {
    int rc = validate_calibration(cal, "qssb_overlap_table_bytes: null calibration");
    if (rc) return rc;
    if (!bytes) return set_error(QSSB_ERR_INVALID, "qssb_overlap_table_bytes: null output");
    const size_t elems = overlap_table_elems(cal->scan_rows);
    if (elems == 0 || cal->scan_cols != cal->scan_rows)
        return set_error(QSSB_ERR_UNSUPPORTED,
                         "qssb_overlap_table: square 128, 256, 512 or 1024 scans only");
    *bytes = sizeof(float2) * elems * (size_t)cal->n_bf;
    return QSSB_OK;
}

extern "C" int qssb_overlap_table(const float* bf_geom, const float* q_row, const float* q_col,
                                  const qssb_calibration_t* cal, float* table, void* stream) {
    size_t need = 0;
    int rc = qssb_overlap_table_bytes(cal, &need);
    if (rc) return rc;
    if (!bf_geom || !q_row || !q_col || !table)
        return set_error(QSSB_ERR_INVALID, "qssb_overlap_table: null pointer");
    if (cal->n_bf > 65535)
        return set_error(QSSB_ERR_UNSUPPORTED, "qssb_overlap_table: more than 65535 BF pixels");
    const Probe p = make_probe_common(*cal, 0.0f, 0.0f, 0.0f, 0.0f);
    auto* t = reinterpret_cast<float2*>(table);
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned gx = (unsigned)((overlap_table_elems(cal->scan_rows) + 255) / 256);
    switch (cal->scan_rows) {
        case 128: { k_overlap_table128<<<dim3(gx, cal->n_bf), 256, 0, st>>>(bf_geom, cal->n_bf, q_row, q_col, p, t); note_launch(); } break;
        case 256: { k_overlap_table_rows<256><<<dim3(gx, cal->n_bf), 256, 0, st>>>(bf_geom, cal->n_bf, q_row, q_col, p, t); note_launch(); } break;
        case 512: { k_overlap_table_rows<512><<<dim3(gx, cal->n_bf), 256, 0, st>>>(bf_geom, cal->n_bf, q_row, q_col, p, t); note_launch(); } break;
        default: { k_overlap_table_rows<1024><<<dim3(gx, cal->n_bf), 256, 0, st>>>(bf_geom, cal->n_bf, q_row, q_col, p, t); note_launch(); } break;
    }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}

extern "C" int qssb_loss_batch_ex(const float* g_half, const float* bf_geom, const float* q_row,
                                  const float* q_col, const qssb_calibration_t* cal,
                                  const qssb_aberrations_t* candidates, int32_t n_cand,
                                  int32_t flags, const float* overlap, void* workspace,
                                  size_t workspace_bytes, float* losses, float* mean_phase,
                                  void* stream) {
    int rc = validate_calibration(cal, "qssb_loss_batch: null calibration");
    if (rc) return rc;
    if (!g_half || !bf_geom || !q_row || !q_col || !candidates || !workspace || !losses)
        return set_error(QSSB_ERR_INVALID, "qssb_loss_batch: null pointer");
    size_t need = 0;
    rc = qssb_loss_workspace_bytes(cal, n_cand, flags, &need);
    if (rc) return rc;
    if (workspace_bytes < need)
        return set_error(QSSB_ERR_WORKSPACE, "qssb_loss_batch: workspace too small");
    if (((uintptr_t)workspace & 255u) != 0)
        return set_error(QSSB_ERR_INVALID, "qssb_loss_batch: workspace must be 256-byte aligned");
    const bool sym = !(flags & QSSB_FLAG_FULL_PLANE);
    const bool chi64 = (flags & QSSB_FLAG_CHI_FP64) != 0;
    const bool quad = (flags & QSSB_FLAG_QUADRATIC) != 0;
    if (overlap && (cal->scan_rows < 128 || cal->scan_cols != cal->scan_rows))
        return set_error(QSSB_ERR_UNSUPPORTED,
                         "qssb_loss_batch_ex: the overlap table is for square 128 .. 1024 scans");
    const float2* ov = reinterpret_cast<const float2*>(overlap);
    cudaStream_t s = (cudaStream_t)stream;
    char* ws = static_cast<char*>(workspace);
    switch (cal->scan_rows) {
        case 64: return dispatch_loss<64>(sym, chi64, quad, g_half, bf_geom, q_row, q_col, *cal, candidates, n_cand, flags, ws, losses, mean_phase, nullptr, s);
        case 128: return dispatch_loss<128>(sym, chi64, quad, g_half, bf_geom, q_row, q_col, *cal, candidates, n_cand, flags, ws, losses, mean_phase, ov, s);
        case 256: return dispatch_loss<256>(sym, chi64, quad, g_half, bf_geom, q_row, q_col, *cal, candidates, n_cand, flags, ws, losses, mean_phase, ov, s);
        case 512: return dispatch_loss<512>(sym, chi64, quad, g_half, bf_geom, q_row, q_col, *cal, candidates, n_cand, flags, ws, losses, mean_phase, ov, s);
        case 1024: return dispatch_loss<1024>(sym, chi64, quad, g_half, bf_geom, q_row, q_col, *cal, candidates, n_cand, flags, ws, losses, mean_phase, ov, s);
        default: return set_error(QSSB_ERR_UNSUPPORTED,
                                  "qssb_loss_batch: scan size must be 64, 128, 256, 512 or 1024");
    }
}

extern "C" int qssb_loss_full_workspace_bytes(const qssb_calibration_t* cal, int32_t n_cand,
                                              int32_t flags, size_t* bytes) {
    int rc = validate_calibration(cal, "qssb_loss_full_workspace_bytes: null calibration");
    if (rc) return rc;
    if (!bytes || n_cand <= 0 || n_cand > 65535)
        return set_error(QSSB_ERR_INVALID, "qssb_loss_full_workspace_bytes: n_cand must be in [1, 65535]");
    const int n = cal->scan_rows;
    if (n != 64 && n != 128 && n != 256 && n != 512 && n != 1024)
        return set_error(QSSB_ERR_UNSUPPORTED,
                         "qssb_loss_batch_full: scan size must be 64, 128, 256, 512 or 1024");
    const LossPlan pl = plan_loss(n, cal->n_bf, n_cand, flag_chunks(flags), true);
    *bytes = loss_workspace(pl);
    return QSSB_OK;
}

extern "C" int qssb_loss_batch_full(const float* g_half, const float* bf_geom, const float* q_row,
                                    const float* q_col, const qssb_calibration_t* cal,
                                    const qssb_full_aberrations_t* candidates, int32_t n_cand,
                                    int32_t flags, void* workspace, size_t workspace_bytes,
                                    float* losses, float* mean_phase, void* stream) {
    int rc = validate_calibration(cal, "qssb_loss_batch_full: null calibration");
    if (rc) return rc;
    if (!g_half || !bf_geom || !q_row || !q_col || !candidates || !workspace || !losses)
        return set_error(QSSB_ERR_INVALID, "qssb_loss_batch_full: null pointer");
    size_t need = 0;
    rc = qssb_loss_full_workspace_bytes(cal, n_cand, flags, &need);
    if (rc) return rc;
    if (workspace_bytes < need)
        return set_error(QSSB_ERR_WORKSPACE, "qssb_loss_batch_full: workspace too small");
    if (((uintptr_t)workspace & 255u) != 0)
        return set_error(QSSB_ERR_INVALID, "qssb_loss_batch_full: workspace must be 256-byte aligned");
    const bool chi64 = (flags & QSSB_FLAG_CHI_FP64) != 0;
    const int chunks = flag_chunks(flags);
    cudaStream_t s = (cudaStream_t)stream;
    char* ws = static_cast<char*>(workspace);
    switch (cal->scan_rows) {
        case 64: return dispatch_loss_full<64>(chi64, g_half, bf_geom, q_row, q_col, *cal, candidates, n_cand, chunks, ws, losses, mean_phase, s);
        case 128: return dispatch_loss_full<128>(chi64, g_half, bf_geom, q_row, q_col, *cal, candidates, n_cand, chunks, ws, losses, mean_phase, s);
        case 256: return dispatch_loss_full<256>(chi64, g_half, bf_geom, q_row, q_col, *cal, candidates, n_cand, chunks, ws, losses, mean_phase, s);
        case 512: return dispatch_loss_full<512>(chi64, g_half, bf_geom, q_row, q_col, *cal, candidates, n_cand, chunks, ws, losses, mean_phase, s);
        case 1024: return dispatch_loss_full<1024>(chi64, g_half, bf_geom, q_row, q_col, *cal, candidates, n_cand, chunks, ws, losses, mean_phase, s);
        default: return set_error(QSSB_ERR_UNSUPPORTED,
                                  "qssb_loss_batch_full: scan size must be 64, 128, 256, 512 or 1024");
    }
}

namespace qssb {
__global__ void k_phase_atan2(const float* __restrict__ y, const float* __restrict__ x,
                              float* __restrict__ out, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = phase_atan2(__ldg(y + i), __ldg(x + i));
}
}  // namespace qssb

extern "C" int qssb_phase_atan2(const float* y, const float* x, float* out, int64_t n,
                                void* stream) {
    if (n < 0 || (n > 0 && (!y || !x || !out)))
        return set_error(QSSB_ERR_INVALID, "qssb_phase_atan2: null pointer or negative size");
    if (n == 0) return QSSB_OK;
    long long blocks = (n + 255) / 256;
    const long long cap = 8LL * device_sm_count();
    if (blocks > cap) blocks = cap;
    { k_phase_atan2<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(y, x, out, n); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}

extern "C" int qssb_set_cancel(const int32_t* flag) {
    g_cancel_flag = flag;
    return QSSB_OK;
}
