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
                const float ph = atan2f(v.y, v.x);
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
        // A) rows 0..64 and the lower Nyquist column
        for (int e = tid; e < 65 * N + 63; e += 512) {
            int r, c;
            if (e < 65 * N) {
                r = e >> 7;
                c = e & 127;
            } else {
                r = N - 1 - (e - 65 * N);  // 127 .. 65
                c = 64;
            }
            const float2 gv = c <= 64 ? __ldg(gb + r * H + c)
                                      : cconj(__ldg(gb + ((N - r) & (N - 1)) * H + (N - c)));
            float2 v;
            if constexpr (kSep) {
                const float2 lo = make_float2(kq.kx_lo, kq.ky_lo);
                v = corrected_quad_e(__ldg(q_row + r), __ldg(q_col + c), r, c,
                                     __ldg(eqc + r * N + c), kq.kx, kq.ky, kq.ak, &lo,
                                     cmul(s_phr[r], s_phc[c]), gv, p);
            } else if constexpr (QUAD) {
                v = corrected_quad<CHI64>(__ldg(q_row + r), __ldg(q_col + c), r, c,
                                          __ldg(eqc + r * N + c), kq, gv, p);
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
                const float ph = atan2f(v[t].y, v[t].x);
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

// ------------------------------------------------------------- N = 256
// The 256^2 half plane (264 KB) does not fit shared memory. Per BF pixel:
//   rows: each warp evaluates C on rows 0..128 one line at a time in its own
//     shared line (the value C(r, 128) saved first), inverse-FFTs the line
//     and writes it to the CTA's staging plane in global memory (L2);
//     C(-r', 128), r' = 1..127, is evaluated directly;
//   columns: after a barrier each warp rebuilds its columns from the staging
//     plane (rows 129..255 by row(-r) = -conj(row(r)) + (-1)^x delta_r,
//     delta_r = conj C(r, 128) + C(-r, 128)), inverse-FFTs them and adds
//     phi and phi^2 to the CTA's own partial planes, stored column-major
//     (x * N + y): every element belongs to one lane, so no atomics.
// The same scheme serves 512^2 and 1024^2 (N/2 + 1 evaluated rows).
constexpr int kL256 = 256;

template <int N>
struct LossStagedSmem {
    static constexpr int rows = N / 2 + 1;
    static constexpr size_t lines = sizeof(float2) * kLossWarps * N;
    static constexpr size_t misc = sizeof(float2) * (N + 3 * (N / 2));  // tw, cpos, cneg, delta
    static constexpr size_t bytes = lines + misc;
    static constexpr size_t stage_per_cta = sizeof(float2) * rows * N;
};

static size_t staged_stage_per_cta(int n) {
    switch (n) {
        case 256: return LossStagedSmem<256>::stage_per_cta;
        case 512: return LossStagedSmem<512>::stage_per_cta;
        case 1024: return LossStagedSmem<1024>::stage_per_cta;
        default: return 0;
    }
}

template <int N, bool CHI64, bool QUAD>
__global__ void __launch_bounds__(kLossThreads, 1) k_loss_staged(
    const float2* __restrict__ g, int n_bf, const float* __restrict__ geom,
    const float* __restrict__ q_row, const float* __restrict__ q_col,
    const qssb_aberrations_t* __restrict__ cands, qssb_calibration_t cal,
    const float2* __restrict__ eq_table, int bf_per_chunk, int n_chunks, float* __restrict__ part,
    float2* __restrict__ stage) {
    constexpr int H = N / 2 + 1;
    constexpr int kRows = LossStagedSmem<N>::rows;
    constexpr bool kSep = QUAD && !CHI64;
    extern __shared__ float4 smem4[];
    float2* lines = reinterpret_cast<float2*>(smem4);
    float2* tw = lines + kLossWarps * N;
    float2* cpos = tw + N;
    float2* cneg = cpos + N / 2;
    float2* delta = cneg + N / 2;
    __shared__ Probe sp;
    __shared__ float2 s_phr[kSep ? N : 1];
    __shared__ float2 s_phc[kSep ? N : 1];
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int chunk = blockIdx.x;
    const int cand = blockIdx.y;
    const size_t cta = (size_t)cand * n_chunks + chunk;
    float2* S = stage + cta * (size_t)kRows * N;
    float* ps = part + cta * 2 * (size_t)N * N;
    float* pq = ps + (size_t)N * N;
    float2* line = lines + warp * N;
    if (tid == 0) {
        const qssb_aberrations_t ab = cands[cand];
        sp = make_probe_common(cal, ab.C10, ab.C12, ab.phi12, ab.C30);
    }
    fill_twiddles<N>(tw, tid, kLossThreads);
    // this lane's accumulator elements: columns warp + 16 j, rows lane + 32 t
    for (int j = 0; j < N / kLossWarps; ++j) {
        const int x = warp + kLossWarps * j;
#pragma unroll
        for (int t = 0; t < N / 32; ++t) {
            ps[(size_t)x * N + lane + 32 * t] = 0.0f;
            pq[(size_t)x * N + lane + 32 * t] = 0.0f;
        }
    }
    __syncthreads();
    const Probe& p = sp;
    const float2* eqc = eq_table + (size_t)cand * N * N;
    auto fill_phase = [&](int b) {  // e^{i 2 q_row(r) u}, e^{i 2 q_col(c) v}
        const float kx = __ldg(geom + b);
        const float ky = __ldg(geom + n_bf + b);
        float sn, cs;
        for (int i = tid; i < 2 * N; i += kLossThreads) {
            if (i < N) {
                sincosf(2.0f * __ldg(q_row + i) * fmaf(p.mxx, kx, p.mxy * ky), &sn, &cs);
                s_phr[i] = make_float2(cs, sn);
            } else {
                sincosf(2.0f * __ldg(q_col + i - N) * fmaf(p.mxy, kx, p.myy * ky), &sn, &cs);
                s_phc[i - N] = make_float2(cs, sn);
            }
        }
    };
    const int b0 = chunk * bf_per_chunk;
    int nb = n_bf - b0;
    if (nb > bf_per_chunk) nb = bf_per_chunk;
    const float2 dc = make_float2((float)cal.dc_re, (float)cal.dc_im);
    if constexpr (kSep) {
        if (nb > 0) fill_phase(b0);
        __syncthreads();
    }
    auto eval = [&](int b, const BFQuad& kq, const float2& pk, int r, int c) -> float2 {
        const float2* gb = g + (size_t)b * N * H;
        const float2 gv = c <= N / 2 ? __ldg(gb + r * H + c)
                                     : cconj(__ldg(gb + ((N - r) & (N - 1)) * H + (N - c)));
        if constexpr (kSep) {
            const float2 lo = make_float2(kq.kx_lo, kq.ky_lo);
            return corrected_quad_e(__ldg(q_row + r), __ldg(q_col + c), r, c, __ldg(eqc + r * N + c),
                                    kq.kx, kq.ky, kq.ak, &lo, cmul(s_phr[r], s_phc[c]), gv, p);
        } else if constexpr (QUAD) {
            return corrected_quad<CHI64>(__ldg(q_row + r), __ldg(q_col + c), r, c,
                                         __ldg(eqc + r * N + c), kq, gv, p);
        } else {
            return corrected<CHI64>(__ldg(q_row + r), __ldg(q_col + c), r, c, kq.kx, kq.ky,
                                    kq.kx_lo, kq.ky_lo, pk, gv, p);
        }
    };
    for (int i = 0; i < nb; ++i) {
        const int b = b0 + i;
        const BFQuad kq = bf_quad(geom, n_bf, b, p);
        float2 pk = make_float2(0.0f, 0.0f);
        if constexpr (!QUAD)
            pk = probe_at_bf<CHI64>(__ldg(geom + 2 * n_bf + b), __ldg(geom + 3 * n_bf + b),
                                    __ldg(geom + 4 * n_bf + b), __ldg(geom + 5 * n_bf + b), p);
        // C(-r', N/2) for r' = 1..N/2-1 (row N - r')
        for (int j = tid; j < N / 2; j += kLossThreads)
            if (j >= 1) cneg[j] = eval(b, kq, pk, N - j, N / 2);
        // rows 0..N/2: evaluate, keep C(r, N/2), inverse FFT, stage
        for (int r = warp; r < kRows; r += kLossWarps) {
#pragma unroll
            for (int t = 0; t < N / 32; ++t) {
                const int c = lane + 32 * t;
                float2 v = (r == 0 && c == 0) ? dc : eval(b, kq, pk, r, c);
                if (c == N / 2 && r >= 1 && r < N / 2) cpos[r] = v;
                line[c] = v;
            }
            __syncwarp();
            line_fft<N, +1>(line, 1, tw, lane);
#pragma unroll
            for (int t = 0; t < N / 32; ++t) S[(size_t)r * N + lane + 32 * t] = line[lane + 32 * t];
            __syncwarp();
        }
        __syncthreads();
        for (int j = tid; j < N / 2; j += kLossThreads)
            if (j >= 1) delta[j] = cadd(cconj(cpos[j]), cneg[j]);
        __syncthreads();
        // columns
        for (int j = 0; j < N / kLossWarps; ++j) {
            const int x = warp + kLossWarps * j;
            const float sign = (x & 1) ? -1.0f : 1.0f;
#pragma unroll
            for (int t = 0; t < N / 32; ++t) {
                const int r = lane + 32 * t;
                float2 v;
                if (r < kRows) {
                    v = S[(size_t)r * N + x];
                } else {
                    const float2 m = S[(size_t)(N - r) * N + x];
                    const float2 d = delta[N - r];
                    v = make_float2(fmaf(sign, d.x, -m.x), fmaf(sign, d.y, m.y));
                }
                line[r] = v;
            }
            __syncwarp();
            line_fft<N, +1>(line, 1, tw, lane);
#pragma unroll
            for (int t = 0; t < N / 32; ++t) {
                const int y = lane + 32 * t;
                const float2 v = line[y];
                const float ph = atan2f(v.y, v.x);
                ps[(size_t)x * N + y] += ph;
                pq[(size_t)x * N + y] = fmaf(ph, ph, pq[(size_t)x * N + y]);
            }
            __syncwarp();
        }
        if constexpr (kSep) {
            if (i + 1 < nb) fill_phase(b + 1);
        }
        __syncthreads();
    }
}

template <int N>
__global__ void k_loss_reduce(const float* __restrict__ part, int n_chunks, int n_bf,
                              double* __restrict__ var, float* __restrict__ mean_phase,
                              int row_major) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;  // col * N + row, or row * N + col
    const int cand = blockIdx.y;
    if (j >= N * N) return;
    double s1 = 0.0, s2 = 0.0;
    for (int k = 0; k < n_chunks; ++k) {
        const float* base = part + ((size_t)(cand * n_chunks + k) * 2) * N * N;
        s1 += (double)base[j];
        s2 += (double)base[(size_t)N * N + j];
    }
    const double inv_b = 1.0 / (double)n_bf;
    const double mean = s1 * inv_b;
    var[(size_t)cand * N * N + j] = s2 * inv_b - mean * mean;
    if (mean_phase) {
        const int hi = j / N;
        const int lo = j - hi * N;
        mean_phase[(size_t)cand * N * N + (row_major ? j : lo * N + hi)] = (float)mean;
    }
}

__global__ void __launch_bounds__(256) k_loss_final(const double* __restrict__ var, int npos,
                                                    float* __restrict__ losses) {
    __shared__ double red[256];
    const int cand = blockIdx.x;
    const double* v = var + (size_t)cand * npos;
    double acc = 0.0;
    for (int i = threadIdx.x; i < npos; i += 256) acc += v[i];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) losses[cand] = (float)(red[0] / (double)npos);
}

struct LossPlan {
    int bf_per_chunk;
    int n_chunks;
    size_t part_bytes;
    size_t var_bytes;
    size_t eq_bytes;
    size_t stage_bytes;  // N = 256: one staging half plane per CTA
};

// Deterministic: about 296 CTAs in total (two per B200 SM), at least one BF
// pixel each.
static LossPlan plan_loss(int n, int n_bf, int n_cand, int chunks_req = 0) {
    LossPlan pl;
    int chunks = chunks_req > 0 ? chunks_req : (296 + n_cand - 1) / n_cand;
    if (chunks < 1) chunks = 1;
    if (chunks > n_bf) chunks = n_bf;
    pl.bf_per_chunk = (n_bf + chunks - 1) / chunks;
    pl.n_chunks = (n_bf + pl.bf_per_chunk - 1) / pl.bf_per_chunk;
    pl.part_bytes = sizeof(float) * 2 * (size_t)n * n * pl.n_chunks * n_cand;
    pl.part_bytes = (pl.part_bytes + 255) & ~(size_t)255;
    pl.var_bytes = sizeof(double) * (size_t)n * n * n_cand;
    pl.eq_bytes = sizeof(float2) * (size_t)n * n * n_cand;
    pl.stage_bytes = staged_stage_per_cta(n) * (size_t)pl.n_chunks * n_cand;
    return pl;
}

template <int N, bool SYM, bool CHI64, bool QUAD>
static int launch_loss(const float* g_half, const float* geom, const float* q_row,
                       const float* q_col, const qssb_calibration_t& cal,
                       const qssb_aberrations_t* cands, int n_cand, int chunks, char* ws,
                       float* losses, float* mean_phase, cudaStream_t s) {
    const LossPlan pl = plan_loss(N, cal.n_bf, n_cand, chunks);
    float* part = reinterpret_cast<float*>(ws);
    double* var = reinterpret_cast<double*>(ws + pl.part_bytes);
    float2* eq = reinterpret_cast<float2*>(ws + pl.part_bytes + pl.var_bytes);
    if (QUAD) {
        k_eq_table<N><<<dim3((N * N + 255) / 256, n_cand), 256, 0, s>>>(cands, cal, eq);
        CUDA_TRY(cudaGetLastError());
    }
    if constexpr (N >= kL256) {
        static_assert(SYM, "the staged loss evaluates the half plane");
        float2* stage = reinterpret_cast<float2*>(ws + pl.part_bytes + pl.var_bytes + pl.eq_bytes);
        const size_t smem = LossStagedSmem<N>::bytes;
        CUDA_TRY(cudaFuncSetAttribute(k_loss_staged<N, CHI64, QUAD>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_loss_staged<N, CHI64, QUAD><<<dim3(pl.n_chunks, n_cand), kLossThreads, smem, s>>>(
            reinterpret_cast<const float2*>(g_half), cal.n_bf, geom, q_row, q_col, cands, cal, eq,
            pl.bf_per_chunk, pl.n_chunks, part, stage);
    } else if constexpr (N == 128) {
        const size_t smem = Loss128Smem::bytes;
        CUDA_TRY(cudaFuncSetAttribute(k_loss_moments128<CHI64, QUAD>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_loss_moments128<CHI64, QUAD><<<dim3(pl.n_chunks, n_cand), 512, smem, s>>>(
            reinterpret_cast<const float2*>(g_half), cal.n_bf, geom, q_row, q_col, cands, cal, eq,
            pl.bf_per_chunk, pl.n_chunks, part);
    } else {
        const size_t smem = LossSmem<N>::bytes;
        CUDA_TRY(cudaFuncSetAttribute(k_loss_moments<N, SYM, CHI64, QUAD>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_loss_moments<N, SYM, CHI64, QUAD><<<dim3(pl.n_chunks, n_cand), kLossThreads, smem, s>>>(
            reinterpret_cast<const float2*>(g_half), cal.n_bf, geom, q_row, q_col, cands, cal, eq,
            pl.bf_per_chunk, pl.n_chunks, part);
    }
    CUDA_TRY(cudaGetLastError());
    k_loss_reduce<N><<<dim3((N * N + 255) / 256, n_cand), 256, 0, s>>>(part, pl.n_chunks, cal.n_bf,
                                                                       var, mean_phase, N == 128 ? 1 : 0);
    CUDA_TRY(cudaGetLastError());
    k_loss_final<<<n_cand, 256, 0, s>>>(var, N * N, losses);
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}

template <int N, bool QUAD>
static int dispatch_loss_q(bool sym, bool chi64, const float* g_half, const float* geom,
                           const float* q_row, const float* q_col, const qssb_calibration_t& cal,
                           const qssb_aberrations_t* cands, int n_cand, int chunks, char* ws,
                           float* losses, float* mean_phase, cudaStream_t s) {
    if constexpr (N >= kL256) {
        if (!sym)
            return set_error(QSSB_ERR_UNSUPPORTED,
                             "qssb_loss_batch: QSSB_FLAG_FULL_PLANE is offered up to 128^2");
        return chi64 ? launch_loss<N, true, true, QUAD>(g_half, geom, q_row, q_col, cal, cands, n_cand, chunks, ws, losses, mean_phase, s)
                     : launch_loss<N, true, false, QUAD>(g_half, geom, q_row, q_col, cal, cands, n_cand, chunks, ws, losses, mean_phase, s);
    } else {
        if (sym)
            return chi64 ? launch_loss<N, true, true, QUAD>(g_half, geom, q_row, q_col, cal, cands, n_cand, chunks, ws, losses, mean_phase, s)
                         : launch_loss<N, true, false, QUAD>(g_half, geom, q_row, q_col, cal, cands, n_cand, chunks, ws, losses, mean_phase, s);
        return chi64 ? launch_loss<N, false, true, QUAD>(g_half, geom, q_row, q_col, cal, cands, n_cand, chunks, ws, losses, mean_phase, s)
                     : launch_loss<N, false, false, QUAD>(g_half, geom, q_row, q_col, cal, cands, n_cand, chunks, ws, losses, mean_phase, s);
    }
}

// Candidates live on the device, so the path is chosen by a flag: the
// general (C30) path unless QSSB_FLAG_QUADRATIC promises C30 == 0 for all.
template <int N>
static int dispatch_loss(bool sym, bool chi64, bool quad, const float* g_half, const float* geom,
                         const float* q_row, const float* q_col, const qssb_calibration_t& cal,
                         const qssb_aberrations_t* cands, int n_cand, int chunks, char* ws,
                         float* losses, float* mean_phase, cudaStream_t s) {
    if (quad)
        return dispatch_loss_q<N, true>(sym, chi64, g_half, geom, q_row, q_col, cal, cands, n_cand, chunks, ws, losses, mean_phase, s);
    return dispatch_loss_q<N, false>(sym, chi64, g_half, geom, q_row, q_col, cal, cands, n_cand, chunks, ws, losses, mean_phase, s);
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
                const float ph = atan2f(v.y, v.x);
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
__global__ void __launch_bounds__(kLossThreads, 1) k_loss_full_staged(
    const float2* __restrict__ g, int n_bf, const float* __restrict__ geom,
    const float* __restrict__ q_row, const float* __restrict__ q_col,
    const qssb_full_aberrations_t* __restrict__ cands, qssb_calibration_t cal, int bf_per_chunk,
    int n_chunks, float* __restrict__ part, float2* __restrict__ stage) {
    constexpr int H = N / 2 + 1;
    extern __shared__ float4 smem4[];
    float2* lines = reinterpret_cast<float2*>(smem4);
    float2* tw = lines + kLossWarps * N;
    __shared__ FullConsts sh;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int chunk = blockIdx.x;
    const int cand = blockIdx.y;
    const size_t cta = (size_t)cand * n_chunks + chunk;
    float2* S = stage + cta * (size_t)N * N;
    float* ps = part + cta * 2 * (size_t)N * N;
    float* pq = ps + (size_t)N * N;
    float2* line = lines + warp * N;
    if (tid == 0) load_full_consts(sh, cands, cand, cal);
    fill_twiddles<N>(tw, tid, kLossThreads);
    for (int j = 0; j < N / kLossWarps; ++j) {
        const int x = warp + kLossWarps * j;
#pragma unroll
        for (int t = 0; t < N / 32; ++t) {
            ps[(size_t)x * N + lane + 32 * t] = 0.0f;
            pq[(size_t)x * N + lane + 32 * t] = 0.0f;
        }
    }
    __syncthreads();
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
        for (int r = warp; r < N; r += kLossWarps) {
#pragma unroll
            for (int t = 0; t < N / 32; ++t) {
                const int c = lane + 32 * t;
                const float2 gv = c <= N / 2 ? __ldg(gb + r * H + c)
                                             : cconj(__ldg(gb + ((N - r) & (N - 1)) * H + (N - c)));
                float2 v = corrected_full<CHI64>(__ldg(q_row + r), __ldg(q_col + c), r, c, kx, ky,
                                                 kx_lo, ky_lo, pk, gv, sh.p, sh.f, sh.d);
                if (r == 0 && c == 0) v = dc;
                line[c] = v;
            }
            __syncwarp();
            line_fft<N, +1>(line, 1, tw, lane);
#pragma unroll
            for (int t = 0; t < N / 32; ++t) S[(size_t)r * N + lane + 32 * t] = line[lane + 32 * t];
            __syncwarp();
        }
        __syncthreads();
        for (int j = 0; j < N / kLossWarps; ++j) {
            const int x = warp + kLossWarps * j;
#pragma unroll
            for (int t = 0; t < N / 32; ++t) line[lane + 32 * t] = S[(size_t)(lane + 32 * t) * N + x];
            __syncwarp();
            line_fft<N, +1>(line, 1, tw, lane);
#pragma unroll
            for (int t = 0; t < N / 32; ++t) {
                const int y = lane + 32 * t;
                const float2 v = line[y];
                const float ph = atan2f(v.y, v.x);
                ps[(size_t)x * N + y] += ph;
                pq[(size_t)x * N + y] = fmaf(ph, ph, pq[(size_t)x * N + y]);
            }
            __syncwarp();
        }
        __syncthreads();
    }
}

static size_t full_stage_bytes(int n, const LossPlan& pl, int n_cand) {
    return n >= kL256 ? sizeof(float2) * (size_t)n * n * pl.n_chunks * n_cand : 0;
}

template <int N, bool CHI64>
static int launch_loss_full(const float* g_half, const float* geom, const float* q_row,
                            const float* q_col, const qssb_calibration_t& cal,
                            const qssb_full_aberrations_t* cands, int n_cand, int chunks, char* ws,
                            float* losses, float* mean_phase, cudaStream_t s) {
    const LossPlan pl = plan_loss(N, cal.n_bf, n_cand, chunks);
    float* part = reinterpret_cast<float*>(ws);
    double* var = reinterpret_cast<double*>(ws + pl.part_bytes);
    const auto* gh = reinterpret_cast<const float2*>(g_half);
    if constexpr (N >= kL256) {
        float2* stage = reinterpret_cast<float2*>(ws + pl.part_bytes + pl.var_bytes);
        const size_t smem = sizeof(float2) * (kLossWarps * N + N);
        CUDA_TRY(cudaFuncSetAttribute(k_loss_full_staged<N, CHI64>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_loss_full_staged<N, CHI64><<<dim3(pl.n_chunks, n_cand), kLossThreads, smem, s>>>(
            gh, cal.n_bf, geom, q_row, q_col, cands, cal, pl.bf_per_chunk, pl.n_chunks, part, stage);
    } else {
        const size_t smem = LossSmem<N>::bytes + sizeof(float) * N * N;
        CUDA_TRY(cudaFuncSetAttribute(k_loss_full<N, CHI64>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_loss_full<N, CHI64><<<dim3(pl.n_chunks, n_cand), kLossThreads, smem, s>>>(
            gh, cal.n_bf, geom, q_row, q_col, cands, cal, pl.bf_per_chunk, pl.n_chunks, part);
    }
    CUDA_TRY(cudaGetLastError());
    k_loss_reduce<N><<<dim3((N * N + 255) / 256, n_cand), 256, 0, s>>>(part, pl.n_chunks, cal.n_bf,
                                                                       var, mean_phase, 0);
    CUDA_TRY(cudaGetLastError());
    k_loss_final<<<n_cand, 256, 0, s>>>(var, N * N, losses);
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
    const LossPlan pl = plan_loss(n, cal->n_bf, n_cand, flag_chunks(flags));
    *bytes = pl.part_bytes + pl.var_bytes + pl.eq_bytes + pl.stage_bytes;
    return QSSB_OK;
}

extern "C" int qssb_loss_batch(const float* g_half, const float* bf_geom, const float* q_row,
                               const float* q_col, const qssb_calibration_t* cal,
                               const qssb_aberrations_t* candidates, int32_t n_cand, int32_t flags,
                               void* workspace, size_t workspace_bytes, float* losses,
                               float* mean_phase, void* stream) {
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
    const int chunks = flag_chunks(flags);
    cudaStream_t s = (cudaStream_t)stream;
    char* ws = static_cast<char*>(workspace);
    switch (cal->scan_rows) {
        case 64: return dispatch_loss<64>(sym, chi64, quad, g_half, bf_geom, q_row, q_col, *cal, candidates, n_cand, chunks, ws, losses, mean_phase, s);
        case 128: return dispatch_loss<128>(sym, chi64, quad, g_half, bf_geom, q_row, q_col, *cal, candidates, n_cand, chunks, ws, losses, mean_phase, s);
        case 256: return dispatch_loss<256>(sym, chi64, quad, g_half, bf_geom, q_row, q_col, *cal, candidates, n_cand, chunks, ws, losses, mean_phase, s);
        case 512: return dispatch_loss<512>(sym, chi64, quad, g_half, bf_geom, q_row, q_col, *cal, candidates, n_cand, chunks, ws, losses, mean_phase, s);
        case 1024: return dispatch_loss<1024>(sym, chi64, quad, g_half, bf_geom, q_row, q_col, *cal, candidates, n_cand, chunks, ws, losses, mean_phase, s);
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
    const LossPlan pl = plan_loss(n, cal->n_bf, n_cand, flag_chunks(flags));
    *bytes = pl.part_bytes + pl.var_bytes + full_stage_bytes(n, pl, n_cand);
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
