// qssb_object.cu - SSB object wave by the corrected Fourier ("trotter") sum.
//
// O = ifft2((1/B) sum_b C_b), C_b(q) = G_b(q) conj(Gamma_hat_b(q)), DC := dc.
// By IFFT linearity this equals the reference's per-BF path
// (ifft2 of every C_b, then mean over b; engine.py:1109-1151) and its
// Fourier-sum path (engine.py:1047-1107), but runs no per-BF inverse FFT.
//
// +-q symmetry: for aberrations whose chi is even in u (C10, C12, C30 - the
// only ones this entry point takes) and the point-symmetric soft aperture,
// P(-u) = P(u), hence Gamma_b(-q) = -conj(Gamma_b(q)) bit for bit, and with
// G_b(-q) = conj(G_b(q)) (real scan images) C_b(-q) = -conj(C_b(q)). The
// frequencies computed are the stored half plane (all rows, columns 0..N/2)
// plus the Nyquist row's remaining columns (whose mirror frequency +N/2 is not
// on the fftfreq grid); the rest is filled by the mirror relation after the
// sum. That is N(N/2+1) + N/2 - 1 of the N^2 overlap evaluations.
//
// Kernels: k_trotter_partial (per BF chunk, Kahan-compensated FP32 sums per
// frequency) -> k_trotter_plane (fixed-order FP64 fold of the chunks, mirror
// fill, DC, 1/B) -> k_ifft_rows -> k_ifft_cols_phase (1/N^2, atan2).
#include <math.h>

#include <mutex>

#include "qssb_internal.h"

namespace qssb {

constexpr int kMaxBfChunk = 256;
constexpr int kTrotterThreads = 256;

struct QMap {
    int r, c, gr, gc;  // scan-frequency (r, c); stored half-plane element (gr, gc)
    bool conj;         // load conj(G[gr][gc])
};

// Index -> frequency for the evaluated set.
template <int N, bool SYM>
__device__ __forceinline__ QMap qmap(int qi) {
    constexpr int H = N / 2 + 1;
    QMap m;
    if constexpr (SYM) {
        if (qi < N * H) {
            m.r = qi / H;
            m.c = qi - m.r * H;
            m.gr = m.r;
            m.gc = m.c;
            m.conj = false;
        } else {
            m.r = N / 2;
            m.c = H + (qi - N * H);
            m.gr = N / 2;
            m.gc = N - m.c;
            m.conj = true;
        }
    } else {
        m.r = qi / N;
        m.c = qi - m.r * N;
        if (m.c <= N / 2) {
            m.gr = m.r;
            m.gc = m.c;
            m.conj = false;
        } else {
            m.gr = (N - m.r) & (N - 1);
            m.gc = N - m.c;
            m.conj = true;
        }
    }
    return m;
}

template <int N, bool SYM>
__host__ __device__ constexpr int n_eval_q() {
    return SYM ? N * (N / 2 + 1) + N / 2 - 1 : N * N;
}

template <int N, bool SYM, bool CHI64, bool QUAD>
__global__ void __launch_bounds__(kTrotterThreads) k_trotter_partial(
    const float2* __restrict__ g, int n_bf, const float* __restrict__ geom,
    const float* __restrict__ q_row, const float* __restrict__ q_col, Probe p, int bf_per_chunk,
    float2* __restrict__ partial) {
    constexpr int H = N / 2 + 1;
    constexpr int NQ = n_eval_q<N, SYM>();
    __shared__ BFQuad s_bf[kMaxBfChunk];
    __shared__ float2 s_pk[QUAD ? 1 : kMaxBfChunk];
    const int tid = threadIdx.x;
    const int chunk = blockIdx.y;
    const int b0 = chunk * bf_per_chunk;
    int nb = n_bf - b0;
    if (nb > bf_per_chunk) nb = bf_per_chunk;
    for (int i = tid; i < nb; i += kTrotterThreads) {
        const int b = b0 + i;
        s_bf[i] = bf_quad(geom, n_bf, b, p);
        if constexpr (!QUAD)
            s_pk[i] = probe_at_bf<CHI64>(__ldg(geom + 2 * n_bf + b), __ldg(geom + 3 * n_bf + b),
                                         __ldg(geom + 4 * n_bf + b), __ldg(geom + 5 * n_bf + b), p);
    }
    __syncthreads();
    const int qi = blockIdx.x * kTrotterThreads + tid;
    if (qi >= NQ) return;
    const QMap m = qmap<N, SYM>(qi);
    const float qx = __ldg(q_row + m.r);
    const float qy = __ldg(q_col + m.c);
    const float2 eq = QUAD ? eq_value(m.r, m.c, p) : make_float2(1.0f, 0.0f);
    const float2* gp = g + (size_t)b0 * N * H + m.gr * H + m.gc;
    float sr = 0.f, si = 0.f, er = 0.f, ei = 0.f;  // Kahan sums and compensations
#pragma unroll 2
    for (int i = 0; i < nb; ++i) {
        float2 gv = __ldg(gp + (size_t)i * N * H);
        if (m.conj) gv.y = -gv.y;
        float2 v;
        if constexpr (QUAD) {
            v = corrected_quad<CHI64>(qx, qy, m.r, m.c, eq, s_bf[i], gv, p);
        } else {
            const BFQuad& k = s_bf[i];
            v = corrected<CHI64>(qx, qy, m.r, m.c, k.kx, k.ky, k.kx_lo, k.ky_lo, s_pk[i], gv, p);
        }
        const float yr = v.x - er;
        const float tr = sr + yr;
        er = (tr - sr) - yr;
        sr = tr;
        const float yi = v.y - ei;
        const float ti = si + yi;
        ei = (ti - si) - yi;
        si = ti;
    }
    partial[(size_t)chunk * NQ + qi] = make_float2(sr, si);
}

// The C10/C12 (quadratic chi, FP32) path with Q adjacent frequencies per
// thread (the tile shape the autotuner picks: 2, 4 - the default - or 8).
// theta = 2 q^T M k is linear in q, so along a row of the stored half plane
// e^{i theta} advances by the per-BF factor w = e^{i 2 dq v}: one sincos per Q
// overlap evaluations. Threads t < N * N/(2Q) take (r, Qj .. Qj+Q-1) of
// columns 0..N/2-1; the rest take column N/2 of every row and the Nyquist
// row's columns N/2+1..N-1 one at a time. The partial layout is the same as
// k_trotter_partial's.
struct BFRow {
    float4 a;  // kx, ky, u, v   with (u, v) = M k
    float4 b;  // A(k), w.x, w.y, unused
};

template <int N, int Q = 4>
__global__ void __launch_bounds__(kTrotterThreads) k_trotter_quad4(
    const float2* __restrict__ g, int n_bf, const float* __restrict__ geom,
    const float* __restrict__ q_row, const float* __restrict__ q_col, Probe p, int bf_per_chunk,
    float2* __restrict__ partial) {
    static_assert(Q == 2 || Q == 4 || Q == 8, "2, 4 or 8 frequencies per thread");
    constexpr int H = N / 2 + 1;
    constexpr int NQ = n_eval_q<N, true>();
    constexpr int GPR = N / (2 * Q);  // groups of Q per row
    constexpr int NG = N * GPR;
    constexpr int NT = N + N / 2 - 1;
    __shared__ BFRow s_bf[kMaxBfChunk];
    __shared__ float2 s_lo[kMaxBfChunk];
    const int tid = threadIdx.x;
    const int chunk = blockIdx.y;
    const int b0 = chunk * bf_per_chunk;
    int nb = n_bf - b0;
    if (nb > bf_per_chunk) nb = bf_per_chunk;
    const float dq = __ldg(q_col + 1);  // fftfreq step 1 / (N d)
    for (int i = tid; i < nb; i += kTrotterThreads) {
        const int b = b0 + i;
        const float kx = __ldg(geom + b);
        const float ky = __ldg(geom + n_bf + b);
        const float u = fmaf(p.mxx, kx, p.mxy * ky);
        const float v = fmaf(p.mxy, kx, p.myy * ky);
        float sw, cw;
        sincosf(2.0f * dq * v, &sw, &cw);
        s_bf[i].a = make_float4(kx, ky, u, v);
        s_bf[i].b = make_float4(__ldg(geom + 5 * n_bf + b), cw, sw, 0.0f);
        s_lo[i] = make_float2(__ldg(geom + 6 * n_bf + b), __ldg(geom + 7 * n_bf + b));
    }
    __syncthreads();
    const int t = blockIdx.x * kTrotterThreads + tid;
    if (t < NG) {
        const int r = t / GPR;
        const int c0 = Q * (t - r * GPR);
        const float qx = __ldg(q_row + r);
        float qy[Q];
        float2 eq[Q];
#pragma unroll
        for (int j = 0; j < Q; ++j) {
            qy[j] = __ldg(q_col + c0 + j);
            eq[j] = eq_value(r, c0 + j, p);
        }
        const float2* gp = g + (size_t)b0 * N * H + r * H + c0;
        float4 acc[Q];
        float2 gc[Q];
#pragma unroll
        for (int j = 0; j < Q; ++j) {
            acc[j] = make_float4(0.f, 0.f, 0.f, 0.f);
            gc[j] = nb > 0 ? __ldg(gp + j) : make_float2(0.f, 0.f);
        }
        for (int i = 0; i < nb; ++i) {
            float2 gn[Q];
            const bool more = i + 1 < nb;
#pragma unroll
            for (int j = 0; j < Q; ++j)
                gn[j] = more ? __ldg(gp + (size_t)(i + 1) * N * H + j) : make_float2(0.f, 0.f);
            const float4 a = s_bf[i].a;
            const float4 bb = s_bf[i].b;
            float st, ct;
            __sincosf(2.0f * fmaf(qx, a.z, qy[0] * a.w), &st, &ct);
            float2 e = make_float2(ct, st);
            const float2 w = make_float2(bb.y, bb.z);
#pragma unroll
            for (int j = 0; j < Q; ++j) {
                const float2 v = corrected_quad_e(qx, qy[j], r, c0 + j, eq[j], a.x, a.y, bb.x,
                                                  &s_lo[i], e, gc[j], p);
                kahan_add(acc[j], v);
                if (j < Q - 1) e = cmul(e, w);
            }
#pragma unroll
            for (int j = 0; j < Q; ++j) gc[j] = gn[j];
        }
        float2* out = partial + (size_t)chunk * NQ + r * H + c0;
#pragma unroll
        for (int j = 0; j < Q; ++j) out[j] = make_float2(acc[j].x, acc[j].y);
    } else if (t < NG + NT) {
        const int tt = t - NG;
        int r, c, gr, gcol, qi;
        bool cj;
        if (tt < N) {
            r = tt; c = N / 2; gr = r; gcol = c; cj = false; qi = r * H + c;
        } else {
            r = N / 2; c = H + (tt - N); gr = N / 2; gcol = N - c; cj = true; qi = N * H + (tt - N);
        }
        const float qx = __ldg(q_row + r);
        const float qy = __ldg(q_col + c);
        const float2 eq = eq_value(r, c, p);
        const float2* gp = g + (size_t)b0 * N * H + gr * H + gcol;
        float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int i = 0; i < nb; ++i) {
            float2 gv = __ldg(gp + (size_t)i * N * H);
            if (cj) gv.y = -gv.y;
            const float4 a = s_bf[i].a;
            float st, ct;
            __sincosf(2.0f * fmaf(qx, a.z, qy * a.w), &st, &ct);
            const float2 v = corrected_quad_e(qx, qy, r, c, eq, a.x, a.y, s_bf[i].b.x, &s_lo[i],
                                              make_float2(ct, st), gv, p);
            kahan_add(acc, v);
        }
        partial[(size_t)chunk * NQ + qi] = make_float2(acc.x, acc.y);
    }
}

template <int N, int Q = 4>
__host__ __device__ constexpr int quad4_threads() {
    return N * (N / (2 * Q)) + N + N / 2 - 1;
}

// Full N x N corrected-mean plane from the chunk partials. A block takes 32
// frequencies; its 8 warps fold every 8th chunk each in FP64 and the 8 slice
// sums are added in a fixed order: deterministic for a given plan.
constexpr int kFoldSlices = 8;

template <int N, bool SYM>
__global__ void __launch_bounds__(32 * kFoldSlices) k_trotter_plane(
    const float2* __restrict__ partial, int n_chunks, int n_bf, float2 dc,
    const double* __restrict__ dc_dev, float2* __restrict__ plane) {
    constexpr int H = N / 2 + 1;
    constexpr int NQ = n_eval_q<N, SYM>();
    __shared__ double2 red[kFoldSlices][32];
    const int ql = threadIdx.x & 31;
    const int sl = threadIdx.x >> 5;
    const int idx = blockIdx.x * 32 + ql;
    const bool valid = idx < N * N;
    const int r = idx / N;
    const int c = idx - r * N;
    int qi = idx;
    bool mirror = false;
    if constexpr (SYM) {
        if (c <= N / 2) {
            qi = r * H + c;
        } else if (r == N / 2) {
            qi = N * H + (c - H);
        } else {
            qi = ((N - r) & (N - 1)) * H + (N - c);
            mirror = true;
        }
    }
    double sr = 0.0, si = 0.0;
    if (valid) {
#pragma unroll 4
        for (int k = sl; k < n_chunks; k += kFoldSlices) {
            const float2 v = __ldg(partial + (size_t)k * NQ + qi);
            sr += (double)v.x;
            si += (double)v.y;
        }
    }
    red[sl][ql] = make_double2(sr, si);
    __syncthreads();
    if (sl != 0 || !valid) return;
    double tr = 0.0, ti = 0.0;
#pragma unroll
    for (int j = 0; j < kFoldSlices; ++j) {
        tr += red[j][ql].x;
        ti += red[j][ql].y;
    }
    const double inv_b = 1.0 / (double)n_bf;
    // S(-q) = -conj(S(q)): real part flips, imaginary part stays
    float2 out = make_float2((float)((mirror ? -tr : tr) * inv_b), (float)(ti * inv_b));
    if (r == 0 && c == 0) out = dc_dev ? make_float2((float)dc_dev[0], (float)dc_dev[1]) : dc;
    plane[idx] = out;
}

// Lines (warps) per block of the plane IFFTs: 8, or 4 at 1024 (static
// shared memory stays under 48 KB).
template <int N>
__host__ __device__ constexpr int ifft_lines() { return N >= 1024 ? 4 : 8; }

// In-place inverse FFT of every row of a N x N plane (one warp per row).
template <int N>
__global__ void __launch_bounds__(32 * ifft_lines<N>()) k_ifft_rows(float2* __restrict__ plane) {
    constexpr int W = ifft_lines<N>();
    __shared__ float2 tw[N];
    __shared__ float2 line[W][N];
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    fill_twiddles<N>(tw, tid, 32 * W);
    const int row = blockIdx.x * W + warp;
    __syncthreads();
    if (row >= N) return;
    float2* src = plane + (size_t)row * N;
    for (int i = lane; i < N; i += 32) line[warp][i] = src[i];
    __syncwarp();
    line_fft<N, +1>(line[warp], 1, tw, lane);
    for (int i = lane; i < N; i += 32) src[i] = line[warp][i];
}

// Inverse FFT of every column, 1/N^2, object and atan2 phase.
template <int N>
__global__ void __launch_bounds__(32 * ifft_lines<N>()) k_ifft_cols_phase(
    const float2* __restrict__ plane, float2* __restrict__ object, float* __restrict__ phase) {
    constexpr int W = ifft_lines<N>();
    __shared__ float2 tw[N];
    __shared__ float2 line[W][N];
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    fill_twiddles<N>(tw, tid, 32 * W);
    const int col = blockIdx.x * W + warp;
    __syncthreads();
    if (col >= N) return;
    for (int i = lane; i < N; i += 32) line[warp][i] = plane[(size_t)i * N + col];
    __syncwarp();
    line_fft<N, +1>(line[warp], 1, tw, lane);
    const float scale = 1.0f / (float)(N * N);
    for (int i = lane; i < N; i += 32) {
        float2 v = line[warp][i];
        v.x *= scale;
        v.y *= scale;
        object[(size_t)i * N + col] = v;
        if (phase) phase[(size_t)i * N + col] = atan2f(v.y, v.x);
    }
}

struct ObjectPlan {
    int n_q;
    int bf_per_chunk;
    int n_chunks;
    size_t partial_bytes;
    size_t plane_bytes;
};

// Deterministic chunking (independent of the GPU's SM count): about 64 BF
// chunks at N <= 128 and 32 at N >= 256 (N^2/4-thread grids per chunk fill
// the GPU), 4..256 BF pixels each. At 128^2 with 1781 BF pixels the object
// takes 87 us with 64 chunks, 91 with 32 or 128, 127 with 16.
static ObjectPlan plan_object(int n, int n_bf, bool sym, int chunks_req = 0) {
    ObjectPlan pl;
    pl.n_q = sym ? n * (n / 2 + 1) + n / 2 - 1 : n * n;
    const int target = chunks_req > 0 ? chunks_req : (n >= 256 ? 32 : 64);
    int bpc = (n_bf + target - 1) / target;
    if (bpc < (chunks_req > 0 ? 1 : 4)) bpc = chunks_req > 0 ? 1 : 4;
    if (bpc > kMaxBfChunk) bpc = kMaxBfChunk;
    pl.bf_per_chunk = bpc;
    pl.n_chunks = (n_bf + bpc - 1) / bpc;
    pl.partial_bytes = sizeof(float2) * (size_t)pl.n_chunks * pl.n_q;
    pl.partial_bytes = (pl.partial_bytes + 255) & ~(size_t)255;
    pl.plane_bytes = sizeof(float2) * (size_t)n * n;
    return pl;
}

Probe make_probe(const qssb_calibration_t& cal, const qssb_aberrations_t& ab) {
    return make_probe_common(cal, ab.C10, ab.C12, ab.phi12, ab.C30);
}

int validate_calibration(const qssb_calibration_t* cal, const char* who) {
    if (!cal) return set_error(QSSB_ERR_INVALID, who);
    if (cal->n_bf <= 0 || cal->scan_rows != cal->scan_cols)
        return set_error(QSSB_ERR_INVALID, "calibration: n_bf must be >= 1 and the scan square");
    if (!(cal->wavelength_A > 0.0) || !(cal->semiangle_rad >= 0.0) ||
        !(cal->det_sampling_row_rad > 0.0) || !(cal->det_sampling_col_rad > 0.0) ||
        !(cal->scan_sampling_row_A > 0.0) || !(cal->scan_sampling_col_A > 0.0))
        return set_error(QSSB_ERR_INVALID, "calibration: wavelength and samplings must be positive");
    if (cal->reserved != 0) return set_error(QSSB_ERR_INVALID, "calibration: reserved must be 0");
    if (!isfinite(cal->dc_re) || !isfinite(cal->dc_im))
        return set_error(QSSB_ERR_INVALID, "calibration: dc must be finite");
    return QSSB_OK;
}

template <int N, int Q>
static void launch_quad(const float* g_half, const float* geom, const float* q_row,
                        const float* q_col, const qssb_calibration_t& cal, const Probe& p,
                        const ObjectPlan& pl, float2* partial, cudaStream_t s) {
    const dim3 grid((quad4_threads<N, Q>() + kTrotterThreads - 1) / kTrotterThreads, pl.n_chunks);
    { k_trotter_quad4<N, Q><<<grid, kTrotterThreads, 0, s>>>(
        reinterpret_cast<const float2*>(g_half), cal.n_bf, geom, q_row, q_col, p, pl.bf_per_chunk,
        partial); note_launch(); }
}

template <int N, bool SYM, bool CHI64, bool QUAD>
static int launch_object(const float* g_half, const float* geom, const float* q_row,
                         const float* q_col, const qssb_calibration_t& cal, const Probe& p,
                         int chunks, int variant, const double* dc_dev, char* ws, float* object,
                         float* phase, cudaStream_t s) {
    const ObjectPlan pl = plan_object(N, cal.n_bf, SYM, chunks);
    float2* partial = reinterpret_cast<float2*>(ws);
    float2* plane = reinterpret_cast<float2*>(ws + pl.partial_bytes);
    if constexpr (SYM && QUAD && !CHI64) {
        // tile shape: variant 1 -> 2 frequencies per thread, 3 -> 8, else 4
        if (variant == 1)
            launch_quad<N, 2>(g_half, geom, q_row, q_col, cal, p, pl, partial, s);
        else if (variant == 3)
            launch_quad<N, 8>(g_half, geom, q_row, q_col, cal, p, pl, partial, s);
        else
            launch_quad<N, 4>(g_half, geom, q_row, q_col, cal, p, pl, partial, s);
    } else {
        const dim3 grid((pl.n_q + kTrotterThreads - 1) / kTrotterThreads, pl.n_chunks);
        { k_trotter_partial<N, SYM, CHI64, QUAD><<<grid, kTrotterThreads, 0, s>>>(
            reinterpret_cast<const float2*>(g_half), cal.n_bf, geom, q_row, q_col, p,
            pl.bf_per_chunk, partial); note_launch(); }
    }
    CUDA_TRY(cudaGetLastError());
    { k_trotter_plane<N, SYM><<<(N * N + 31) / 32, 32 * kFoldSlices, 0, s>>>(
        partial, pl.n_chunks, cal.n_bf, make_float2((float)cal.dc_re, (float)cal.dc_im), dc_dev,
        plane); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    constexpr int W = ifft_lines<N>();
    { k_ifft_rows<N><<<N / W, 32 * W, 0, s>>>(plane); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    { k_ifft_cols_phase<N><<<N / W, 32 * W, 0, s>>>(plane, reinterpret_cast<float2*>(object), phase); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}

template <int N, bool QUAD>
static int dispatch_object_q(bool sym, bool chi64, const float* g_half, const float* geom,
                             const float* q_row, const float* q_col, const qssb_calibration_t& cal,
                             const Probe& p, int chunks, int variant, const double* dc_dev,
                             char* ws, float* object, float* phase, cudaStream_t s) {
    if (sym) {
        return chi64 ? launch_object<N, true, true, QUAD>(g_half, geom, q_row, q_col, cal, p, chunks, variant, dc_dev, ws, object, phase, s)
                     : launch_object<N, true, false, QUAD>(g_half, geom, q_row, q_col, cal, p, chunks, variant, dc_dev, ws, object, phase, s);
    }
    return chi64 ? launch_object<N, false, true, QUAD>(g_half, geom, q_row, q_col, cal, p, chunks, variant, dc_dev, ws, object, phase, s)
                 : launch_object<N, false, false, QUAD>(g_half, geom, q_row, q_col, cal, p, chunks, variant, dc_dev, ws, object, phase, s);
}

template <int N>
static int dispatch_object(bool sym, bool chi64, const float* g_half, const float* geom,
                           const float* q_row, const float* q_col, const qssb_calibration_t& cal,
                           const Probe& p, int chunks, int variant, const double* dc_dev, char* ws,
                           float* object, float* phase, cudaStream_t s) {
    if (p.quadratic)
        return dispatch_object_q<N, true>(sym, chi64, g_half, geom, q_row, q_col, cal, p, chunks, variant, dc_dev, ws, object, phase, s);
    return dispatch_object_q<N, false>(sym, chi64, g_half, geom, q_row, q_col, cal, p, chunks, variant, dc_dev, ws, object, phase, s);
}

}  // namespace qssb

using namespace qssb;

extern "C" int qssb_object_workspace_bytes(const qssb_calibration_t* cal, int32_t flags,
                                           size_t* bytes) {
    int rc = validate_calibration(cal, "qssb_object_workspace_bytes: null calibration");
    if (rc) return rc;
    if (!bytes) return set_error(QSSB_ERR_INVALID, "qssb_object_workspace_bytes: null output");
    const int n = cal->scan_rows;
    if (n != 64 && n != 128 && n != 256 && n != 512 && n != 1024)
        return set_error(QSSB_ERR_UNSUPPORTED,
                         "qssb_object: scan size must be 64, 128, 256, 512 or 1024");
    const ObjectPlan pl = plan_object(n, cal->n_bf, !(flags & QSSB_FLAG_FULL_PLANE), flag_chunks(flags));
    *bytes = pl.partial_bytes + pl.plane_bytes;
    return QSSB_OK;
}

extern "C" int qssb_object_ex(const float* g_half, const float* bf_geom, const float* q_row,
                              const float* q_col, const qssb_calibration_t* cal,
                              const qssb_aberrations_t* ab, int32_t flags, const double* dc_device,
                              void* workspace, size_t workspace_bytes, float* object, float* phase,
                              void* stream) {
    if (dc_device && ((uintptr_t)dc_device & 7u) != 0)
        return set_error(QSSB_ERR_INVALID, "qssb_object_ex: dc_device must be 8-byte aligned");
    int rc = validate_calibration(cal, "qssb_object: null calibration");
    if (rc) return rc;
    if (!g_half || !bf_geom || !q_row || !q_col || !ab || !workspace || !object)
        return set_error(QSSB_ERR_INVALID, "qssb_object: null pointer");
    if (!isfinite(ab->C10) || !isfinite(ab->C12) || !isfinite(ab->phi12) || !isfinite(ab->C30))
        return set_error(QSSB_ERR_INVALID, "qssb_object: aberrations must be finite");
    size_t need = 0;
    rc = qssb_object_workspace_bytes(cal, flags, &need);
    if (rc) return rc;
    if (workspace_bytes < need) return set_error(QSSB_ERR_WORKSPACE, "qssb_object: workspace too small");
    if (((uintptr_t)workspace & 255u) != 0)
        return set_error(QSSB_ERR_INVALID, "qssb_object: workspace must be 256-byte aligned");
    const Probe p = make_probe(*cal, *ab);
    const bool sym = !(flags & QSSB_FLAG_FULL_PLANE);
    const bool chi64 = (flags & QSSB_FLAG_CHI_FP64) != 0;
    const int chunks = flag_chunks(flags);
    const double* dc_dev = dc_device;
    cudaStream_t s = (cudaStream_t)stream;
    char* ws = static_cast<char*>(workspace);
    switch (cal->scan_rows) {
        case 64: return dispatch_object<64>(sym, chi64, g_half, bf_geom, q_row, q_col, *cal, p, chunks, flag_variant(flags), dc_dev, ws, object, phase, s);
        case 128: return dispatch_object<128>(sym, chi64, g_half, bf_geom, q_row, q_col, *cal, p, chunks, flag_variant(flags), dc_dev, ws, object, phase, s);
        case 256: return dispatch_object<256>(sym, chi64, g_half, bf_geom, q_row, q_col, *cal, p, chunks, flag_variant(flags), dc_dev, ws, object, phase, s);
        case 512: return dispatch_object<512>(sym, chi64, g_half, bf_geom, q_row, q_col, *cal, p, chunks, flag_variant(flags), dc_dev, ws, object, phase, s);
        case 1024: return dispatch_object<1024>(sym, chi64, g_half, bf_geom, q_row, q_col, *cal, p, chunks, flag_variant(flags), dc_dev, ws, object, phase, s);
        default: return set_error(QSSB_ERR_UNSUPPORTED,
                                  "qssb_object: scan size must be 64, 128, 256, 512 or 1024");
    }
}

extern "C" int qssb_object(const float* g_half, const float* bf_geom, const float* q_row,
                           const float* q_col, const qssb_calibration_t* cal,
                           const qssb_aberrations_t* ab, int32_t flags, void* workspace,
                           size_t workspace_bytes, float* object, float* phase, void* stream) {
    return qssb_object_ex(g_half, bf_geom, q_row, q_col, cal, ab, flags, nullptr, workspace,
                          workspace_bytes, object, phase, stream);
}

// ---------------------------------------------------------------------------
// qssb_object_noalloc: the same launch sequence with its scratch in a fixed
// file-scope device array (see include/qssb.h for the callers it serves and
// the sharing rules). The host must not pass the array's name to a kernel:
// in host code it is a stand-in, not a device address. Its device address is
// looked up once per device with cudaGetSymbolAddress and cached for the
// life of the process (a device reset, which destroys the context the
// address belongs to, makes it stale; the header says so).
static __device__ __align__(256) unsigned char g_noalloc_scratch[QSSB_NOALLOC_SCRATCH_BYTES];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_addr[kMaxDevices] = {nullptr};
}  // namespace

extern "C" int qssb_object_noalloc(const float* g_half, const float* bf_geom, const float* q_row,
                                   const float* q_col, const qssb_calibration_t* cal,
                                   const qssb_aberrations_t* ab, int32_t flags, float* object,
                                   float* phase, void* stream) {
    int rc = validate_calibration(cal, "qssb_object_noalloc: null calibration");
    if (rc) return rc;
    size_t need = 0;
    rc = qssb_object_workspace_bytes(cal, flags, &need);
    if (rc) return rc;
    if (need > (size_t)QSSB_NOALLOC_SCRATCH_BYTES)
        return set_error(QSSB_ERR_WORKSPACE,
                         "qssb_object_noalloc: this scan size and BF count need more than the "
                         "16 MiB fixed scratch; use qssb_object with a caller workspace");
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices)
        return set_error(QSSB_ERR_UNSUPPORTED, "qssb_object_noalloc: device ordinal out of range");
    void* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        if (g_noalloc_addr[dev] == nullptr) {
            void* addr = nullptr;
            const cudaError_t err = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
            if (err != cudaSuccess) return set_cuda_error(err, "qssb_object_noalloc: cudaGetSymbolAddress");
            g_noalloc_addr[dev] = addr;
        }
        scratch = g_noalloc_addr[dev];
    }
    return qssb_object(g_half, bf_geom, q_row, q_col, cal, ab, flags, scratch,
                       (size_t)QSSB_NOALLOC_SCRATCH_BYTES, object, phase, stream);
}
