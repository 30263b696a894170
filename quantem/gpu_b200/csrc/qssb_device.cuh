// qssb_device.cuh - device building blocks of the SSB engine (sm_100a).
//
// * complex helpers and radix-2/4/8 butterflies;
// * a warp-cooperative Stockham FFT over one line held in shared memory
//   (any stride), N in {64, 128, 256, 512, 1024}, forward (exp(-2 pi i nk/N)) or
//   inverse (exp(+2 pi i nk/N), unnormalised);
// * the probe transfer function P(u) = A(u) exp(-i chi(u)) and the
//   normalised double-overlap correction of the reference SSB kernels
//   (bobleesj/quantem.gpu src/quantem/gpu/ssb/compute/cuda/kernels/
//   common.py:115-236), restated.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../../include/qssb.h"

namespace qssb {

// ---------------------------------------------------------------- complex
// On sm_100 the FP32 pipe executes two-wide packed instructions (FADD2,
// FMUL2, FFMA2), each lane rounded exactly as its scalar counterpart, so the
// (re, im) pairs below cost one instruction where two scalar ones did, with
// the same bits. Negation and the exact subtraction a - b == a + (-b) keep
// every result identical to the scalar forms.
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) {
    return __fadd2_rn(a, make_float2(-b.x, -b.y));
}
// (a.x b.x - a.y b.y, a.x b.y + a.y b.x) with the products of a.y rounded
// first: fma(a.x, b.x, -(a.y b.y)), fma(a.x, b.y, a.y b.x)
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    const float2 t = __fmul2_rn(make_float2(a.y, a.y), make_float2(-b.y, b.x));
    return __ffma2_rn(make_float2(a.x, a.x), b, t);
}
// a * s for a real s
__device__ __forceinline__ float2 cscale(float2 a, float s) { return __fmul2_rn(a, make_float2(s, s)); }
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cneg_conj(float2 a) { return make_float2(-a.x, a.y); }
// multiply by DIR * i  (DIR = -1: -i, DIR = +1: +i)
template <int DIR>
__device__ __forceinline__ float2 mul_dir_i(float2 a) {
    return DIR < 0 ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
}

// Twiddles tw[m] = exp(-2 pi i m / N), correctly rounded from FP64.
template <int N>
__device__ __forceinline__ void fill_twiddles(float2* tw, int tid, int nthreads) {
    for (int m = tid; m < N; m += nthreads) {
        double s, c;
        sincospi(-2.0 * (double)m / (double)N, &s, &c);
        tw[m] = make_float2((float)c, (float)s);
    }
}

// ------------------------------------------------------------- butterflies
template <int DIR>
__device__ __forceinline__ void dft2(float2& a, float2& b) {
    float2 t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

template <int DIR>
__device__ __forceinline__ void dft4(float2* v) {
    float2 s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
    float2 s13 = cadd(v[1], v[3]), d13 = mul_dir_i<DIR>(csub(v[1], v[3]));
    v[0] = cadd(s02, s13);
    v[2] = csub(s02, s13);
    v[1] = cadd(d02, d13);
    v[3] = csub(d02, d13);
}

template <int DIR>
__device__ __forceinline__ void dft8(float2* v) {
    float2 e[4] = {v[0], v[2], v[4], v[6]};
    float2 o[4] = {v[1], v[3], v[5], v[7]};
    dft4<DIR>(e);
    dft4<DIR>(o);
    const float h = 0.70710678118654752440f;
    // W8^k = exp(DIR 2 pi i k / 8)
    float2 w1o = cmul(o[1], make_float2(h, DIR * h));
    float2 w2o = mul_dir_i<DIR>(o[2]);
    float2 w3o = cmul(o[3], make_float2(-h, DIR * h));
    v[0] = cadd(e[0], o[0]);
    v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], w1o);
    v[5] = csub(e[1], w1o);
    v[2] = cadd(e[2], w2o);
    v[6] = csub(e[2], w2o);
    v[3] = cadd(e[3], w3o);
    v[7] = csub(e[3], w3o);
}

template <int R, int DIR>
__device__ __forceinline__ void dft_r(float2* v) {
    if constexpr (R == 2) {
        dft2<DIR>(v[0], v[1]);
    } else if constexpr (R == 4) {
        dft4<DIR>(v);
    } else {
        static_assert(R == 8, "radix 2, 4 or 8");
        dft8<DIR>(v);
    }
}

// --------------------------------------------------------- Stockham stage
// One radix-R pass of the self-sorting (Stockham) FFT over a line of N
// complex values at x[i * stride], executed by the 32 lanes of one warp.
// Butterfly j (of N/R) reads x[j + r N/R], twiddles by W_{Ns R}^{k r}
// (k = j mod Ns), transforms and writes x[(j - k) R + k + r Ns]. All lanes
// read before any lane writes (the __syncwarp between), so it runs in place.
template <int N, int R, int NS, int DIR>
__device__ __forceinline__ void stockham_stage(float2* x, int stride, const float2* tw, int lane) {
    constexpr int NB = N / R;
    constexpr int PER = (NB + 31) / 32;
    constexpr int TWS = N / (NS * R);
    float2 v[PER][R];
#pragma unroll
    for (int t = 0; t < PER; ++t) {
        const int j = lane + 32 * t;
        if (NB % 32 == 0 || j < NB) {
            const int k = j & (NS - 1);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                float2 a = x[(j + r * NB) * stride];
                if (NS > 1 && r > 0) {
                    float2 w = tw[k * r * TWS];
                    if (DIR > 0) w.y = -w.y;
                    a = cmul(a, w);
                }
                v[t][r] = a;
            }
            dft_r<R, DIR>(v[t]);
        }
    }
    __syncwarp();
#pragma unroll
    for (int t = 0; t < PER; ++t) {
        const int j = lane + 32 * t;
        if (NB % 32 == 0 || j < NB) {
            const int k = j & (NS - 1);
            const int base = (j - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) x[(base + r * NS) * stride] = v[t][r];
        }
    }
    __syncwarp();
}

// 16-point DFT in registers (natural order in and out): 4 x 4 with the
// W16 twiddles between the two radix-4 passes.
template <int DIR>
__device__ __forceinline__ void dft16(float2* x) {
    const float c1 = 0.92387953251128675613f;  // cos(pi/8)
    const float s1 = 0.38268343236508977173f;  // sin(pi/8)
    const float h = 0.70710678118654752440f;
    float2 y[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        float2 t[4] = {x[a], x[a + 4], x[a + 8], x[a + 12]};
        dft4<DIR>(t);
#pragma unroll
        for (int c = 0; c < 4; ++c) y[a][c] = t[c];
    }
    // W16^m = (cos(2 pi m / 16), DIR sin(2 pi m / 16)), m = a * c
    y[1][1] = cmul(y[1][1], make_float2(c1, DIR * s1));   // m = 1
    y[1][2] = cmul(y[1][2], make_float2(h, DIR * h));     // m = 2
    y[1][3] = cmul(y[1][3], make_float2(s1, DIR * c1));   // m = 3
    y[2][1] = cmul(y[2][1], make_float2(h, DIR * h));     // m = 2
    y[2][2] = mul_dir_i<DIR>(y[2][2]);                    // m = 4
    y[2][3] = cmul(y[2][3], make_float2(-h, DIR * h));    // m = 6
    y[3][1] = cmul(y[3][1], make_float2(s1, DIR * c1));   // m = 3
    y[3][2] = cmul(y[3][2], make_float2(-h, DIR * h));    // m = 6
    y[3][3] = cmul(y[3][3], make_float2(-c1, -DIR * s1)); // m = 9
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float2 t[4] = {y[0][c], y[1][c], y[2][c], y[3][c]};
        dft4<DIR>(t);
#pragma unroll
        for (int d = 0; d < 4; ++d) x[c + 4 * d] = t[d];
    }
}

// A 128-point FFT by a group of 8 lanes (sub-lane s), 16 values per lane:
// four-step 128 = 16 x 8. In: v[n1] = x[s + 8 n1]. DFT-16 over n1 in
// registers, twiddle W128^(s k1), transpose through the group's scratch T
// (16 rows of pitch 9, conflict-free for two groups per half-warp when the
// groups' T bases differ by 8 mod 16 float2), DFT-8 over s for k1 = s and
// s + 8. Out: v[t] = X[fft128_g8_index(s, t)] = X[s + 8 (t / 8) + 16 (t % 8)].
// The 8 lanes of a group must belong to one warp; all 32 lanes call it.
constexpr int kG8Pitch = 9;
constexpr int kG8Scratch = 16 * kG8Pitch + 8;  // float2 per group (152)

__device__ __forceinline__ int fft128_g8_index(int s, int t) { return s + 8 * (t >> 3) + 16 * (t & 7); }

template <int DIR>
__device__ __forceinline__ void fft128_g8(float2 (&v)[16], float2* T, int s, const float2* tw) {
    dft16<DIR>(v);
#pragma unroll
    for (int k1 = 1; k1 < 16; ++k1) {
        float2 w = tw[s * k1];
        if (DIR > 0) w.y = -w.y;
        v[k1] = cmul(v[k1], w);
    }
#pragma unroll
    for (int k1 = 0; k1 < 16; ++k1) T[k1 * kG8Pitch + s] = v[k1];
    __syncwarp();
    float2 u0[8], u1[8];
#pragma unroll
    for (int n2 = 0; n2 < 8; ++n2) {
        u0[n2] = T[s * kG8Pitch + n2];
        u1[n2] = T[(s + 8) * kG8Pitch + n2];
    }
    __syncwarp();
    dft8<DIR>(u0);
    dft8<DIR>(u1);
#pragma unroll
    for (int k2 = 0; k2 < 8; ++k2) {
        v[k2] = u0[k2];
        v[8 + k2] = u1[k2];
    }
}

// Whole line FFT of length N (natural order in, natural order out).
template <int N, int DIR>
__device__ __forceinline__ void line_fft(float2* x, int stride, const float2* tw, int lane) {
    if constexpr (N == 64) {
        stockham_stage<64, 4, 1, DIR>(x, stride, tw, lane);
        stockham_stage<64, 4, 4, DIR>(x, stride, tw, lane);
        stockham_stage<64, 4, 16, DIR>(x, stride, tw, lane);
    } else if constexpr (N == 128) {
        stockham_stage<128, 4, 1, DIR>(x, stride, tw, lane);
        stockham_stage<128, 4, 4, DIR>(x, stride, tw, lane);
        stockham_stage<128, 4, 16, DIR>(x, stride, tw, lane);
        stockham_stage<128, 2, 64, DIR>(x, stride, tw, lane);
    } else if constexpr (N == 256) {
        stockham_stage<256, 8, 1, DIR>(x, stride, tw, lane);
        stockham_stage<256, 8, 8, DIR>(x, stride, tw, lane);
        stockham_stage<256, 4, 64, DIR>(x, stride, tw, lane);
    } else if constexpr (N == 512) {
        stockham_stage<512, 8, 1, DIR>(x, stride, tw, lane);
        stockham_stage<512, 8, 8, DIR>(x, stride, tw, lane);
        stockham_stage<512, 8, 64, DIR>(x, stride, tw, lane);
    } else {
        static_assert(N == 1024, "line FFT sizes 64, 128, 256, 512, 1024");
        stockham_stage<1024, 8, 1, DIR>(x, stride, tw, lane);
        stockham_stage<1024, 8, 8, DIR>(x, stride, tw, lane);
        stockham_stage<1024, 4, 64, DIR>(x, stride, tw, lane);
        stockham_stage<1024, 4, 256, DIR>(x, stride, tw, lane);
    }
}

// ------------------------------------------- register-resident warp FFT
// N = R * 32 (N in {256, 512, 1024}; R = 8, 16, 32 values per lane), four
// steps with one shared-memory transpose:
//   in:  v[n1] = x[32 n1 + lane];
//   DFT-R over n1 in registers, twiddle W_N^(lane k1);
//   transpose through T[k1][n2] (pitch 32 + G: conflict-free both ways);
//   lane (k1 = lane / G, h = lane % G), G = 32 / R, takes n2 = h + G m:
//   DFT-R over m, twiddle W_32^(h k2'), DFT-G across the G lanes of k1
//   (warp shuffles);
//   out: v[j] = X[warp_fft_index<N>(lane, j)] = X[k1 + R (j + R (lane % G))].
// tw: the N-entry table of fill_twiddles<N>. T: warp_fft_scratch<N>() float2.
template <int DIR>
__device__ __forceinline__ void dft32(float2* x, const float2* tw, int step) {
    float2 e[16], o[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        e[i] = x[2 * i];
        o[i] = x[2 * i + 1];
    }
    dft16<DIR>(e);
    dft16<DIR>(o);
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        float2 w = tw[k * step];
        if (DIR > 0) w.y = -w.y;
        const float2 t = cmul(o[k], w);
        x[k] = cadd(e[k], t);
        x[k + 16] = csub(e[k], t);
    }
}

template <int R, int DIR>
__device__ __forceinline__ void dft_reg(float2* v, const float2* tw, int step32) {
    if constexpr (R == 8) {
        dft8<DIR>(v);
    } else if constexpr (R == 16) {
        dft16<DIR>(v);
    } else {
        static_assert(R == 32, "warp FFT radix 8, 16 or 32");
        dft32<DIR>(v, tw, step32);
    }
}

template <int N>
__host__ __device__ constexpr int warp_fft_scratch() {
    return (N / 32) * (32 + 32 / (N / 32));
}

template <int N>
__device__ __forceinline__ int warp_fft_index(int lane, int j) {
    constexpr int R = N / 32;
    constexpr int G = 32 / R;
    return lane / G + R * (j + R * (lane % G));
}

template <int N, int DIR>
__device__ __forceinline__ void warp_fft(float2 (&v)[N / 32], float2* T, const float2* tw, int lane) {
    constexpr int R = N / 32;
    constexpr int G = 32 / R;
    constexpr int P = 32 + G;
    constexpr int S32 = N / 32;  // W_32^e = tw[e * S32]
    dft_reg<R, DIR>(v, tw, S32);
#pragma unroll
    for (int k1 = 1; k1 < R; ++k1) {
        float2 w = tw[lane * k1];
        if (DIR > 0) w.y = -w.y;
        v[k1] = cmul(v[k1], w);
    }
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) T[k1 * P + lane] = v[k1];
    __syncwarp();
    const int k1 = lane / G;
    const int h = lane % G;
#pragma unroll
    for (int m = 0; m < R; ++m) v[m] = T[k1 * P + h + G * m];
    __syncwarp();
    dft_reg<R, DIR>(v, tw, S32);
    if constexpr (G > 1) {
#pragma unroll
        for (int k2 = 1; k2 < R; ++k2) {
            float2 w = tw[((h * k2) & 31) * S32];
            if (DIR > 0) w.y = -w.y;
            v[k2] = cmul(v[k2], w);
        }
        if constexpr (G == 2) {
#pragma unroll
            for (int j = 0; j < R; ++j) {
                float2 o;
                o.x = __shfl_xor_sync(0xffffffffu, v[j].x, 1);
                o.y = __shfl_xor_sync(0xffffffffu, v[j].y, 1);
                v[j] = h == 0 ? cadd(v[j], o) : csub(o, v[j]);
            }
        } else {
            static_assert(G == 4, "cross-lane radix 2 or 4");
            const int base = lane & ~3;
#pragma unroll
            for (int j = 0; j < R; ++j) {
                float2 s[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    s[i].x = __shfl_sync(0xffffffffu, v[j].x, base + i);
                    s[i].y = __shfl_sync(0xffffffffu, v[j].y, base + i);
                }
                // X_h = sum_i W4^(i h) s_i, W4 = exp(DIR 2 pi i / 4) = DIR i
                float2 acc = s[0];
#pragma unroll
                for (int i = 1; i < 4; ++i) {
                    const int e = (i * h) & 3;
                    float2 t = s[i];
                    if (e == 1) t = mul_dir_i<DIR>(t);
                    else if (e == 2) t = make_float2(-t.x, -t.y);
                    else if (e == 3) t = mul_dir_i<-DIR>(t);
                    acc = cadd(acc, t);
                }
                v[j] = acc;
            }
        }
    }
}

// --------------------------------------------------------------- physics
// Per-candidate probe constants. chi(u) = factor * alpha^2 *
// (C10 + C12 (cos2phi cos2phi12 + sin2phi sin2phi12)) + c30_half * alpha^4,
// factor = pi / lambda, c30_half = (pi / (2 lambda)) C30.
struct Probe {
    float wavelength;
    float semiangle;
    float ang_r;
    float ang_c;
    float inner2;     // (|u| <= inner) => aperture == 1 exactly; <= 0 disables
    float outer2;     // (|u| >= outer) => aperture == 0 exactly
    float inv_ang;    // 1 / d_row (isotropic detector sampling)
    bool iso;         // d_row == d_col: denom == d_row for every direction
    float factor;
    float C10;
    float C12;
    float cos2p;
    float sin2p;
    float c30_half;
    // FP64 calibration for near-tied aperture pairs (soft_aperture_fp64)
    double semi_d, lam_d, ang_r_d, ang_c_d;
    double qval_r, qval_c;  // 1 / (R d): q = fftfreq index * qval
    int n_r, n_c;
    // chi(u) = u^T M u for the quadratic (C10, C12) part; M symmetric
    float mxx, mxy, myy;
    double mxx_d, mxy_d, myy_d;
    bool quadratic;   // C30 == 0: the factorised overlap applies
    double factor_d;  // FP64 copies for QSSB_FLAG_CHI_FP64
    double C10_d;
    double C12_d;
    double cos2p_d;
    double sin2p_d;
    double c30_half_d;
};

// Soft aperture at displacement (dx, dy) with r2 = dx^2 + dy^2:
// clip((alpha_max - lambda |u|) / denom + 0.5, 0, 1),
// denom = sqrt((dx d_row)^2 + (dy d_col)^2) / |u|. Both shortcuts are exact:
// denom <= max(d_row, d_col) makes the clipped edge 1 inside `inner` and 0
// outside `outer`; only the band between them is evaluated.
__device__ __forceinline__ float soft_aperture(float dx, float dy, float r2, const Probe& p) {
    if (p.inner2 > 0.0f && r2 <= p.inner2) return 1.0f;
    if (r2 >= p.outer2) return 0.0f;
    const float r = sqrtf(r2);
    const float alpha = r * p.wavelength;
    const float num2 = fmaf(dx * p.ang_r, dx * p.ang_r, (dy * p.ang_c) * (dy * p.ang_c));
    const float inv_r = r > 1e-15f ? 1.0f / r : 0.0f;
    const float denom = sqrtf(num2) * inv_r;
    const float edge = denom > 1e-15f ? (p.semiangle - alpha) / denom + 0.5f : 1.0f;
    return fminf(fmaxf(edge, 0.0f), 1.0f);
}

// The same aperture without branches and with reciprocal square roots only
// (the arithmetic class of a --use_fast_math build): r = r2 rsqrt(r2); with
// isotropic sampling denom == d exactly, so one MUFU op per call. The exact
// 1 inside `inner` and 0 outside `outer` are kept by selects: the tied-overlap
// refinement depends on them.
__device__ __forceinline__ float soft_aperture_fast(float dx, float dy, float r2, const Probe& p) {
    const float r = r2 * rsqrtf(r2);
    const float num = p.semiangle - r * p.wavelength;
    float edge;
    if (p.iso) {
        edge = fmaf(num, p.inv_ang, 0.5f);
    } else {
        const float ar = dx * p.ang_r;
        const float ac = dy * p.ang_c;
        edge = fmaf(num * r, rsqrtf(fmaf(ar, ar, ac * ac)), 0.5f);
    }
    float a = __saturatef(edge);          // clip to [0, 1]; NaN (r2 == 0) -> 0
    a = r2 >= p.outer2 ? 0.0f : a;
    a = r2 <= p.inner2 ? 1.0f : a;        // inner2 >= 0, so r2 == 0 gives 1
    return a;
}

// The apertures at two displacements at once, (A(dm), A(dp)) for squared
// radii r2 = (|dm|^2, |dp|^2): the isotropic form in packed FP32 (lane by
// lane the same operations as soft_aperture_fast), the other form per lane.
__device__ __forceinline__ float2 soft_aperture_fast2(float2 dm, float2 dp, float2 r2,
                                                      const Probe& p) {
    if (!p.iso)
        return make_float2(soft_aperture_fast(dm.x, dm.y, r2.x, p),
                           soft_aperture_fast(dp.x, dp.y, r2.y, p));
    const float2 r = __fmul2_rn(r2, make_float2(rsqrtf(r2.x), rsqrtf(r2.y)));
    const float2 num = __ffma2_rn(make_float2(-r.x, -r.y), make_float2(p.wavelength, p.wavelength),
                                  make_float2(p.semiangle, p.semiangle));
    const float2 edge = __ffma2_rn(num, make_float2(p.inv_ang, p.inv_ang), make_float2(0.5f, 0.5f));
    float am = __saturatef(edge.x), ap = __saturatef(edge.y);
    am = r2.x >= p.outer2 ? 0.0f : am;
    ap = r2.y >= p.outer2 ? 0.0f : ap;
    am = r2.x <= p.inner2 ? 1.0f : am;
    ap = r2.y <= p.inner2 ? 1.0f : ap;
    return make_float2(am, ap);
}

__device__ __forceinline__ bool in_edge_band(float r2, const Probe& p) {
    return !(p.inner2 > 0.0f && r2 <= p.inner2) && r2 < p.outer2;
}

// The same aperture in FP64 at displacement (dx, dy) (u = q -+ k from FP64
// q and k), with the FP64 calibration.
static __device__ __noinline__ float soft_aperture_fp64(double dx, double dy, double semiangle,
                                                        double wavelength, double ang_r,
                                                        double ang_c) {
    const double r = sqrt(dx * dx + dy * dy);
    const double ar = dx * ang_r;
    const double ac = dy * ang_c;
    const double num = sqrt(ar * ar + ac * ac);
    if (!(r > 1e-300) || !(num > 0.0)) return 1.0f;
    const double edge = (semiangle - r * wavelength) / (num / r) + 0.5;
    return (float)fmin(fmax(edge, 0.0), 1.0);
}

// numpy.fft.fftfreq(n, d)[i] in FP64: (i < n/2 ? i : i - n) * (1 / (n d)).
__device__ __forceinline__ double fftfreq_d(int i, int n, double val) {
    return (double)(i < (n >> 1) ? i : i - n) * val;
}

// chi from (alpha^2, cos 2phi, sin 2phi).
template <bool CHI64>
__device__ __forceinline__ float chi_value(float alpha2, float cos2, float sin2, const Probe& p) {
    if constexpr (CHI64) {
        const double a2 = (double)alpha2;
        const double term = fma(p.C12_d, fma((double)cos2, p.cos2p_d, (double)sin2 * p.sin2p_d), p.C10_d);
        double chi = p.factor_d * a2 * term + p.c30_half_d * a2 * a2;
        // exact reduction to [-pi, pi] in FP64
        chi -= 6.283185307179586476925 * rint(chi * 0.15915494309189533577);
        return (float)chi;
    } else {
        const float term = fmaf(p.C12, fmaf(cos2, p.cos2p, sin2 * p.sin2p), p.C10);
        return fmaf(p.c30_half * alpha2, alpha2, p.factor * alpha2 * term);
    }
}

// Geometry of one displacement as compute_geometry (common.py:115-157):
// alpha^2 = r2 lambda^2, cos 2phi = (dx^2 - dy^2)/r2, sin 2phi = 2 dx dy / r2
// (0 at the origin).
struct Disp {
    float r2, alpha2, cos2, sin2;
};

__device__ __forceinline__ Disp displacement(float dx, float dy, const Probe& p) {
    Disp d;
    const float dx2 = dx * dx;
    const float dy2 = dy * dy;
    d.r2 = dx2 + dy2;
    d.alpha2 = (d.r2 * p.wavelength) * p.wavelength;
    const float inv_r2 = d.r2 > 1e-30f ? 1.0f / d.r2 : 0.0f;
    d.cos2 = (dx2 - dy2) * inv_r2;
    d.sin2 = 2.0f * dx * dy * inv_r2;
    return d;
}

template <bool CHI64>
__device__ __forceinline__ float2 probe_from(const Disp& d, float ap, const Probe& p) {
    if (ap == 0.0f) return make_float2(0.0f, 0.0f);
    float s, c;
    __sincosf(chi_value<CHI64>(d.alpha2, d.cos2, d.sin2, p), &s, &c);
    return make_float2(ap * c, -ap * s);
}

// P(k_b) from the cached BF geometry (engine.py:217-231, _pk_kernel).
template <bool CHI64>
__device__ __forceinline__ float2 probe_at_bf(float alpha2, float cos2, float sin2, float aperture,
                                              const Probe& p) {
    float s, c;
    __sincosf(chi_value<CHI64>(alpha2, cos2, sin2, p), &s, &c);
    return make_float2(aperture * c, -aperture * s);
}

// Aperture pairs closer than this are re-evaluated in FP64 when either lies
// in the edge band. For an aberration-free (real) Gamma = A(k)(A(q-k) -
// A(q+k)) the sign of the unit-normalised Gamma is decided by that
// difference; where q is (nearly) perpendicular to k it is pure float32
// rounding (the edge carries ~1e-6 absolute), and on an integer-centred BF
// lattice exactly perpendicular pairs are common. Evaluating both apertures
// from FP64 q and k (k = kx + kx_lo) reproduces the FP64 result there.
constexpr float kApertureTie = 1.0e-4f;

// G conj(Gamma_hat) from the displacements and apertures of q - k and q + k:
// Gamma = P(q - k) conj(P(k)) - conj(P(q + k)) P(k), unit-normalised.
template <bool CHI64>
__device__ __forceinline__ float2 corrected_from_apertures(const Disp& dm, const Disp& dp, float am,
                                                           float ap, float2 pk, float2 g,
                                                           const Probe& p) {
    const float2 pm = probe_from<CHI64>(dm, am, p);
    const float2 pp = probe_from<CHI64>(dp, ap, p);
    // t1 = pm * conj(pk); t2 = conj(pp) * pk
    const float t1r = fmaf(pm.x, pk.x, pm.y * pk.y);
    const float t1i = fmaf(pm.y, pk.x, -pm.x * pk.y);
    const float t2r = fmaf(pp.x, pk.x, pp.y * pk.y);
    const float t2i = fmaf(pp.x, pk.y, -pp.y * pk.x);
    float gr = t1r - t2r;
    float gi = t1i - t2i;
    const float m2 = fmaf(gr, gr, gi * gi);
    const float inv = m2 > 1e-16f ? rsqrtf(m2) : 1e8f;
    gr *= inv;
    gi *= inv;
    return make_float2(fmaf(g.x, gr, g.y * gi), fmaf(g.y, gr, -g.x * gi));
}

// C = G conj(Gamma_hat), Gamma = P(q-k) conj(P(k)) - conj(P(q+k)) P(k),
// Gamma_hat = Gamma * (|Gamma|^2 > 1e-16 ? 1/|Gamma| : 1e8)
// (gamma_mul_pk_onthefly, common.py:173-236). (r, c) index the scan
// frequency (qx, qy); kx_lo/ky_lo are the FP64 residuals of k.
template <bool CHI64>
__device__ __forceinline__ float2 corrected(float qx, float qy, int r, int c, float kx, float ky,
                                            float kx_lo, float ky_lo, float2 pk, float2 g,
                                            const Probe& p) {
    const Disp dm = displacement(qx - kx, qy - ky, p);
    const Disp dp = displacement(qx + kx, qy + ky, p);
    float am = soft_aperture(qx - kx, qy - ky, dm.r2, p);
    float ap = soft_aperture(qx + kx, qy + ky, dp.r2, p);
    if (fabsf(am - ap) < kApertureTie && (in_edge_band(dm.r2, p) || in_edge_band(dp.r2, p))) {
        const double qx64 = fftfreq_d(r, p.n_r, p.qval_r);
        const double qy64 = fftfreq_d(c, p.n_c, p.qval_c);
        const double kx64 = (double)kx + (double)kx_lo;
        const double ky64 = (double)ky + (double)ky_lo;
        am = soft_aperture_fp64(qx64 - kx64, qy64 - ky64, p.semi_d, p.lam_d, p.ang_r_d, p.ang_c_d);
        ap = soft_aperture_fp64(qx64 + kx64, qy64 + ky64, p.semi_d, p.lam_d, p.ang_r_d, p.ang_c_d);
    }
    return corrected_from_apertures<CHI64>(dm, dp, am, ap, pk, g, p);
}

// Probe constants of one candidate from the calibration (FP64 trig of phi12).
__host__ __device__ inline Probe make_probe_common(const qssb_calibration_t& cal, float C10,
                                                   float C12, float phi12, float C30) {
    Probe p;
    p.wavelength = (float)cal.wavelength_A;
    p.semiangle = (float)cal.semiangle_rad;
    p.ang_r = (float)cal.det_sampling_row_rad;
    p.ang_c = (float)cal.det_sampling_col_rad;
    const float max_ang = fmaxf(p.ang_r, p.ang_c);
    const float inner = (p.semiangle - 0.5f * max_ang) / p.wavelength;
    p.inner2 = inner > 0.0f ? inner * inner : 0.0f;
    const float outer = (p.semiangle + 0.5f * max_ang) / p.wavelength;
    p.outer2 = outer * outer;
    p.iso = cal.det_sampling_row_rad == cal.det_sampling_col_rad;
    p.inv_ang = (float)(1.0 / cal.det_sampling_row_rad);
    p.semi_d = cal.semiangle_rad;
    p.lam_d = cal.wavelength_A;
    p.ang_r_d = cal.det_sampling_row_rad;
    p.ang_c_d = cal.det_sampling_col_rad;
    p.n_r = cal.scan_rows;
    p.n_c = cal.scan_cols;
    p.qval_r = 1.0 / ((double)cal.scan_rows * cal.scan_sampling_row_A);
    p.qval_c = 1.0 / ((double)cal.scan_cols * cal.scan_sampling_col_A);
    const double factor = 3.14159265358979323846 / cal.wavelength_A;
    const double c2 = cos(2.0 * (double)phi12);
    const double s2 = sin(2.0 * (double)phi12);
    p.factor = (float)factor;
    p.C10 = C10;
    p.C12 = C12;
    p.cos2p = (float)c2;
    p.sin2p = (float)s2;
    p.c30_half = (float)(0.5 * factor * (double)C30);
    p.factor_d = factor;
    p.C10_d = C10;
    p.C12_d = C12;
    p.cos2p_d = c2;
    p.sin2p_d = s2;
    p.c30_half_d = 0.5 * factor * (double)C30;
    // M = (pi / lambda) lambda^2 [[C10 + C12 c2, C12 s2], [C12 s2, C10 - C12 c2]]
    const double fl2 = factor * cal.wavelength_A * cal.wavelength_A;
    p.mxx_d = fl2 * ((double)C10 + (double)C12 * c2);
    p.mxy_d = fl2 * (double)C12 * s2;
    p.myy_d = fl2 * ((double)C10 - (double)C12 * c2);
    p.mxx = (float)p.mxx_d;
    p.mxy = (float)p.mxy_d;
    p.myy = (float)p.myy_d;
    p.quadratic = (C30 == 0.0f);
    return p;
}

// Reduce an FP64 angle to [-pi, pi] and round to float32.
__device__ __forceinline__ float reduce_angle(double a) {
    return (float)(a - 6.283185307179586476925 * rint(a * 0.15915494309189533577));
}

// (cos Q(q), sin Q(q)), Q(q) = q^T M q, from the FP64 grid value of q.
__device__ __forceinline__ float2 eq_value(int r, int c, const Probe& p) {
    const double qx = fftfreq_d(r, p.n_r, p.qval_r);
    const double qy = fftfreq_d(c, p.n_c, p.qval_c);
    const double q = fma(p.mxx_d * qx, qx, fma(2.0 * p.mxy_d * qx, qy, p.myy_d * qy * qy));
    float s, co;
    sincosf(reduce_angle(q), &s, &co);
    return make_float2(co, s);
}

// Per-BF constants of the factorised overlap: (u, v) = M k.
struct BFQuad {
    float kx, ky, kx_lo, ky_lo, ak, u, v;
    double ud, vd;  // FP64 M k (QSSB_FLAG_CHI_FP64)
};

__device__ __forceinline__ BFQuad bf_quad(const float* __restrict__ geom, int n_bf, int b,
                                          const Probe& p) {
    BFQuad q;
    q.kx = __ldg(geom + b);
    q.ky = __ldg(geom + n_bf + b);
    q.ak = __ldg(geom + 5 * n_bf + b);
    q.kx_lo = __ldg(geom + 6 * n_bf + b);
    q.ky_lo = __ldg(geom + 7 * n_bf + b);
    q.u = fmaf(p.mxx, q.kx, p.mxy * q.ky);
    q.v = fmaf(p.mxy, q.kx, p.myy * q.ky);
    const double kx = (double)q.kx + (double)q.kx_lo;
    const double ky = (double)q.ky + (double)q.ky_lo;
    q.ud = fma(p.mxx_d, kx, p.mxy_d * ky);
    q.vd = fma(p.mxy_d, kx, p.myy_d * ky);
    return q;
}

// Factorised C = G conj(Gamma_hat) for quadratic chi (C10, C12). With
// chi(u) = u^T M u: chi(q -+ k) = Q(q) -+ 2 q^T M k + Q(k), so
// Gamma = A(k) e^{i theta} [(A(q-k) - A(q+k)) cos Q(q) - i (A(q-k) + A(q+k)) sin Q(q)],
// theta = 2 q^T M k: one sincos per (b, q) and no polar geometry. The
// normalisation threshold is applied to |Gamma|^2 as in the reference.
template <bool CHI64>
__device__ __forceinline__ float2 corrected_quad(float qx, float qy, int r, int c, float2 eq,
                                                 const BFQuad& k, float2 g, const Probe& p) {
    const float dxm = qx - k.kx, dym = qy - k.ky;
    const float dxp = qx + k.kx, dyp = qy + k.ky;
    const float r2m = fmaf(dxm, dxm, dym * dym);
    const float r2p = fmaf(dxp, dxp, dyp * dyp);
    float am = soft_aperture(dxm, dym, r2m, p);
    float ap = soft_aperture(dxp, dyp, r2p, p);
    if (fabsf(am - ap) < kApertureTie && (in_edge_band(r2m, p) || in_edge_band(r2p, p))) {
        const double qx64 = fftfreq_d(r, p.n_r, p.qval_r);
        const double qy64 = fftfreq_d(c, p.n_c, p.qval_c);
        const double kx64 = (double)k.kx + (double)k.kx_lo;
        const double ky64 = (double)k.ky + (double)k.ky_lo;
        am = soft_aperture_fp64(qx64 - kx64, qy64 - ky64, p.semi_d, p.lam_d, p.ang_r_d, p.ang_c_d);
        ap = soft_aperture_fp64(qx64 + kx64, qy64 + ky64, p.semi_d, p.lam_d, p.ang_r_d, p.ang_c_d);
    }
    if (am == 0.0f && ap == 0.0f) return make_float2(0.0f, 0.0f);  // Gamma == 0
    const float dr = (am - ap) * eq.x;
    const float di = -(am + ap) * eq.y;
    float st, ct;
    if constexpr (CHI64) {
        const double qx64 = fftfreq_d(r, p.n_r, p.qval_r);
        const double qy64 = fftfreq_d(c, p.n_c, p.qval_c);
        __sincosf(reduce_angle(2.0 * fma(qx64, k.ud, qy64 * k.vd)), &st, &ct);
    } else {
        __sincosf(2.0f * fmaf(qx, k.u, qy * k.v), &st, &ct);
    }
    float gr = k.ak * fmaf(ct, dr, -st * di);
    float gi = k.ak * fmaf(ct, di, st * dr);
    const float m2 = fmaf(gr, gr, gi * gi);
    const float inv = m2 > 1e-16f ? rsqrtf(m2) : 1e8f;
    gr *= inv;
    gi *= inv;
    return make_float2(fmaf(g.x, gr, g.y * gi), fmaf(g.y, gr, -g.x * gi));
}

// corrected_quad (FP32 chi) with e^{i theta} supplied by the caller (a phase
// recurrence or a separable table) and the branch-free aperture. Gamma == 0
// (both apertures 0) gives m2 == 0 and C == 0 without a branch.
__device__ __forceinline__ float2 corrected_quad_e(float qx, float qy, int r, int c, float2 eq,
                                                   float kx, float ky, float ak,
                                                   const float2* lo, float2 e, float2 g,
                                                   const Probe& p) {
    // packed (re, im) / (m, p) pairs throughout; lane by lane the scalar
    // operations of the definition, so the bits do not depend on the packing
    const float2 q2 = make_float2(qx, qy), k2 = make_float2(kx, ky);
    const float2 dm = csub(q2, k2);  // q - k
    const float2 dp = cadd(q2, k2);  // q + k
    const float2 yy = __fmul2_rn(make_float2(dm.y, dp.y), make_float2(dm.y, dp.y));
    const float2 r2 = __ffma2_rn(make_float2(dm.x, dp.x), make_float2(dm.x, dp.x), yy);
    float2 a = soft_aperture_fast2(dm, dp, r2, p);
    if (fabsf(a.x - a.y) < kApertureTie && (in_edge_band(r2.x, p) || in_edge_band(r2.y, p))) {
        const float2 l = *lo;
        const double qx64 = fftfreq_d(r, p.n_r, p.qval_r);
        const double qy64 = fftfreq_d(c, p.n_c, p.qval_c);
        const double kx64 = (double)kx + (double)l.x;
        const double ky64 = (double)ky + (double)l.y;
        a.x = soft_aperture_fp64(qx64 - kx64, qy64 - ky64, p.semi_d, p.lam_d, p.ang_r_d, p.ang_c_d);
        a.y = soft_aperture_fp64(qx64 + kx64, qy64 + ky64, p.semi_d, p.lam_d, p.ang_r_d, p.ang_c_d);
    }
    // (dr, di) = ((am - ap) eq.x, -(am + ap) eq.y)
    const float2 d = __fmul2_rn(__fadd2_rn(make_float2(a.x, a.x), make_float2(-a.y, a.y)),
                                make_float2(eq.x, -eq.y));
    // (gr, gi) = ak (e.x dr - e.y di, e.x di + e.y dr)
    float2 gg = cscale(cmul(e, d), ak);
    const float m2 = fmaf(gg.x, gg.x, gg.y * gg.y);
    const float inv = m2 > 1e-16f ? rsqrtf(m2) : 1e8f;
    gg = cscale(gg, inv);
    // G conj(Gamma_hat) = (g.x gr + g.y gi, g.y gr - g.x gi)
    const float2 t = __fmul2_rn(make_float2(g.y, -g.x), make_float2(gg.y, gg.y));
    return __ffma2_rn(g, make_float2(gg.x, gg.x), t);
}

// ------------------------------------------------ 14-term Krivanek chi
// chi(u) = (2 pi / lambda) sum_i alpha^(n_i+1) C_i / (n_i+1) cos(m_i (phi - phi_i)),
// alpha = lambda |u|, phi = atan2(dy, dx) (chi_full, common.py:410-471 of the
// reference; slots C10, C12, C21, C23, C30, C32, C34, C41, C43, C45, C50, C52,
// C54, C56). Every term has n + 1 - m even, so with z = dx + i dy and
// r2 = |z|^2,
//   alpha^(n+1) cos(m (phi - phi_i)) = lambda^(n+1) r2^j Re(e^{-i m phi_i} z^m),
//   j = (n + 1 - m) / 2,
// and chi is a polynomial in (dx, dy):
//   chi = r2 (K10 + r2 (K30 + r2 K50)) + Re(sum_{m=1..6} w_m(r2) z^m),
//   w_m(r2) = sum_j K_{m,j} e^{-i m phi_{m,j}} r2^j,  K = 2 pi lambda^n C / (n + 1),
// evaluated by Horner in r2 and in z: no angle, no square root, no division.
constexpr int kFullTerms = 14;

template <typename T, typename T2>
struct FullChiT {
    T c0[3];     // r2 coefficients of the m = 0 terms: K10, K30, K50
    T2 w[6][3];  // w[m - 1][j] = K e^{-i m phi}; zero where no term exists
};
using FullChi = FullChiT<float, float2>;
using FullChi64 = FullChiT<double, double2>;

// Coefficients from magnitudes (length unit of 1 / q, as C10) and angles.
__host__ __device__ inline void make_full_chi(const float* mag, const float* ang, double wavelength,
                                              FullChi& f, FullChi64& d) {
    const int kn[kFullTerms] = {1, 1, 2, 2, 3, 3, 3, 4, 4, 4, 5, 5, 5, 5};
    const int km[kFullTerms] = {0, 2, 1, 3, 0, 2, 4, 1, 3, 5, 0, 2, 4, 6};
    for (int j = 0; j < 3; ++j) {
        d.c0[j] = 0.0;
        for (int m = 0; m < 6; ++m) d.w[m][j] = make_double2(0.0, 0.0);
    }
    for (int i = 0; i < kFullTerms; ++i) {
        const int n = kn[i];
        const int m = km[i];
        const int j = (n + 1 - m) / 2;
        double lam_n = 1.0;
        for (int e = 0; e < n; ++e) lam_n *= wavelength;
        const double k = 6.283185307179586476925 * lam_n * (double)mag[i] / (double)(n + 1);
        if (m == 0) {
            d.c0[j - 1] += k;
        } else {
            const double a = (double)m * (double)ang[i];
            d.w[m - 1][j].x += k * cos(a);
            d.w[m - 1][j].y -= k * sin(a);
        }
    }
    for (int j = 0; j < 3; ++j) {
        f.c0[j] = (float)d.c0[j];
        for (int m = 0; m < 6; ++m) f.w[m][j] = make_float2((float)d.w[m][j].x, (float)d.w[m][j].y);
    }
}

template <typename T, typename T2>
__device__ __forceinline__ T chi_full_poly(T dx, T dy, const FullChiT<T, T2>& f) {
    const T r2 = dx * dx + dy * dy;
    T sr = 0, si = 0;  // complex Horner in z over m = 6 .. 1
    auto step = [&](int m) {
        const T2* w = f.w[m - 1];
        const T wr = w[0].x + r2 * (w[1].x + r2 * w[2].x);
        const T wi = w[0].y + r2 * (w[1].y + r2 * w[2].y);
        const T tr = sr * dx - si * dy + wr;
        const T ti = sr * dy + si * dx + wi;
        sr = tr;
        si = ti;
    };
    if constexpr (sizeof(T) == 4) {
#pragma unroll
        for (int m = 6; m >= 1; --m) step(m);
    } else {
        // FP64 coefficients stay in shared memory (a rolled loop keeps them
        // from being hoisted into 72 registers)
#pragma unroll 1
        for (int m = 6; m >= 1; --m) step(m);
    }
    const T re = sr * dx - si * dy;  // Re(S z)
    return r2 * (f.c0[0] + r2 * (f.c0[1] + r2 * f.c0[2])) + re;
}

// C = G conj(Gamma_hat) (as `corrected`) with the 14-term chi at q -+ k.
// CHI64: chi from FP64 q and k (k = kx + kx_lo), reduced to [-pi, pi] in FP64.
template <bool CHI64>
__device__ __forceinline__ float2 corrected_full(float qx, float qy, int r, int c, float kx,
                                                 float ky, float kx_lo, float ky_lo, float2 pk,
                                                 float2 g, const Probe& p, const FullChi& f,
                                                 const FullChi64& fd) {
    const float dxm = qx - kx, dym = qy - ky;
    const float dxp = qx + kx, dyp = qy + ky;
    const float r2m = dxm * dxm + dym * dym;
    const float r2p = dxp * dxp + dyp * dyp;
    float am = soft_aperture(dxm, dym, r2m, p);
    float ap = soft_aperture(dxp, dyp, r2p, p);
    const bool tie = fabsf(am - ap) < kApertureTie && (in_edge_band(r2m, p) || in_edge_band(r2p, p));
    if (CHI64 || tie) {
        const double qx64 = fftfreq_d(r, p.n_r, p.qval_r);
        const double qy64 = fftfreq_d(c, p.n_c, p.qval_c);
        const double kx64 = (double)kx + (double)kx_lo;
        const double ky64 = (double)ky + (double)ky_lo;
        if (tie) {
            am = soft_aperture_fp64(qx64 - kx64, qy64 - ky64, p.semi_d, p.lam_d, p.ang_r_d, p.ang_c_d);
            ap = soft_aperture_fp64(qx64 + kx64, qy64 + ky64, p.semi_d, p.lam_d, p.ang_r_d, p.ang_c_d);
        }
        if constexpr (CHI64) {
            float s, co;
            sincosf(reduce_angle(chi_full_poly(qx64 - kx64, qy64 - ky64, fd)), &s, &co);
            const float2 pm = make_float2(am * co, -am * s);
            sincosf(reduce_angle(chi_full_poly(qx64 + kx64, qy64 + ky64, fd)), &s, &co);
            const float2 pp = make_float2(ap * co, -ap * s);
            const float t1r = fmaf(pm.x, pk.x, pm.y * pk.y);
            const float t1i = fmaf(pm.y, pk.x, -pm.x * pk.y);
            const float t2r = fmaf(pp.x, pk.x, pp.y * pk.y);
            const float t2i = fmaf(pp.x, pk.y, -pp.y * pk.x);
            float gr = t1r - t2r;
            float gi = t1i - t2i;
            const float m2 = fmaf(gr, gr, gi * gi);
            const float inv = m2 > 1e-16f ? rsqrtf(m2) : 1e8f;
            gr *= inv;
            gi *= inv;
            return make_float2(fmaf(g.x, gr, g.y * gi), fmaf(g.y, gr, -g.x * gi));
        }
    }
    float s, co;
    sincosf(chi_full_poly(dxm, dym, f), &s, &co);
    const float2 pm = make_float2(am * co, -am * s);
    sincosf(chi_full_poly(dxp, dyp, f), &s, &co);
    const float2 pp = make_float2(ap * co, -ap * s);
    const float t1r = fmaf(pm.x, pk.x, pm.y * pk.y);
    const float t1i = fmaf(pm.y, pk.x, -pm.x * pk.y);
    const float t2r = fmaf(pp.x, pk.x, pp.y * pk.y);
    const float t2i = fmaf(pp.x, pk.y, -pp.y * pk.x);
    float gr = t1r - t2r;
    float gi = t1i - t2i;
    const float m2 = fmaf(gr, gr, gi * gi);
    const float inv = m2 > 1e-16f ? rsqrtf(m2) : 1e8f;
    gr *= inv;
    gi *= inv;
    return make_float2(fmaf(g.x, gr, g.y * gi), fmaf(g.y, gr, -g.x * gi));
}

// P(k_b) with the 14-term chi from FP64 k (once per BF pixel).
__device__ __forceinline__ float2 probe_full_at_bf(double kx, double ky, float aperture,
                                                   const FullChi64& fd) {
    float s, c;
    sincosf(reduce_angle(chi_full_poly(kx, ky, fd)), &s, &c);
    return make_float2(aperture * c, -aperture * s);
}

// Kahan-compensated complex accumulation: (s.x, s.y) sums, (s.z, s.w) compensations.
__device__ __forceinline__ void kahan_add(float4& s, float2 v) {
    // (re, im) in step: y = v - c, t = sum + y, c = (t - sum) - y, sum = t
    const float2 sum = make_float2(s.x, s.y);
    const float2 y = csub(v, make_float2(s.z, s.w));
    const float2 t = cadd(sum, y);
    const float2 c = csub(csub(t, sum), y);
    s = make_float4(t.x, t.y, c.x, c.y);
}

// atan2(y, x) of the phase-variance loss: octant reduction to
// t = min(|x|, |y|) / max(|x|, |y|) in [0, 1], atan(t) = t P(t^2) with P of
// degree 8 (coefficients fitted towards the minimax error on [0, 1] by
// tests/phase_atan2_fit.py), then pi/2 - r and pi - r (constants split hi +
// lo) and the sign of y. |error| <= 4e-7 rad (rms < 1e-7) against IEEE
// atan2 for finite |x|, |y| < 2^126 (the fast divide's range; 2.4e-7 of it
// is the polynomial, the rest the divide's 2 ulp);
// atan2(+-0, +0) = +-0, atan2(+-0, -0) = +-pi; NaN in, NaN out.
__device__ __forceinline__ float phase_atan2(float y, float x) {
    const float ax = fabsf(x), ay = fabsf(y);
    const float mx = fmaxf(ax, ay), mn = fminf(ax, ay);
    const float t = mx > 0.0f ? __fdividef(mn, mx) : 0.0f;
    const float u = t * t;
    float p = 2.974573988e-03f;
    p = fmaf(p, u, -1.658112369e-02f);
    p = fmaf(p, u, 4.355344921e-02f);
    p = fmaf(p, u, -7.580571622e-02f);
    p = fmaf(p, u, 1.067893729e-01f);
    p = fmaf(p, u, -1.421420872e-01f);
    p = fmaf(p, u, 1.999413669e-01f);
    p = fmaf(p, u, -3.333316743e-01f);
    p = fmaf(p, u, 1.0f);
    float r = t * p;
    if (ay > ax) r = (1.5707963705062866f - r) + -4.371139000186243e-08f;
    if (__float_as_int(x) < 0) r = (3.1415927410125732f - r) + -8.742278000372485e-08f;
    r = copysignf(r, y);
    return (x == x && y == y) ? r : x + y;
}

}  // namespace qssb
