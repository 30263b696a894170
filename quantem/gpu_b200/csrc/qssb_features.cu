// qssb_features.cu - input features of the learned aberration proposer.
//
// A feature map is the trotter amplitude |G_b(Q)| at one scan frequency Q,
// over the BF pixels b, resampled onto a fixed G x G grid in k (the aperture
// disk, |k| <= k_max in 1/A) with a separable tent of half-width h:
//   F(Q, cell) = sum_b w_b v_b,  w_b = tent(kx_b - kx_c) tent(ky_b - ky_c) / sum_b' w_b',
// then divided by its mean over covered cells (scale-free per Q). The weights
// depend only on the geometry and come in as a CSR table (cell -> pixels),
// built once per geometry on the host, so the kernel is a fixed-order gather.
// The same resampling serves
//   * inference: v_b = |G_b(Q)| from a dataset's resident Hermitian G;
//   * training:  v_b = |Gamma(Q, k_b) Phi + Gamma+(Q, k_b) Phi_a + n| from the
//     SSB forward model of a weak object (Gamma as in kernels/common.py:115-236
//     of bobleesj/quantem.gpu for its phase part, Gamma+ = P(Q-k) conj P(k) +
//     conj P(Q+k) P(k) for its amplitude part, which a strong phase object's
//     second order also feeds), Phi, Phi_a random spectrum values, n complex
//     Gaussian noise of relative level sigma (one level per map, so training
//     covers noise-dominated frequencies too).
// No counterpart in the reference (it has no learned component).
#include <cuda_bf16.h>
#include <math.h>

#include "qssb_internal.h"

namespace qssb {

constexpr int kFeatThreads = 256;
constexpr int kFeatMaxCells = 4096;  // 64 x 64

// |G_b(Q)| for Q given as fftfreq indices (row, col), any sign.
__global__ void k_values_from_g(const float2* __restrict__ g, int n_bf, int n,
                                const int32_t* __restrict__ q_idx, int n_q, float* __restrict__ vals) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    const int q = blockIdx.y;
    if (b >= n_bf || q >= n_q) return;
    const int h = n / 2 + 1;
    int r = q_idx[2 * q], c = q_idx[2 * q + 1];
    r = ((r % n) + n) % n;
    c = ((c % n) + n) % n;
    if (c >= h) {  // G(r, c) = conj G(-r, -c): same magnitude
        r = (n - r) & (n - 1);
        c = n - c;
    }
    const float2 v = g[((size_t)b * n + r) * h + c];
    vals[(size_t)q * n_bf + b] = sqrtf(fmaf(v.x, v.x, v.y * v.y));
}

// Counter-based uniform in (0, 1]: a 64-bit mix of (seed, index).
__device__ __forceinline__ float hash_uniform(unsigned long long seed, unsigned long long i) {
    unsigned long long z = seed + 0x9E3779B97F4A7C15ULL * (i + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return ((float)(z >> 40) + 1.0f) * (1.0f / 16777216.0f);
}

// Forward-model values for sample s (blockIdx.y), frequency q (blockIdx.x).
__global__ void __launch_bounds__(kFeatThreads) k_values_synth(
    const float* __restrict__ geom, int n_bf, const float* __restrict__ q_vec, int n_q,
    const qssb_aberrations_t* __restrict__ ab, const float2* __restrict__ phi,
    const float* __restrict__ sigma, qssb_calibration_t cal, unsigned long long seed,
    float* __restrict__ vals) {
    __shared__ Probe sp;
    const int q = blockIdx.x;
    const int s = blockIdx.y;
    if (threadIdx.x == 0) {
        const qssb_aberrations_t a = ab[s];
        sp = make_probe_common(cal, a.C10, a.C12, a.phi12, a.C30);
    }
    __syncthreads();
    const Probe& p = sp;
    const float qx = q_vec[2 * q], qy = q_vec[2 * q + 1];
    const float2 f = phi[2 * ((size_t)s * n_q + q)];       // phase-object spectrum
    const float2 fa = phi[2 * ((size_t)s * n_q + q) + 1];  // amplitude-object spectrum
    const float sg = sigma[(size_t)s * n_q + q] * sqrtf(fmaf(f.x, f.x, f.y * f.y));
    for (int b = threadIdx.x; b < n_bf; b += kFeatThreads) {
        const float kx = geom[b], ky = geom[n_bf + b];
        const float2 pk = probe_at_bf<false>(geom[2 * n_bf + b], geom[3 * n_bf + b],
                                             geom[4 * n_bf + b], geom[5 * n_bf + b], p);
        const Disp dm = displacement(qx - kx, qy - ky, p);
        const Disp dp = displacement(qx + kx, qy + ky, p);
        const float2 pm = probe_from<false>(dm, soft_aperture(qx - kx, qy - ky, dm.r2, p), p);
        const float2 pp = probe_from<false>(dp, soft_aperture(qx + kx, qy + ky, dp.r2, p), p);
        // t1 = P(q-k) conj P(k), t2 = conj P(q+k) P(k); a phase object couples
        // through Gamma = t1 - t2, an amplitude object through t1 + t2
        const float t1r = fmaf(pm.x, pk.x, pm.y * pk.y), t1i = fmaf(pm.y, pk.x, -pm.x * pk.y);
        const float t2r = fmaf(pp.x, pk.x, pp.y * pk.y), t2i = fmaf(pp.x, pk.y, -pp.y * pk.x);
        const float gr = t1r - t2r, gi = t1i - t2i;
        const float hr = t1r + t2r, hi = t1i + t2i;
        float vr = gr * f.x - gi * f.y + hr * fa.x - hi * fa.y;
        float vi = gr * f.y + gi * f.x + hr * fa.y + hi * fa.x;
        const unsigned long long id =
            (((unsigned long long)s * n_q + q) * (unsigned long long)n_bf + b) * 2ULL;
        const float u1 = hash_uniform(seed, id), u2 = hash_uniform(seed, id + 1);
        const float rad = sqrtf(-2.0f * logf(u1));
        float sn, cs;
        sincospif(2.0f * u2, &sn, &cs);
        vr = fmaf(sg * rad, cs, vr);
        vi = fmaf(sg * rad, sn, vi);
        vals[((size_t)s * n_q + q) * n_bf + b] = sqrtf(fmaf(vr, vr, vi * vi));
    }
}

// Resample + normalise: one CTA per (q, sample); thread t owns cells t, t+256,
// ...; covered cells (non-empty CSR rows) set the mean.
__global__ void __launch_bounds__(kFeatThreads) k_resample(
    const float* __restrict__ vals, int n_bf, int n_q, const int32_t* __restrict__ off,
    const int32_t* __restrict__ idx, const float* __restrict__ w, int cells,
    float* __restrict__ out_f32, __nv_bfloat16* __restrict__ out_bf16) {
    __shared__ float red_s[kFeatThreads / 32], red_n[kFeatThreads / 32];
    constexpr int kPer = kFeatMaxCells / kFeatThreads;
    const int q = blockIdx.x;
    const int s = blockIdx.y;
    const int tid = threadIdx.x;
    const float* v = vals + ((size_t)s * n_q + q) * n_bf;
    float acc[kPer];
    float tot = 0.0f, cnt = 0.0f;
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
        acc[j] = 0.0f;
        const int cell = tid + kFeatThreads * j;
        if (cell >= cells) continue;
        const int e0 = off[cell], e1 = off[cell + 1];
        float a = 0.0f;
        for (int e = e0; e < e1; ++e) a = fmaf(w[e], __ldg(v + idx[e]), a);
        acc[j] = a;
        if (e1 > e0) {
            tot += a;
            cnt += 1.0f;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        tot += __shfl_xor_sync(0xffffffffu, tot, o);
        cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    }
    if ((tid & 31) == 0) {
        red_s[tid >> 5] = tot;
        red_n[tid >> 5] = cnt;
    }
    __syncthreads();
    float all = 0.0f, alln = 0.0f;
    for (int k = 0; k < kFeatThreads / 32; ++k) {
        all += red_s[k];
        alln += red_n[k];
    }
    const float mean = alln > 0.0f ? all / alln : 0.0f;
    const float inv_mean = mean > 0.0f ? 1.0f / mean : 0.0f;
    const size_t base = ((size_t)s * n_q + q) * cells;
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
        const int cell = tid + kFeatThreads * j;
        if (cell >= cells) continue;
        const float fv = acc[j] * inv_mean;
        if (out_f32) out_f32[base + cell] = fv;
        if (out_bf16) out_bf16[base + cell] = __float2bfloat16_rn(fv);
    }
}

static int check_csr(const int32_t* off, const int32_t* idx, const float* w, int cells) {
    if (!off || !idx || !w) return set_error(QSSB_ERR_INVALID, "features: null resampling table");
    if (cells < 1 || cells > kFeatMaxCells)
        return set_error(QSSB_ERR_INVALID, "features: cells must be 1..4096");
    return QSSB_OK;
}

}  // namespace qssb

using namespace qssb;

extern "C" int qssb_trotter_features(const float* g_half, int32_t n_bf, int32_t scan_n,
                                     const int32_t* q_idx, int32_t n_q, const int32_t* csr_off,
                                     const int32_t* csr_idx, const float* csr_w, int32_t cells,
                                     float* scratch, float* out_f32, void* out_bf16, void* stream) {
    if (!g_half || !q_idx || !scratch || (!out_f32 && !out_bf16))
        return set_error(QSSB_ERR_INVALID, "qssb_trotter_features: null pointer");
    if (n_bf <= 0 || n_q <= 0 || n_q > 65535 || (scan_n != 64 && scan_n != 128 && scan_n != 256))
        return set_error(QSSB_ERR_INVALID, "qssb_trotter_features: bad n_bf, n_q or scan size");
    int rc = check_csr(csr_off, csr_idx, csr_w, cells);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    { k_values_from_g<<<dim3((n_bf + 255) / 256, n_q), 256, 0, s>>>(
        reinterpret_cast<const float2*>(g_half), n_bf, scan_n, q_idx, n_q, scratch); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    { k_resample<<<dim3(n_q, 1), kFeatThreads, 0, s>>>(scratch, n_bf, n_q, csr_off, csr_idx, csr_w,
                                                      cells, out_f32,
                                                      static_cast<__nv_bfloat16*>(out_bf16)); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}

extern "C" int qssb_synth_features(const float* bf_geom, int32_t n_bf, const float* q_vec,
                                   int32_t n_q, const qssb_aberrations_t* aberrations,
                                   const float* phi, const float* sigma, int32_t n_samples,
                                   const qssb_calibration_t* cal, uint64_t seed,
                                   const int32_t* csr_off, const int32_t* csr_idx,
                                   const float* csr_w, int32_t cells, float* scratch,
                                   float* out_f32, void* out_bf16, void* stream) {
    if (!bf_geom || !q_vec || !aberrations || !phi || !sigma || !cal || !scratch ||
        (!out_f32 && !out_bf16))
        return set_error(QSSB_ERR_INVALID, "qssb_synth_features: null pointer");
    if (n_bf <= 0 || n_q <= 0 || n_q > 65535 || n_samples <= 0 || n_samples > 65535)
        return set_error(QSSB_ERR_INVALID, "qssb_synth_features: bad n_bf, n_q or n_samples");
    int rc = check_csr(csr_off, csr_idx, csr_w, cells);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    { k_values_synth<<<dim3(n_q, n_samples), kFeatThreads, 0, s>>>(
        bf_geom, n_bf, q_vec, n_q, aberrations, reinterpret_cast<const float2*>(phi), sigma, *cal,
        (unsigned long long)seed, scratch); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    { k_resample<<<dim3(n_q, n_samples), kFeatThreads, 0, s>>>(
        scratch, n_bf, n_q, csr_off, csr_idx, csr_w, cells, out_f32,
        static_cast<__nv_bfloat16*>(out_bf16)); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}
