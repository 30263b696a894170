// qssb_select.cu - bright-field selection and per-BF geometry on the device.
//
// The reference takes these small decisions on the GPU with CuPy reductions
// and reads them back (ssb/compute/cuda/backend.py:448-518,
// _compute_bf_mask_from_mean_dp; engine.py:784-830, SSBEngine.cache_rotation).
// Here they are two kernels, so a cold reconstruction needs one 48-byte
// readback (the BF count) instead of host work on the mean pattern.
//
// Precision: every float32 decision is evaluated with one IEEE rounding per
// operation (__fadd_rn, __fmul_rn, ...), the order the reference's CuPy
// element-wise kernels round in, so FMA contraction cannot move a pixel across
// a threshold. Sums feeding those decisions (mean, std, weighted centroid) are
// FP64 over a fixed thread order and rounded once to float32; integer sums are
// exact. The intensity-weighted centroid (explicit bf_radius only) can
// therefore differ from a pairwise float32 sum by a few ulps; the results
// behind atan2f / cosf / sinf (cos 2phi, sin 2phi, aperture) by an ulp or two.
#include <math.h>

#include "qssb_internal.h"

namespace qssb {

constexpr int kSelThreads = 1024;

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum in a fixed order (lane tree, then warp tree); every thread
// gets the result.
template <typename T>
__device__ T block_sum(T v, T* sh) {
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    if (warp == 0) {
        T x = lane < (int)(blockDim.x >> 5) ? sh[lane] : T(0);
        x = warp_sum(x);
        if (lane == 0) sh[0] = x;
    }
    __syncthreads();
    return sh[0];
}

__device__ float block_max(float v, float* sh) {
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    if (warp == 0) {
        float x = lane < (int)(blockDim.x >> 5) ? sh[lane] : -INFINITY;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x = fmaxf(x, __shfl_xor_sync(0xffffffffu, x, o));
        if (lane == 0) sh[0] = x;
    }
    __syncthreads();
    return sh[0];
}

__device__ __forceinline__ float mean_at(const unsigned long long* sums, int i, float n_frames_f) {
    return __fdiv_rn(__ull2float_rn(sums[i]), n_frames_f);
}

// One CTA. Each thread owns the contiguous pixel segment [t*seg, (t+1)*seg)
// so the compaction below keeps row-major (np.nonzero) order.
__global__ void __launch_bounds__(kSelThreads) k_select_bf(
    const unsigned long long* __restrict__ sums, int k0, int k1, float n_frames_f,
    float threshold, float bf_radius, float* __restrict__ mean_dp,
    int32_t* __restrict__ bf_linear, qssb_bf_info_t* __restrict__ info) {
    __shared__ double sh_d[32];
    __shared__ float sh_f[32];
    __shared__ long long sh_l[32];
    __shared__ unsigned long long sh_u[32];
    __shared__ int s_off[kSelThreads / 32];
    const int tid = threadIdx.x;
    const int npix = k0 * k1;
    const int seg = (npix + kSelThreads - 1) / kSelThreads;
    const int p0 = tid * seg;
    const int p1 = min(p0 + seg, npix);

    // mean pattern, its maximum and mean
    float vmax = -INFINITY;
    double vsum = 0.0;
    for (int i = p0; i < p1; ++i) {
        const float m = mean_at(sums, i, n_frames_f);
        if (mean_dp) mean_dp[i] = m;
        vmax = fmaxf(vmax, m);
        vsum += (double)m;
    }
    vmax = block_max(vmax, sh_f);
    vsum = block_sum(vsum, sh_d);
    const float mean_f = (float)(vsum / (double)npix);
    const float thr = __fmul_rn(vmax, threshold);

    // intensity mask (dp > max * threshold)
    long long n_mask = 0;
    for (int i = p0; i < p1; ++i) n_mask += mean_at(sums, i, n_frames_f) > thr;
    n_mask = block_sum(n_mask, sh_l);

    float cr, cc;  // selection centre (float32 values)
    double radius;
    if (!(bf_radius > 0.0f)) {
        // probe disk: dp > mean + std; centre = its centroid, radius = sqrt(|disk| / pi)
        double v2 = 0.0;
        for (int i = p0; i < p1; ++i) {
            const float d = __fsub_rn(mean_at(sums, i, n_frames_f), mean_f);
            v2 += (double)__fmul_rn(d, d);
        }
        v2 = block_sum(v2, sh_d);
        const float std_f = __fsqrt_rn((float)(v2 / (double)npix));
        const float pthr = __fadd_rn(mean_f, std_f);
        long long cnt = 0, sr = 0, sc = 0;
        for (int i = p0; i < p1; ++i) {
            if (mean_at(sums, i, n_frames_f) > pthr) {
                ++cnt;
                sr += i / k1;
                sc += i % k1;
            }
        }
        cnt = block_sum(cnt, sh_l);
        sr = block_sum(sr, sh_l);
        sc = block_sum(sc, sh_l);
        if (cnt > 0) {
            cr = __fdiv_rn((float)sr, (float)cnt);
            cc = __fdiv_rn((float)sc, (float)cnt);
            radius = sqrt((double)cnt / 3.14159265358979323846);
        } else {
            cr = (float)(k0 / 2.0);
            cc = (float)(k1 / 2.0);
            radius = (double)min(k0, k1) * 0.25;
        }
    } else {
        // explicit radius: intensity-weighted centroid of the mask
        double w = 0.0, wr = 0.0, wc = 0.0;
        long long nr = 0, nc = 0;
        for (int i = p0; i < p1; ++i) {
            const float m = mean_at(sums, i, n_frames_f);
            if (m > thr) {
                w += (double)m;
                wr += (double)__fmul_rn((float)(i / k1), m);
                wc += (double)__fmul_rn((float)(i % k1), m);
                nr += i / k1;
                nc += i % k1;
            }
        }
        w = block_sum(w, sh_d);
        wr = block_sum(wr, sh_d);
        wc = block_sum(wc, sh_d);
        nr = block_sum(nr, sh_l);
        nc = block_sum(nc, sh_l);
        const float wf = (float)w;
        if (wf > 0.0f) {
            cr = __fdiv_rn((float)wr, wf);
            cc = __fdiv_rn((float)wc, wf);
        } else {
            cr = (float)((double)nr / (double)max(n_mask, 1LL));
            cc = (float)((double)nc / (double)max(n_mask, 1LL));
        }
        radius = (double)bf_radius;
    }
    const float r2 = (float)(radius * radius);

    // keep = mask && (row - cr)^2 + (col - cc)^2 <= r^2, compacted in order
    int mine = 0;
    for (int i = p0; i < p1; ++i) {
        const float dr = __fsub_rn((float)(i / k1), cr);
        const float dc = __fsub_rn((float)(i % k1), cc);
        const float d2 = __fadd_rn(__fmul_rn(dr, dr), __fmul_rn(dc, dc));
        mine += (mean_at(sums, i, n_frames_f) > thr) && (d2 <= r2);
    }
    // exclusive scan of `mine` over the block
    const int lane = tid & 31;
    const int warp = tid >> 5;
    int incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) s_off[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const int x = lane < kSelThreads / 32 ? s_off[lane] : 0;
        int xi = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, xi, o);
            if (lane >= o) xi += y;
        }
        if (lane < kSelThreads / 32) s_off[lane] = xi - x;
    }
    __syncthreads();
    int pos = s_off[warp] + incl - mine;
    unsigned long long dc_sum = 0;
    for (int i = p0; i < p1; ++i) {
        const float dr = __fsub_rn((float)(i / k1), cr);
        const float dc = __fsub_rn((float)(i % k1), cc);
        const float d2 = __fadd_rn(__fmul_rn(dr, dr), __fmul_rn(dc, dc));
        if ((mean_at(sums, i, n_frames_f) > thr) && (d2 <= r2)) {
            bf_linear[pos++] = i;
            dc_sum += sums[i];
        }
    }
    dc_sum = block_sum(dc_sum, sh_u);
    const int n_bf = (int)block_sum((long long)mine, sh_l);
    if (tid == 0) {
        info->n_bf = n_bf;
        info->n_mask = (int32_t)n_mask;
        info->center_row = (double)cr;
        info->center_col = (double)cc;
        info->radius = radius;
        // dc = mean over the selected pixels of G_b(0,0) = sum over frames (exact integers)
        info->dc_re = n_bf > 0 ? (double)dc_sum / (double)n_bf : 0.0;
        info->dc_im = 0.0;
    }
}

// Per-BF geometry (cache_rotation, engine.py:784-830) for the n_bf pixels the
// selection wrote; rows are n_bf apart (the [8][n_bf] layout of bf_geom).
__global__ void __launch_bounds__(256) k_bf_geometry(
    const int32_t* __restrict__ bf_linear, const qssb_bf_info_t* __restrict__ info, int k1,
    int capacity, qssb_geometry_params_t gp, float* __restrict__ geom) {
    const int n = info->n_bf;
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (n > capacity || b >= n) return;  // rows are n apart: n <= capacity keeps them inside
    const int lin = bf_linear[b];
    const int row = lin / k1;
    const int col = lin - row * k1;
    const float cr = (float)info->center_row;
    const float cc = (float)info->center_col;
    const float ksr = (float)gp.k_step_row_inv_A;
    const float ksc = (float)gp.k_step_col_inv_A;
    const float cs = (float)gp.rot_cos;
    const float sn = (float)gp.rot_sin;
    const float kxa = __fmul_rn(__fsub_rn((float)row, cr), ksr);
    const float kya = __fmul_rn(__fsub_rn((float)col, cc), ksc);
    const float kx = __fadd_rn(__fmul_rn(kxa, cs), __fmul_rn(kya, sn));
    const float ky = __fadd_rn(__fmul_rn(-kxa, sn), __fmul_rn(kya, cs));
    const float kmag = __fsqrt_rn(__fadd_rn(__fmul_rn(kx, kx), __fmul_rn(ky, ky)));
    const float phi = atan2f(ky, kx);
    const float alpha = __fmul_rn(kmag, (float)gp.wavelength_A);
    const float cphi = cosf(phi);
    const float sphi = sinf(phi);
    const float t1 = __fmul_rn(cphi, (float)gp.det_sampling_row_rad);
    const float t2 = __fmul_rn(sphi, (float)gp.det_sampling_col_rad);
    const float denom = __fsqrt_rn(__fadd_rn(__fmul_rn(t1, t1), __fmul_rn(t2, t2)));
    float ap = __fadd_rn(__fdiv_rn(__fsub_rn((float)gp.semiangle_rad, alpha), denom), 0.5f);
    ap = fminf(fmaxf(ap, 0.0f), 1.0f);
    // the same k in FP64 (rounded per operation, no contraction)
    const double kr64 = __dmul_rn((double)row - (double)cr, gp.k_step_row_inv_A);
    const double kc64 = __dmul_rn((double)col - (double)cc, gp.k_step_col_inv_A);
    const double kx64 = __dadd_rn(__dmul_rn(kr64, gp.rot_cos), __dmul_rn(kc64, gp.rot_sin));
    const double ky64 = __dadd_rn(__dmul_rn(-kr64, gp.rot_sin), __dmul_rn(kc64, gp.rot_cos));
    geom[b] = kx;
    geom[n + b] = ky;
    geom[2 * n + b] = __fmul_rn(alpha, alpha);
    geom[3 * n + b] = __fsub_rn(__fmul_rn(cphi, cphi), __fmul_rn(sphi, sphi));
    geom[4 * n + b] = __fmul_rn(__fmul_rn(2.0f, sphi), cphi);
    geom[5 * n + b] = ap;
    geom[6 * n + b] = (float)(kx64 - (double)kx);
    geom[7 * n + b] = (float)(ky64 - (double)ky);
}

}  // namespace qssb

using namespace qssb;

extern "C" int qssb_select_bf(const uint64_t* sums, int32_t det_rows, int32_t det_cols,
                              int64_t n_frames, float threshold, float bf_radius,
                              float* mean_dp, int32_t* bf_linear, qssb_bf_info_t* info,
                              void* stream) {
    if (!sums || !bf_linear || !info)
        return set_error(QSSB_ERR_INVALID, "qssb_select_bf: null pointer");
    if (det_rows <= 0 || det_cols <= 0 || (int64_t)det_rows * det_cols > (1 << 20))
        return set_error(QSSB_ERR_INVALID, "qssb_select_bf: detector must have 1 .. 2^20 pixels");
    if (n_frames <= 0) return set_error(QSSB_ERR_INVALID, "qssb_select_bf: n_frames must be >= 1");
    if (!isfinite(threshold) || !isfinite(bf_radius))
        return set_error(QSSB_ERR_INVALID, "qssb_select_bf: threshold and radius must be finite");
    if (((uintptr_t)sums & 7u) != 0 || ((uintptr_t)info & 7u) != 0)
        return set_error(QSSB_ERR_INVALID, "qssb_select_bf: sums and info must be 8-byte aligned");
    k_select_bf<<<1, kSelThreads, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<const unsigned long long*>(sums), det_rows, det_cols, (float)n_frames,
        threshold, bf_radius, mean_dp, bf_linear, info);
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}

extern "C" int qssb_bf_geometry(const int32_t* bf_linear, const qssb_bf_info_t* info,
                                int32_t det_rows, int32_t det_cols, int32_t capacity,
                                const qssb_geometry_params_t* params, float* bf_geom,
                                void* stream) {
    if (!bf_linear || !info || !params || !bf_geom)
        return set_error(QSSB_ERR_INVALID, "qssb_bf_geometry: null pointer");
    if (det_rows <= 0 || det_cols <= 0 || capacity <= 0 ||
        (int64_t)capacity > (int64_t)det_rows * det_cols)
        return set_error(QSSB_ERR_INVALID,
                         "qssb_bf_geometry: capacity must be 1 .. det_rows * det_cols");
    if (!(params->k_step_row_inv_A > 0.0) || !(params->k_step_col_inv_A > 0.0) ||
        !(params->wavelength_A > 0.0) || !(params->det_sampling_row_rad > 0.0) ||
        !(params->det_sampling_col_rad > 0.0) || !isfinite(params->rot_cos) ||
        !isfinite(params->rot_sin) || !isfinite(params->semiangle_rad))
        return set_error(QSSB_ERR_INVALID, "qssb_bf_geometry: invalid geometry parameters");
    k_bf_geometry<<<(capacity + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        bf_linear, info, det_cols, capacity, *params, bf_geom);
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}
