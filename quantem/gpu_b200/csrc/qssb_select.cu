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
#include <cooperative_groups.h>
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

// Sums NV values over the block at once (one pass of barriers); every thread
// gets the results in v. Fixed order: lane tree, then warp tree.
template <typename T, int NV>
__device__ void block_sums(T (&v)[NV], T* sh /* [NV][32] */) {
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < NV; ++j) v[j] = warp_sum(v[j]);
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int j = 0; j < NV; ++j) sh[j * 32 + warp] = v[j];
    }
    __syncthreads();
    if (warp < NV) {
        T x = lane < (int)(blockDim.x >> 5) ? sh[warp * 32 + lane] : T(0);
        x = warp_sum(x);
        if (lane == 0) sh[warp * 32] = x;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < NV; ++j) v[j] = sh[j * 32];
}

// Mean patterns up to this many pixels are cached in shared memory.
constexpr int kSelSmemPixels = 16384;

// One CTA of 32 warps. Warp w owns the contiguous pixel range
// [w*S, (w+1)*S), S a multiple of 32, read 32 consecutive pixels at a time:
// loads are coalesced and the ballot compaction keeps row-major
// (np.nonzero) order.
__global__ void __launch_bounds__(kSelThreads) k_select_bf(
    const unsigned long long* __restrict__ sums, int k0, int k1, float n_frames_f,
    float threshold, float bf_radius, float* __restrict__ mean_dp,
    int32_t* __restrict__ bf_linear, qssb_bf_info_t* __restrict__ info) {
    extern __shared__ float s_m[];  // [npix] when npix <= kSelSmemPixels
    __shared__ double sh_d[4 * 32];
    __shared__ float sh_f[32];
    __shared__ long long sh_l[4 * 32];
    __shared__ unsigned long long sh_u[32];
    __shared__ int s_off[kSelThreads / 32];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int npix = k0 * k1;
    const bool cached = npix <= kSelSmemPixels;
    const int span = ((npix + 32 * 32 - 1) / (32 * 32)) * 32;  // pixels per warp
    const int base = warp * span;
    const int end = min(base + span, npix);
    const float inv_k1 = 1.0f / (float)k1;
    // exact for npix <= 2^20: (i + 0.5) / k1 is >= 0.5 / k1 away from an integer
#define QSSB_ROW(i) __float2int_rz(((float)(i) + 0.5f) * inv_k1)
#define QSSB_VAL(i) (cached ? s_m[i] : mean_at(sums, (i), n_frames_f))

    // pass 1: mean pattern, its maximum and mean
    float vmax = -INFINITY;
    double vsum[1] = {0.0};
    for (int i = base + lane; i < end; i += 32) {
        const float m = mean_at(sums, i, n_frames_f);
        if (cached) s_m[i] = m;
        if (mean_dp) mean_dp[i] = m;
        vmax = fmaxf(vmax, m);
        vsum[0] += (double)m;
    }
    vmax = block_max(vmax, sh_f);
    block_sums(vsum, sh_d);
    const float mean_f = (float)(vsum[0] / (double)npix);
    const float thr = __fmul_rn(vmax, threshold);
    const bool auto_radius = !(bf_radius > 0.0f);

    // pass 2: mask count, variance (auto radius) or weighted centroid sums
    double dsum[3] = {0.0, 0.0, 0.0};   // auto: v2 | explicit: w, w*row, w*col
    long long lsum[3] = {0, 0, 0};      // n_mask, sum row, sum col (explicit)
    for (int i = base + lane; i < end; i += 32) {
        const float m = QSSB_VAL(i);
        const bool in_mask = m > thr;
        lsum[0] += in_mask;
        if (auto_radius) {
            const float d = __fsub_rn(m, mean_f);
            dsum[0] += (double)__fmul_rn(d, d);
        } else if (in_mask) {
            const int row = QSSB_ROW(i);
            const int col = i - row * k1;
            dsum[0] += (double)m;
            dsum[1] += (double)__fmul_rn((float)row, m);
            dsum[2] += (double)__fmul_rn((float)col, m);
            lsum[1] += row;
            lsum[2] += col;
        }
    }
    block_sums(dsum, sh_d);
    block_sums(lsum, sh_l);
    const long long n_mask = lsum[0];

    float cr, cc;  // selection centre (float32 values)
    double radius;
    if (auto_radius) {
        // probe disk: dp > mean + std; centre = its centroid, radius = sqrt(|disk| / pi)
        const float std_f = __fsqrt_rn((float)(dsum[0] / (double)npix));
        const float pthr = __fadd_rn(mean_f, std_f);
        long long c3[3] = {0, 0, 0};
        for (int i = base + lane; i < end; i += 32) {
            if (QSSB_VAL(i) > pthr) {
                const int row = QSSB_ROW(i);
                c3[0] += 1;
                c3[1] += row;
                c3[2] += i - row * k1;
            }
        }
        block_sums(c3, sh_l);
        if (c3[0] > 0) {
            cr = __fdiv_rn((float)c3[1], (float)c3[0]);
            cc = __fdiv_rn((float)c3[2], (float)c3[0]);
            radius = sqrt((double)c3[0] / 3.14159265358979323846);
        } else {
            cr = (float)(k0 / 2.0);
            cc = (float)(k1 / 2.0);
            radius = (double)min(k0, k1) * 0.25;
        }
    } else {
        const float wf = (float)dsum[0];
        if (wf > 0.0f) {
            cr = __fdiv_rn((float)dsum[1], wf);
            cc = __fdiv_rn((float)dsum[2], wf);
        } else {
            cr = (float)((double)lsum[1] / (double)max(n_mask, 1LL));
            cc = (float)((double)lsum[2] / (double)max(n_mask, 1LL));
        }
        radius = (double)bf_radius;
    }
    const float r2 = (float)(radius * radius);

    // pass 3: keep = mask && (row - cr)^2 + (col - cc)^2 <= r^2; each warp
    // counts its kept pixels, an exclusive scan over the warps gives their
    // offsets, then every warp writes its pixels in order
    auto keep = [&](int i) -> bool {
        const int row = QSSB_ROW(i);
        const float dr = __fsub_rn((float)row, cr);
        const float dc = __fsub_rn((float)(i - row * k1), cc);
        const float d2 = __fadd_rn(__fmul_rn(dr, dr), __fmul_rn(dc, dc));
        return (QSSB_VAL(i) > thr) && (d2 <= r2);
    };
    int count = 0;
    for (int i0 = base; i0 < end; i0 += 32) {
        const int i = i0 + lane;
        count += __popc(__ballot_sync(0xffffffffu, i < end && keep(i)));
    }
    if (lane == 0) s_off[warp] = count;
    __syncthreads();
    if (warp == 0) {
        const int x = s_off[lane];
        int xi = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, xi, o);
            if (lane >= o) xi += y;
        }
        s_off[lane] = xi - x;
        if (lane == 31) sh_l[0] = xi;  // total, read after the barrier
    }
    __syncthreads();
    const int n_bf = (int)sh_l[0];
    int pos = s_off[warp];
    unsigned long long dc_sum[1] = {0};
    for (int i0 = base; i0 < end; i0 += 32) {
        const int i = i0 + lane;
        const bool k = i < end && keep(i);
        const unsigned ball = __ballot_sync(0xffffffffu, k);
        if (k) {
            bf_linear[pos + __popc(ball & ((1u << lane) - 1u))] = i;
            dc_sum[0] += sums[i];
        }
        pos += __popc(ball);
    }
#undef QSSB_ROW
#undef QSSB_VAL
    block_sums(dc_sum, sh_u);
    if (threadIdx.x == 0) {
        info->n_bf = n_bf;
        info->n_mask = (int32_t)n_mask;
        info->center_row = (double)cr;
        info->center_col = (double)cc;
        info->radius = radius;
        // dc = mean over the selected pixels of G_b(0,0) = sum over frames (exact integers)
        info->dc_re = n_bf > 0 ? (double)dc_sum[0] / (double)n_bf : 0.0;
        info->dc_im = 0.0;
    }
}

// The same selection on a cluster of kSelCluster CTAs of 1024 threads. CTA r
// owns pixels [r*chunk, (r+1)*chunk) (chunk a multiple of 32, at most 4096),
// thread t the pixels r*chunk + t + 1024 k, whose mean values stay in
// registers across the passes. Every reduction is a fixed-order block
// reduction; the kSelCluster partials are exchanged through distributed
// shared memory (one slot set per phase, so one cluster barrier per exchange)
// and folded in rank order by every CTA: identical results on every CTA and
// on every launch. The compaction scans 32-pixel groups in order, so the
// output keeps row-major order.
constexpr int kSelCluster = 8;
constexpr int kSelCThreads = 1024;
constexpr int kSelPer = 4;  // pixels per thread held in registers

namespace cgx = cooperative_groups;

// After a cluster barrier: kSelCluster * NV threads fetch the ranks' slots
// into local shared memory (one remote read each), then every thread folds
// the local copy in rank order.
template <typename T, int NV>
__device__ __forceinline__ void cluster_fold(T (&v)[NV], const T* slot, T* local,
                                             cgx::cluster_group& cl) {
    if (threadIdx.x < kSelCluster * NV) {
        const int r = threadIdx.x / NV, j = threadIdx.x - (threadIdx.x / NV) * NV;
        local[threadIdx.x] = cl.map_shared_rank(slot, r)[j];
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < NV; ++j) v[j] = T(0);
    for (int r = 0; r < kSelCluster; ++r) {
#pragma unroll
        for (int j = 0; j < NV; ++j) v[j] += local[r * NV + j];
    }
}

__global__ void __cluster_dims__(kSelCluster, 1, 1) __launch_bounds__(kSelCThreads)
    k_select_bf_cluster(const unsigned long long* __restrict__ sums, int k0, int k1,
                        float n_frames_f, float threshold, float bf_radius,
                        float* __restrict__ mean_dp, int32_t* __restrict__ bf_linear,
                        qssb_bf_info_t* __restrict__ info) {
    cgx::cluster_group cl = cgx::this_cluster();
    const int rank = (int)cl.block_rank();
    __shared__ double sh_d[4 * 32];
    __shared__ float sh_f[32];
    __shared__ long long sh_l[4 * 32];
    __shared__ unsigned long long sh_u[32];
    __shared__ float slot1_f;
    __shared__ double slot1_d;
    __shared__ double slot2_d[3];
    __shared__ long long slot2_l[3];
    __shared__ long long slot3_l[3];
    __shared__ unsigned long long slot5_u;
    __shared__ int s_count;
    __shared__ double loc_d[kSelCluster * 3];
    __shared__ long long loc_l[kSelCluster * 3];
    __shared__ long long loc_l3[kSelCluster * 3];
    __shared__ float loc1_f[kSelCluster];
    __shared__ double loc1_d[kSelCluster];
    __shared__ int loc_cnt[kSelCluster];
    __shared__ int s_gcnt[kSelPer * kSelCThreads / 32];
    __shared__ int s_off[kSelCThreads / 32];
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int npix = k0 * k1;
    const int chunk = ((npix + kSelCluster * 32 - 1) / (kSelCluster * 32)) * 32;
    const int p0 = rank * chunk;
    const int p1 = min(p0 + chunk, npix);
    const float inv_k1 = 1.0f / (float)k1;
    float m[kSelPer];
    unsigned long long sv[kSelPer];
    // phase 1: mean pattern, max, mean
    float vmax = -INFINITY;
    double vsum[1] = {0.0};
#pragma unroll
    for (int k = 0; k < kSelPer; ++k) {
        const int i = p0 + tid + kSelCThreads * k;
        sv[k] = 0ULL;
        m[k] = 0.0f;
        if (i < p1) {
            sv[k] = sums[i];
            m[k] = __fdiv_rn(__ull2float_rn(sv[k]), n_frames_f);
            if (mean_dp) mean_dp[i] = m[k];
            vmax = fmaxf(vmax, m[k]);
            vsum[0] += (double)m[k];
        }
    }
    vmax = block_max(vmax, sh_f);
    block_sums(vsum, sh_d);
    if (tid == 0) {
        slot1_f = vmax;
        slot1_d = vsum[0];
    }
    cl.sync();
    if (tid < kSelCluster) {
        loc1_f[tid] = *cl.map_shared_rank(&slot1_f, tid);
        loc1_d[tid] = *cl.map_shared_rank(&slot1_d, tid);
    }
    __syncthreads();
    vmax = -INFINITY;
    double tot = 0.0;
    for (int r = 0; r < kSelCluster; ++r) {
        vmax = fmaxf(vmax, loc1_f[r]);
        tot += loc1_d[r];
    }
    const float mean_f = (float)(tot / (double)npix);
    const float thr = __fmul_rn(vmax, threshold);
    const bool auto_radius = !(bf_radius > 0.0f);
    // phase 2: mask count; variance (auto) or weighted centroid sums (explicit)
    double dsum[3] = {0.0, 0.0, 0.0};
    long long lsum[3] = {0, 0, 0};
#pragma unroll
    for (int k = 0; k < kSelPer; ++k) {
        const int i = p0 + tid + kSelCThreads * k;
        if (i >= p1) continue;
        const bool in_mask = m[k] > thr;
        lsum[0] += in_mask;
        if (auto_radius) {
            const float d = __fsub_rn(m[k], mean_f);
            dsum[0] += (double)__fmul_rn(d, d);
        } else if (in_mask) {
            const int row = __float2int_rz(((float)i + 0.5f) * inv_k1);
            const int col = i - row * k1;
            dsum[0] += (double)m[k];
            dsum[1] += (double)__fmul_rn((float)row, m[k]);
            dsum[2] += (double)__fmul_rn((float)col, m[k]);
            lsum[1] += row;
            lsum[2] += col;
        }
    }
    block_sums(dsum, sh_d);
    block_sums(lsum, sh_l);
    if (tid == 0) {
        for (int j = 0; j < 3; ++j) {
            slot2_d[j] = dsum[j];
            slot2_l[j] = lsum[j];
        }
    }
    cl.sync();
    cluster_fold(dsum, slot2_d, loc_d, cl);
    cluster_fold(lsum, slot2_l, loc_l, cl);
    const long long n_mask = lsum[0];
    float cr, cc;
    double radius;
    if (auto_radius) {
        const float std_f = __fsqrt_rn((float)(dsum[0] / (double)npix));
        const float pthr = __fadd_rn(mean_f, std_f);
        long long c3[3] = {0, 0, 0};
#pragma unroll
        for (int k = 0; k < kSelPer; ++k) {
            const int i = p0 + tid + kSelCThreads * k;
            if (i < p1 && m[k] > pthr) {
                const int row = __float2int_rz(((float)i + 0.5f) * inv_k1);
                c3[0] += 1;
                c3[1] += row;
                c3[2] += i - row * k1;
            }
        }
        block_sums(c3, sh_l);
        if (tid == 0)
            for (int j = 0; j < 3; ++j) slot3_l[j] = c3[j];
        cl.sync();
        cluster_fold(c3, slot3_l, loc_l3, cl);
        if (c3[0] > 0) {
            cr = __fdiv_rn((float)c3[1], (float)c3[0]);
            cc = __fdiv_rn((float)c3[2], (float)c3[0]);
            radius = sqrt((double)c3[0] / 3.14159265358979323846);
        } else {
            cr = (float)(k0 / 2.0);
            cc = (float)(k1 / 2.0);
            radius = (double)min(k0, k1) * 0.25;
        }
    } else {
        const float wf = (float)dsum[0];
        if (wf > 0.0f) {
            cr = __fdiv_rn((float)dsum[1], wf);
            cc = __fdiv_rn((float)dsum[2], wf);
        } else {
            cr = (float)((double)lsum[1] / (double)max(n_mask, 1LL));
            cc = (float)((double)lsum[2] / (double)max(n_mask, 1LL));
        }
        radius = (double)bf_radius;
    }
    const float r2 = (float)(radius * radius);
    // phase 4: keep flags, per-group counts, group-order scan, cluster offsets
    bool keep[kSelPer];
#pragma unroll
    for (int k = 0; k < kSelPer; ++k) {
        const int i = p0 + tid + kSelCThreads * k;
        keep[k] = false;
        if (i < p1) {
            const int row = __float2int_rz(((float)i + 0.5f) * inv_k1);
            const float dr = __fsub_rn((float)row, cr);
            const float dc = __fsub_rn((float)(i - row * k1), cc);
            const float d2 = __fadd_rn(__fmul_rn(dr, dr), __fmul_rn(dc, dc));
            keep[k] = (m[k] > thr) && (d2 <= r2);
        }
    }
    const int n_groups = (p1 > p0) ? (p1 - p0 + 31) / 32 : 0;  // group g = warp + 32 k
#pragma unroll
    for (int k = 0; k < kSelPer; ++k) {
        const int c = __popc(__ballot_sync(0xffffffffu, keep[k]));
        const int gi = warp + 32 * k;
        if (lane == 0 && gi < n_groups) s_gcnt[gi] = c;
    }
    __syncthreads();
    {
        // exclusive scan of s_gcnt[0 .. n_groups) (n_groups <= 128): warp 0..3
        const int ng = n_groups;
        int x = tid < ng ? s_gcnt[tid] : 0;
        int incl = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) s_off[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            const int wv = s_off[lane];
            int wi = wv;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, wi, o);
                if (lane >= o) wi += y;
            }
            s_off[lane] = wi - wv;
            if (lane == 31) s_count = wi;
        }
        __syncthreads();
        if (tid < ng) s_gcnt[tid] = s_off[warp] + incl - x;
    }
    cl.sync();
    if (tid < kSelCluster) loc_cnt[tid] = *cl.map_shared_rank(&s_count, tid);
    __syncthreads();
    int base = 0, total = 0;
    for (int r = 0; r < kSelCluster; ++r) {
        const int c = loc_cnt[r];
        if (r < rank) base += c;
        total += c;
    }
    unsigned long long dcs[1] = {0ULL};
#pragma unroll
    for (int k = 0; k < kSelPer; ++k) {
        const unsigned ball = __ballot_sync(0xffffffffu, keep[k]);
        if (keep[k]) {
            const int gi = warp + 32 * k;
            bf_linear[base + s_gcnt[gi] + __popc(ball & ((1u << lane) - 1u))] =
                p0 + tid + kSelCThreads * k;
            dcs[0] += sv[k];
        }
    }
    block_sums(dcs, sh_u);
    if (tid == 0) slot5_u = dcs[0];
    cl.sync();
    if (rank == 0 && tid == 0) {
        unsigned long long dc_sum = 0;
        for (int r = 0; r < kSelCluster; ++r) dc_sum += *cl.map_shared_rank(&slot5_u, r);
        info->n_bf = total;
        info->n_mask = (int32_t)n_mask;
        info->center_row = (double)cr;
        info->center_col = (double)cc;
        info->radius = radius;
        info->dc_re = total > 0 ? (double)dc_sum / (double)total : 0.0;
        info->dc_im = 0.0;
    }
    cl.sync();  // no CTA leaves while rank 0 still reads its slot
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
    const int npix = det_rows * det_cols;
    if (npix <= kSelCluster * kSelCThreads * kSelPer) {  // every pixel has a register slot
        { k_select_bf_cluster<<<kSelCluster, kSelCThreads, 0, (cudaStream_t)stream>>>(
            reinterpret_cast<const unsigned long long*>(sums), det_rows, det_cols,
            (float)n_frames, threshold, bf_radius, mean_dp, bf_linear, info); note_launch(); }
        CUDA_TRY(cudaGetLastError());
        return QSSB_OK;
    }
    const size_t smem = npix <= kSelSmemPixels ? sizeof(float) * (size_t)npix : 0;
    CUDA_TRY(cudaFuncSetAttribute(k_select_bf, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(sizeof(float) * kSelSmemPixels)));
    { k_select_bf<<<1, kSelThreads, smem, (cudaStream_t)stream>>>(
        reinterpret_cast<const unsigned long long*>(sums), det_rows, det_cols, (float)n_frames,
        threshold, bf_radius, mean_dp, bf_linear, info); note_launch(); }
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
    { k_bf_geometry<<<(capacity + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        bf_linear, info, det_cols, capacity, *params, bf_geom); note_launch(); }
    CUDA_TRY(cudaGetLastError());
    return QSSB_OK;
}
