/*
 * qssb.h - C ABI of the B200-native single-sideband (SSB) ptychography engine.
 *
 * Every entry point is a plain C function: raw device pointers, sizes and a
 * cudaStream_t passed as void*. No PyTorch or CuPy types cross this boundary.
 * Each returns QSSB_OK (0) or a negative QSSB_ERR_* code and never aborts;
 * qssb_last_error() gives a message for the calling thread's last failure.
 * All kernels are enqueued on the given stream; nothing synchronises it.
 *
 * The entry points replace the device work of the reference backend
 * (bobleesj/quantem.gpu 0.0.1rc6, src/quantem/gpu/ssb/compute/cuda/), as
 * cited on each declaration. Complex arrays are interleaved float32 pairs
 * (complex64); the Hermitian spectrum layout is the reference's
 * G_qk[n_bf][scan_rows][scan_cols/2 + 1].
 */
#ifndef QSSB_H
#define QSSB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QSSB_VERSION 1

#define QSSB_OK 0
#define QSSB_ERR_INVALID (-1)     /* bad argument, shape, alignment or size */
#define QSSB_ERR_CUDA (-2)        /* a CUDA launch or runtime call failed */
#define QSSB_ERR_UNSUPPORTED (-3) /* valid request this build cannot serve */
#define QSSB_ERR_WORKSPACE (-4)   /* workspace smaller than the query said */

/* Flags for qssb_object / qssb_loss_batch. */
#define QSSB_FLAG_CHI_FP64 1      /* chi polynomial and its 2*pi reduction in FP64 */
#define QSSB_FLAG_FULL_PLANE 2    /* evaluate every scan frequency; no +-q symmetry */
#define QSSB_FLAG_QUADRATIC 4     /* qssb_loss_batch: every candidate has C30 == 0, so the
                                     factorised quadratic-chi overlap applies (qssb_object
                                     decides this itself from its host-side candidate) */
#define QSSB_FLAG_PERSISTENT 8    /* qssb_loss_batch at 256^2 (float32 chi): one persistent
                                     launch runs every row and column item of the batch
                                     instead of a row and a column launch per BF chunk
                                     (the same plan; the same bits with
                                     QSSB_FLAG_QUADRATIC, float32 rounding without;
                                     within 3% of the sequence's time) */
/* Tile-shape variant (another tuning knob): bits 8..11 of flags. qssb_object
 * on the quadratic-chi path: 1 = 2 adjacent frequencies per thread, 2 or 0
 * (the default) = 4, 3 = 8. Results agree to float32 rounding across
 * variants; each variant repeats its own bits. */
#define QSSB_FLAG_VARIANT_SHIFT 8
#define QSSB_FLAG_VARIANT(v) ((int32_t)(v) << QSSB_FLAG_VARIANT_SHIFT)
#define QSSB_FLAG_VARIANT_MAX 15
/* Work partition (the tuning knob of an autotuner): bits 16..30 of flags hold
 * the number of BF chunks - per candidate for qssb_loss_batch, in total for
 * qssb_object. 0 keeps the built-in plan. Any value gives the same result up
 * to float32 summation order, and the same bits on every repeat of that value;
 * query the workspace with the same flags. */
#define QSSB_FLAG_CHUNKS_SHIFT 16
#define QSSB_FLAG_CHUNKS(n) ((int32_t)(n) << QSSB_FLAG_CHUNKS_SHIFT)
#define QSSB_FLAG_CHUNKS_MAX 32767

/* Calibration shared by the object and loss entry points. Scalars follow
 * SSBEngine's cache (engine.py:784-848): wavelength in Angstrom, angles in
 * radians, the per-axis detector angular sampling in radians per pixel, the
 * scan step in Angstrom. The float32 kernels use these rounded to float32,
 * as the reference passes them (np.float32 kernel arguments); the FP64
 * aperture evaluation at near-tied overlaps uses them as given. */
typedef struct qssb_calibration {
    int32_t n_bf;                 /* selected BF pixels (B), >= 1 */
    int32_t scan_rows;            /* R0: 64, 128, 256, 512 or 1024 */
    int32_t scan_cols;            /* R1: == scan_rows */
    int32_t reserved;             /* must be 0 */
    double wavelength_A;
    double semiangle_rad;
    double det_sampling_row_rad;  /* reference "ang_y" */
    double det_sampling_col_rad;  /* reference "ang_x" */
    double scan_sampling_row_A;   /* q_row = fftfreq(R0, scan_sampling_row_A) */
    double scan_sampling_col_A;
    double dc_re;                 /* dc = mean_b G_b(0,0) (backend.py:587) */
    double dc_im;
} qssb_calibration_t;

/* Layout of bf_geom (device float32 [8][n_bf]): rows 0-5 are cache_rotation's
 * kx, ky, alpha_k2, cos2phi_k, sin2phi_k, aperture_k (engine.py:784-830, in
 * float32 like the reference); rows 6-7 are kx_lo, ky_lo with
 * kx_fp64 = (double)kx + (double)kx_lo. */
#define QSSB_GEOM_ROWS 8

/* One aberration candidate in the reference's numeric convention: C10, C12
 * and C30 enter chi as Angstrom values, phi12 in radians
 * (engine.py:217-231, common.py:410-471 slot 4 for C30). */
typedef struct qssb_aberrations {
    float C10;
    float C12;
    float phi12;
    float C30;
} qssb_aberrations_t;

int qssb_version(void);
const char* qssb_last_error(void);
/* Kernel launches this library has made in this process, all threads and
 * devices (launches recorded into a CUDA graph count once, at capture; its
 * replays run them again without host calls). No reference counterpart: the
 * count behind the bench's launch figures. */
int64_t qssb_kernel_launches(void);

/* Mean diffraction pattern: sums[k] = sum over frames of counts[f][k] in
 * exact u64 arithmetic, mean_dp[k] = float32(sums[k]) / n_frames (IEEE
 * round-to-nearest). Replaces CudaSSBBackend._compute_bf_mask's reduction
 * (backend.py:432-441) and probe.mean_dp (detector/compute/cuda/probe.py:
 * 122-147). counts: [n_frames][det_pixels] u16; sums: [det_pixels]
 * (overwritten); mean_dp: [det_pixels] or NULL. */
int qssb_mean_dp_u64(const uint16_t* counts, int64_t n_frames, int32_t det_pixels,
                     uint64_t* sums, float* mean_dp, void* stream);

/* BF-column gather: columns[b][f] = counts[f][bf_linear[b]] (exact u16).
 * Replaces the fancy-index + transpose of _extract_gqk (backend.py:561-572).
 * bf_linear: device int32 [n_bf], each in [0, det_pixels). */
int qssb_gather_bf_columns(const uint16_t* counts, int64_t n_frames, int32_t det_pixels,
                           const int32_t* bf_linear, int32_t n_bf, uint16_t* columns,
                           void* stream);

/* Result of qssb_select_bf (device memory, written by the kernel). */
typedef struct qssb_bf_info {
    int32_t n_bf;        /* selected BF pixels B (0: nothing selected) */
    int32_t n_mask;      /* pixels with mean_dp > max(mean_dp) * threshold */
    double center_row;   /* selection centre in detector pixels (float32 values) */
    double center_col;
    double radius;       /* selection radius in pixels */
    double dc_re;        /* dc = mean over the B pixels of their exact frame sums */
    double dc_im;        /* 0 (the scan images are real) */
} qssb_bf_info_t;

/* Bright-field selection from the exact frame sums (the reference's
 * _compute_bf_mask_from_mean_dp, backend.py:448-518, and the dc of
 * _extract_gqk, backend.py:587): mean_dp = float32(sums) / n_frames; mask =
 * mean_dp > max(mean_dp) * threshold; with bf_radius <= 0 the probe disk
 * mean_dp > mean + std gives the centre (its centroid) and the radius
 * sqrt(|disk| / pi), otherwise the centre is the intensity-weighted centroid
 * of the mask and the radius bf_radius; the kept pixels are the mask pixels
 * within the radius, in row-major order. sums: device u64 [det_rows*det_cols];
 * mean_dp: device float32 [det_rows*det_cols] or NULL; bf_linear: device
 * int32 with room for det_rows*det_cols entries (the first info->n_bf are
 * written); info: device. One CTA; nothing is read back. */
int qssb_select_bf(const uint64_t* sums, int32_t det_rows, int32_t det_cols, int64_t n_frames,
                   float threshold, float bf_radius, float* mean_dp, int32_t* bf_linear,
                   qssb_bf_info_t* info, void* stream);

/* Detector-to-k calibration of qssb_bf_geometry. rot_cos / rot_sin are
 * cos(-theta) and sin(-theta) of the scan rotation theta (the passive
 * rotation of engine.py:800-805). */
typedef struct qssb_geometry_params {
    double k_step_row_inv_A;      /* detector pixel pitch in 1/A: 1 / (sampling_row * det_rows) */
    double k_step_col_inv_A;
    double rot_cos;
    double rot_sin;
    double wavelength_A;
    double semiangle_rad;
    double det_sampling_row_rad;
    double det_sampling_col_rad;
} qssb_geometry_params_t;

/* Per-BF geometry of SSBEngine.cache_rotation (engine.py:784-830) for the
 * info->n_bf pixels of bf_linear, relative to info's centre, written as
 * bf_geom [QSSB_GEOM_ROWS][n_bf] (rows n_bf floats apart; bf_geom must hold
 * QSSB_GEOM_ROWS * capacity floats, capacity >= n_bf, else nothing is
 * written). Needs no host copy of n_bf: launch it right after qssb_select_bf. */
int qssb_bf_geometry(const int32_t* bf_linear, const qssb_bf_info_t* info, int32_t det_rows,
                     int32_t det_cols, int32_t capacity, const qssb_geometry_params_t* params,
                     float* bf_geom, void* stream);

/* The same gather with the detector shape known: reads each frame's BF
 * bounding box with 16-byte loads (det_cols a multiple of 8, counts and
 * columns 16-byte aligned; otherwise it runs qssb_gather_bf_columns). */
int qssb_gather_bf_columns_2d(const uint16_t* counts, int64_t n_frames, int32_t det_rows,
                              int32_t det_cols, const int32_t* bf_linear, int32_t n_bf,
                              uint16_t* columns, void* stream);
/* The same with the tile shape named (the autotuner's knob; every variant
 * copies the same bits): 0 = the built-in rule above; bounding-box tiles of
 * (frames x band pixels) 1 = 32 x 768, 2 = 16 x 1536, 3 = 64 x 384,
 * 4 = 8 x 3072; 64-frame pixel-major tiles of 5 = 320 and 6 = 704 band pixels
 * (5 and 6 need n_frames % 8 == 0, else the built-in rule applies). */
int qssb_gather_bf_columns_2d_ex(const uint16_t* counts, int64_t n_frames, int32_t det_rows,
                                 int32_t det_cols, const int32_t* bf_linear, int32_t n_bf,
                                 uint16_t* columns, int32_t variant, void* stream);

/* Largest count of a whole loaded block of n u8 (elem_bytes 1) or u16
 * (elem_bytes 2) detector counts, written to the device word *max_out (set
 * to 0 first, on the stream). Replaces the cp.max(data) that decides whether
 * the exact BF companion may be narrowed to u8 (engine.py:603-604). */
int qssb_count_max(const void* counts, int32_t elem_bytes, int64_t n, uint32_t* max_out,
                   void* stream);

/* Exact BF companion columns: out[b][f] = (out type) counts[f][bf_linear[b]]
 * for b < n_bf, f < n_scan; counts u8/u16 [n_scan][det_pixels] (in_bytes 1/2),
 * out u8/u16 [n_bf][n_scan] (out_bytes 1/2). Narrowing u16 to u8 keeps the
 * low byte, so callers narrow only when qssb_count_max says the block fits.
 * An index outside [0, det_pixels) writes 0. Replaces the gather_transpose
 * RawKernel of write_exact_bf_source (engine.py:620-660); callers pass a
 * chunk's bf_linear + offset and its output rows. */
int qssb_export_bf_columns(const void* counts, int32_t in_bytes, int64_t n_scan,
                           int64_t det_pixels, const int32_t* bf_linear, int32_t n_bf, void* out,
                           int32_t out_bytes, void* stream);

/* Forward scan FFT of each BF image, Hermitian half plane:
 * g_half[b][r][c] = sum_R columns[b][R] exp(-2 pi i (r R_r/R0 + c R_c/R1)),
 * c in [0, R1/2]. Replaces cp.fft.fft2 + the half-plane slice of
 * _extract_gqk (backend.py:573-585). columns: u16 [n_bf][R0*R1];
 * g_half: complex64 [n_bf][R0][R1/2+1]. */
int qssb_scan_fft_half(const uint16_t* columns, int32_t n_bf, int32_t scan_rows,
                       int32_t scan_cols, float* g_half, void* stream);
/* The same with the launch shape named (the autotuner's knob; every variant
 * gives the same bits): 0 = built-in, 1 .. qssb_scan_fft_variants(scan_rows).
 * 128: persistent CTAs per SM, 1 = two (built-in), 2 = one. 256 / 512 / 1024:
 * the column pass's (columns per strip = warps per CTA, CTAs per SM) -
 * 256: 1 = (8, 3) built-in, 2 = (16, 1), 3 = (8, 2), 4 = (16, 2);
 * 512: 1 = (16, 1) built-in, 2 = (8, 1), 3 = (8, 2); 1024: 1 = (8, 1)
 * built-in, 2 = (4, 2). 64: one shape. */
int qssb_scan_fft_half_ex(const uint16_t* columns, int32_t n_bf, int32_t scan_rows,
                          int32_t scan_cols, float* g_half, int32_t variant, void* stream);
int qssb_scan_fft_variants(int32_t scan_rows, int32_t* count);

/* The BF columns written by the frame-sum pass (no counterpart as one step in
 * the reference, whose _extract_gqk gathers after the selection,
 * backend.py:520-589). A cold reconstruction then reads the counts once:
 *
 * qssb_bf_box_estimate: from u64 sums of some frames (e.g. the first 512, by
 * qssb_mean_dp_u64 on that prefix), a superset box of the BF disk: the
 * bounding box of the pixels at >= 1/4 of the largest sum (or, with
 * radius_px > 0, their centroid +- radius_px), widened by margin, columns
 * rounded out to multiples of 8. box: device int32[8] = r0, r1, c0, c1
 * (half-open), width, pixel count, valid (pixel count <= capacity), unused. */
int qssb_bf_box_estimate(const uint64_t* sums, int32_t det_rows, int32_t det_cols,
                         float radius_px, int32_t margin, int64_t capacity, int32_t* box,
                         void* stream);

/* qssb_mean_dp_u64 (sums only) that also writes, when the box is valid and
 * consistent (inside the detector, 8-pixel columns, at most capacity
 * pixels), the box's columns box_cols[(r - r0) * width + (c - c0)][f] =
 * counts[f][r][c] (u16, capacity x n_frames). det_cols and n_frames multiples
 * of 8, counts and box_cols 16-byte aligned. */
int qssb_mean_dp_u64_box(const uint16_t* counts, int64_t n_frames, int32_t det_rows,
                         int32_t det_cols, uint64_t* sums, const int32_t* box, int64_t capacity,
                         uint16_t* box_cols, void* stream);

/* After qssb_select_bf: map[b] = box column of BF pixel b (-1 outside the
 * box) for b < min(n_bf, capacity), and *ok = 1 when every BF pixel lies in
 * a valid box of at most box_capacity pixels (else the caller gathers with
 * qssb_gather_bf_columns_2d). */
int qssb_bf_box_map(const int32_t* bf_linear, const qssb_bf_info_t* info, int32_t det_rows,
                    int32_t det_cols, int32_t capacity, int64_t box_capacity,
                    const int32_t* box, int32_t* map, int32_t* ok, void* stream);

/* qssb_scan_fft_half for 128x128 scans reading BF pixel b's image from
 * column map[b] of the n_cols columns [n_cols][R0*R1] (the box columns);
 * map entries must come from a qssb_bf_box_map whose ok flag was set. */
int qssb_scan_fft_half_mapped(const uint16_t* columns, int64_t n_cols, const int32_t* map,
                              int32_t n_bf, int32_t scan_rows, int32_t scan_cols, float* g_half,
                              void* stream);

/* Workspace bytes needed by qssb_object for this calibration. */
int qssb_object_workspace_bytes(const qssb_calibration_t* cal, int32_t flags, size_t* bytes);

/* Object wave O = ifft2((1/B) sum_b G_b conj(Gamma_hat_b)), DC := dc, and
 * phase = atan2(Im O, Re O). Replaces SSBEngine.reconstruct_object
 * (engine.py:1109-1151; identical by IFFT linearity to its per-BF fused
 * path K5+K6+K7+mean, and to _reconstruct_object_fourier_sum,
 * engine.py:1047-1107). bf_geom: device float32 [QSSB_GEOM_ROWS][n_bf]
 * (layout above); q_row/q_col: device float32 fftfreq grids; object: complex64 [R0][R1];
 * phase: float32 [R0][R1] or NULL. */
int qssb_object(const float* g_half, const float* bf_geom, const float* q_row,
                const float* q_col, const qssb_calibration_t* cal,
                const qssb_aberrations_t* ab, int32_t flags, void* workspace,
                size_t workspace_bytes, float* object, float* phase, void* stream);

/* qssb_object with dc read from device memory at run time: dc_device points
 * to two doubles (re, im) - e.g. &info->dc_re of a qssb_bf_info_t written by
 * qssb_select_bf - or is NULL to use cal->dc_re/dc_im. Lets a captured CUDA
 * graph serve datasets whose dc differs. */
int qssb_object_ex(const float* g_half, const float* bf_geom, const float* q_row,
                   const float* q_col, const qssb_calibration_t* cal,
                   const qssb_aberrations_t* ab, int32_t flags, const double* dc_device,
                   void* workspace, size_t workspace_bytes, float* object, float* phase,
                   void* stream);

/* Capacity of the fixed device scratch used by qssb_object_noalloc. */
#define QSSB_NOALLOC_SCRATCH_BYTES (16u << 20)

/* qssb_object without a workspace argument and without allocating: for
 * callers that cannot allocate device memory where they call us - a host
 * application whose own memory pool already owns the whole device, a
 * real-time acquisition loop that must not enter the CUDA allocator (an
 * allocation can synchronise the device and stall the stream), or a plugin
 * host that forbids third-party allocations. No counterpart in the reference
 * (its CuPy engine always allocates through CuPy's memory pool).
 *
 * The scratch (partial Fourier sums and the spectrum plane) is one
 * QSSB_NOALLOC_SCRATCH_BYTES (16 MiB) array inside this library; every GPU
 * that loads the library holds it until the process exits. Requests whose
 * qssb_object_workspace_bytes exceed it fail with QSSB_ERR_WORKSPACE (up to
 * 63488 BF pixels fit at 128^2 scans, 15616 at 256^2).
 * The first call on each device looks up the array's device address and
 * keeps it; make that first call before any stream capture. The kept address
 * belongs to the device's current primary context: after cudaDeviceReset (or
 * anything else that destroys that context) it is stale, so a process that
 * resets a device must not call this entry on it again. All calls share the one array:
 * calls whose work overlaps on the GPU (other streams, other host threads)
 * race and corrupt each other's results, so serialise them. Each call writes
 * every scratch byte it reads, so nothing has to be cleared between calls.
 * Arguments and results are those of qssb_object. */
int qssb_object_noalloc(const float* g_half, const float* bf_geom, const float* q_row,
                        const float* q_col, const qssb_calibration_t* cal,
                        const qssb_aberrations_t* ab, int32_t flags, float* object,
                        float* phase, void* stream);

/* Workspace bytes needed by qssb_loss_batch for n_cand candidates. */
int qssb_loss_workspace_bytes(const qssb_calibration_t* cal, int32_t n_cand, int32_t flags,
                              size_t* bytes);

/* Phase-variance loss for n_cand candidates in one launch sequence:
 * phi_b = atan2(ifft2(C_b)), L = mean_R[(1/B) sum phi_b^2 - ((1/B) sum phi_b)^2].
 * Replaces SSBEngine.reconstruct_with_loss (engine.py:1464-1514) and
 * variance_loss_batch (engine.py:2120-2295). candidates: DEVICE array of
 * n_cand qssb_aberrations_t; losses: device float32 [n_cand];
 * mean_phase: device float32 [n_cand][R0][R1] (mean over b of phi_b) or NULL.
 * The per-candidate reduction order is fixed: repeated calls return
 * identical bits. */
int qssb_loss_batch(const float* g_half, const float* bf_geom, const float* q_row,
                    const float* q_col, const qssb_calibration_t* cal,
                    const qssb_aberrations_t* candidates, int32_t n_cand, int32_t flags,
                    void* workspace, size_t workspace_bytes, float* losses,
                    float* mean_phase, void* stream);

/* Registers a cancel flag: a device int32 (device memory, or pinned host
 * memory mapped into the device address space for a live cancel) that the
 * table-driven loss kernel (qssb_loss_batch_ex with a table) reads once per
 * BF-pixel pair. Nonzero stops every CTA at its next pair; the batch's losses
 * come back NaN. NULL unregisters. The pointer is a launch argument, so a
 * CUDA graph keeps the one registered when it was captured. The reference
 * cancels a remote job between stages (remote/ssb_api.py:624-679); this
 * reaches into a running loss batch. The kernels have no unbounded loop: a
 * flag that is never set changes nothing. */
int qssb_set_cancel(const int32_t* flag);

/* Bytes of the overlap table of a square scan of side N: float2 [n_bf][E],
 * E = 8383 at N = 128, (N/2 + 1) N + N/2 at N = 256, 512, 1024 (1.05 MB per
 * BF pixel at 512, 4.2 MB at 1024: check the size against the device). */
int qssb_overlap_table_bytes(const qssb_calibration_t* cal, size_t* bytes);

/* The candidate-independent part of the overlap, the aperture pair
 * table[b][e] = (A(q - k_b), A(q + k_b)) at the frequencies the loss
 * evaluates, with the loss kernels' aperture rule (FP64 where the two
 * apertures tie in the soft edge). N = 128: the half set (rows 0..64 x all
 * columns, then (127 - j, 64) for j < 63) in the pair kernel's order; N >= 256:
 * the two-pass row kernel's, rows 0 .. N/2 x all N columns row-major, then
 * at (N/2 + 1) N + r the partner (N - r, N/2) of its Nyquist-column relation
 * (r = 1 .. N/2 - 1). The reference recomputes these apertures for every
 * candidate inside gamma_mul_pk_onthefly (common.py:115-236); computing them
 * once per dataset is this engine's own step. Depends on the geometry only:
 * rebuild after cache_rotation. */
int qssb_overlap_table(const float* bf_geom, const float* q_row, const float* q_col,
                       const qssb_calibration_t* cal, float* table, void* stream);

/* qssb_loss_batch with an optional overlap table (NULL: as qssb_loss_batch).
 * With a table and 128x128 scans (symmetric half set, i.e. without
 * QSSB_FLAG_FULL_PLANE) the loss runs two BF pixels per inverse 2D FFT (their
 * anti-Hermitian parts packed as one complex plane, the Hermitian DC and
 * Nyquist-line parts transformed on their own) with the apertures read from
 * the table: for QSSB_FLAG_QUADRATIC batches through the factorised overlap,
 * otherwise (C30) through the direct probe phases. With a table and 256 .. 1024
 * scans, the row pass of QSSB_FLAG_QUADRATIC batches (without
 * QSSB_FLAG_CHI_FP64) reads the apertures instead of evaluating them; other
 * batches there ignore the table. The workspace is the same. The reduction
 * order is fixed for a given plan; the result differs from the table-free path
 * by float32 rounding only. */
int qssb_loss_batch_ex(const float* g_half, const float* bf_geom, const float* q_row,
                       const float* q_col, const qssb_calibration_t* cal,
                       const qssb_aberrations_t* candidates, int32_t n_cand, int32_t flags,
                       const float* overlap, void* workspace, size_t workspace_bytes,
                       float* losses, float* mean_phase, void* stream);

/* The phase function of qssb_loss_batch and qssb_loss_batch_full:
 * out[i] = atan2(y[i], x[i]) by an octant reduction and a degree-17 odd
 * polynomial, |error| <= 4e-7 rad against IEEE atan2 for finite
 * |x|, |y| < 2^126, signed zeros and NaN as IEEE atan2. The reference's loss
 * takes cupy.angle (engine.py:2120-2295); this entry exposes the GPU
 * replacement so its error can be checked. y, x, out: device float32 [n]. */
int qssb_phase_atan2(const float* y, const float* x, float* out, int64_t n, void* stream);

/* The 14 Krivanek coefficients of one candidate, slots C10, C12, C21, C23,
 * C30, C32, C34, C41, C43, C45, C50, C52, C54, C56 (aberration.py:63,
 * engine.py:1244-1262): magnitudes in the length unit of C10 (Angstrom, as
 * qssb_aberrations_t), angles phi_nm in radians (ignored for m = 0 slots).
 * chi = (2 pi / lambda) sum alpha^(n+1) C_nm / (n+1) cos(m (phi - phi_nm))
 * (chi_full and pack_aberration_coefs, common.py:410-471, 646-674). */
#define QSSB_FULL_TERMS 14
typedef struct qssb_full_aberrations {
    float magnitude[QSSB_FULL_TERMS];
    float angle_rad[QSSB_FULL_TERMS];
} qssb_full_aberrations_t;

/* Workspace bytes needed by qssb_loss_batch_full for n_cand candidates. */
int qssb_loss_full_workspace_bytes(const qssb_calibration_t* cal, int32_t n_cand,
                                   int32_t flags, size_t* bytes);

/* qssb_loss_batch with the 14-term chi: replaces reconstruct_full /
 * reconstruct_full_with_loss (engine.py:1244-1458; the reference raises
 * NotImplementedError at 128, engine.py:1276-1280, 1373-1377 - this entry
 * serves 64, 128 and 256). Odd-m terms break C(-q) = -conj C(q), so every
 * scan frequency is evaluated. candidates: DEVICE array of n_cand
 * qssb_full_aberrations_t. Flags: QSSB_FLAG_CHI_FP64 (chi from FP64 q and k,
 * reduced in FP64) and QSSB_FLAG_CHUNKS; the others are ignored. */
int qssb_loss_batch_full(const float* g_half, const float* bf_geom, const float* q_row,
                         const float* q_col, const qssb_calibration_t* cal,
                         const qssb_full_aberrations_t* candidates, int32_t n_cand,
                         int32_t flags, void* workspace, size_t workspace_bytes,
                         float* losses, float* mean_phase, void* stream);

/* ------------------------------------------------------------------------
 * Time series of object waves (ssb/temporal.py:77-257): drift correction by
 * a Fourier phase ramp and the (phase-referenced) weighted complex mean.
 *
 * qssb_fourier_shift: out[t] = ifft2(fft2(in[t]) exp(-2 pi i (f_r s_r + f_c s_c))),
 * f = fftfreq(n, 1), shifts [t] = (s_r, s_c) in pixels (fourier_shift_2d,
 * temporal.py:77-107). in, out: device complex64 [n_frames][rows][cols]
 * (may alias); shifts: device float32 [n_frames][2]; rows, cols powers of two
 * in 64..1024. */
int qssb_fourier_shift(const float* in, float* out, int32_t n_frames, int32_t rows,
                       int32_t cols, const float* shifts, void* stream);

/* Workspace bytes of qssb_join_object_waves with phase_reference = 1. */
int qssb_join_workspace_bytes(int32_t n_frames, size_t* bytes);

/* joined = sum_t w_t r_t frames[t] (join_object_waves, temporal.py:192-257):
 * weights device float32 [n_frames], already normalised to sum 1
 * (temporal.py:127-140); phase_reference 1 ("first"): r_t =
 * exp(-i angle(sum_p frames[t] conj frames[0])) for t > 0, the overlap summed
 * in FP64 in a fixed order (temporal.py:154-180); 0 ("none"): r_t = 1.
 * write_back != 0 stores r_t frames[t] over frames (the aligned stack).
 * frames: device complex64 [n_frames][n_pix]; joined: complex64 [n_pix]. */
int qssb_join_object_waves(float* frames, const float* weights, int32_t n_frames, int64_t n_pix,
                           int32_t phase_reference, void* workspace, size_t workspace_bytes,
                           float* joined, int32_t write_back, void* stream);

/* ------------------------------------------------------------------------
 * HDF5 bitshuffle + LZ4 chunks (filter 32008, element size 2, 8192-byte
 * blocks) <-> u16 detector frames: the reference's acquisition decode
 * (io/load.py:3271-3320, io/backends/cuda/decoder.py:258-403) and writer
 * (io/save.py, decoder.py:496-1003). Chunk: big-endian u64 uncompressed bytes,
 * big-endian u32 block bytes, then per block a big-endian u32 size and an LZ4
 * block of the bit-shuffled elements; elements beyond the last multiple of 8
 * follow raw. */
#define QSSB_BSLZ4_OK 0
#define QSSB_BSLZ4_BAD_HEADER 1   /* header size or block size wrong, chunk too short */
#define QSSB_BSLZ4_BAD_CHAIN 2    /* a block runs past the chunk's end */
#define QSSB_BSLZ4_BAD_LZ4 3      /* malformed LZ4 sequence or wrong decoded size */

/* Decode n_chunks chunks: chunk c occupies compressed[chunk_offsets[c],
 * chunk_offsets[c+1]) (the last ends at compressed_bytes) and decodes to
 * chunk_bytes bytes at out + c * chunk_bytes / 2. compressed, chunk_offsets
 * (int64), out: device. status: device int32 [n_chunks] (QSSB_BSLZ4_*) or
 * NULL; a chunk that fails is zero-filled. Every offset and length is checked
 * against the chunk's end. */
int qssb_decode_bslz4_u16(const uint8_t* compressed, int64_t compressed_bytes,
                          const int64_t* chunk_offsets, int32_t n_chunks, int64_t chunk_bytes,
                          uint16_t* out, int32_t* status, void* stream);

/* Scratch bytes of qssb_encode_bslz4_u16. */
int qssb_encode_bslz4_scratch_bytes(int32_t n_chunks, int64_t chunk_bytes, size_t* bytes);

/* Compress n_chunks frames (device u16, chunk_bytes each) into scratch and
 * write each chunk's packed size (device int64 [n_chunks]). */
int qssb_encode_bslz4_u16(const uint16_t* frames, int32_t n_chunks, int64_t chunk_bytes,
                          uint8_t* scratch, int64_t* chunk_sizes, void* stream);

/* Lay the chunks out at chunk_offsets (device int64, e.g. the exclusive sum
 * of chunk_sizes) in packed (device u8, room for the total). */
int qssb_pack_bslz4(const uint8_t* scratch, const uint16_t* frames, int32_t n_chunks,
                    int64_t chunk_bytes, const int64_t* chunk_offsets, uint8_t* packed,
                    void* stream);

/* ------------------------------------------------------------------------
 * Learned aberration proposer (no counterpart in the reference, which has no
 * learned component). Features: trotter amplitudes |G_b(Q)| at n_q scan
 * frequencies, resampled onto a k grid through a caller-built CSR table
 * (cells x BF pixels: csr_off [cells+1], csr_idx, csr_w with row sums 1) and
 * divided by their mean over covered cells. scratch: float [n_q * n_bf]
 * (times n_samples for qssb_synth_features). Outputs [n_samples][n_q][cells]
 * as float32 and/or BF16 (either pointer may be NULL, not both).
 */
/* Inference features from a resident Hermitian G [n_bf][scan_n][scan_n/2+1];
 * q_idx: device int32 [n_q][2] fftfreq indices (row, col), any sign. */
int qssb_trotter_features(const float* g_half, int32_t n_bf, int32_t scan_n, const int32_t* q_idx,
                          int32_t n_q, const int32_t* csr_off, const int32_t* csr_idx,
                          const float* csr_w, int32_t cells, float* scratch, float* out_f32,
                          void* out_bf16, void* stream);

/* Training features from the SSB forward model of a weak object:
 * v = |Gamma(Q, k_b) phi + Gamma+(Q, k_b) phi_a + n|,
 * Gamma = P(Q-k) conj P(k) - conj P(Q+k) P(k) (kernels/common.py:115-236),
 * Gamma+ = P(Q-k) conj P(k) + conj P(Q+k) P(k) (amplitude contrast), phi:
 * complex64 [n_samples][n_q][2] = (phi, phi_a) per map, n complex
 * Gaussian of standard deviation sigma[s][q] |phi| (float [n_samples][n_q])
 * from a counter-based hash of (seed, index). bf_geom: the [8][n_bf] geometry of the training detector
 * lattice; q_vec: device float [n_q][2] in 1/A; cal supplies wavelength,
 * aperture and detector sampling (n_bf and dc unused). */
int qssb_synth_features(const float* bf_geom, int32_t n_bf, const float* q_vec, int32_t n_q,
                        const qssb_aberrations_t* aberrations, const float* phi,
                        const float* sigma, int32_t n_samples, const qssb_calibration_t* cal,
                        uint64_t seed, const int32_t* csr_off, const int32_t* csr_idx,
                        const float* csr_w, int32_t cells, float* scratch, float* out_f32,
                        void* out_bf16, void* stream);

/* C[M][N] (+)= op(A)[M][K] op(B)[K][N] on the tensor cores: A, B BF16
 * (op = transpose when trans_*), FP32 accumulation; M, N, K multiples of 16,
 * leading dimensions multiples of 8, A and B 32-byte aligned. Epilogue: + bias
 * [N] (or NULL); C (FP32, NULL allowed) stores or, with accumulate, adds;
 * act_bf16 (NULL allowed) receives BF16 GELU(result) (tanh form). */
int qssb_gemm_bf16(const void* A, int32_t lda, int32_t trans_a, const void* B, int32_t ldb,
                   int32_t trans_b, int32_t M, int32_t N, int32_t K, const float* bias,
                   int32_t accumulate, float* C, int32_t ldc, void* act_bf16, int32_t ld_act,
                   void* stream);

/* The same GEMM on the 5th-generation tensor cores (tcgen05.mma kind::f16,
 * FP32 accumulator in tensor memory), split over K: 128 x 128 output tiles,
 * splits K ranges each; with splits > 1 the partial tiles go to the workspace
 * and are summed in split order (deterministic), then the epilogue of
 * qssb_gemm_bf16; with splits == 1 the MMA kernel applies that epilogue and
 * writes C itself (C then 16-byte aligned, ldc a multiple of 4). M and N
 * multiples of 128, K a multiple of 64 x splits, leading dimensions multiples
 * of 8, A and B 16-byte aligned, workspace 256-byte aligned and at least
 * qssb_gemm_tc_workspace_bytes (4 splits M N + 256 bytes with split K, 256
 * without); its last 256 bytes hold an int set to 1 when a bounded wait
 * inside the kernel gave up (the result is then invalid). */
int qssb_gemm_tc_workspace_bytes(int32_t M, int32_t N, int32_t K, int32_t splits, size_t* bytes);
int qssb_gemm_bf16_tc(const void* A, int32_t lda, int32_t trans_a, const void* B, int32_t ldb,
                      int32_t trans_b, int32_t M, int32_t N, int32_t K, int32_t splits,
                      const float* bias, int32_t accumulate, float* C, int32_t ldc, void* act_bf16,
                      int32_t ld_act, void* workspace, size_t workspace_bytes, void* stream);
/* dz = dy * GELU'(pre) (FP32 and BF16 copies), n elements. */
int qssb_gelu_backward(const float* dy, const float* pre, int64_t n, void* dz_bf16, float* dz,
                       void* stream);
/* db[c] = sum over rows of dz[r][c] (FP64 accumulation: eight interleaved
 * row slices folded in a fixed order). */
int qssb_bias_grad(const float* dz, int32_t rows, int32_t cols, float* db, void* stream);
/* Mean squared error over the first n_out of ld columns and its gradient dy
 * (zero in columns n_out..ld-1); loss (device float) may be NULL. */
int qssb_mse(const float* y, const float* target, int32_t rows, int32_t n_out, int32_t ld,
             float* dy, float* loss, void* stream);
/* Multi-head (winner-takes-all) MSE: row r of y (ld columns) holds `heads`
 * groups of n_out outputs against target[r][0..n_out). Per row the winner is
 * the head with the least squared error over its first n_select outputs
 * (ties: lowest index; written to winner[r] when winner is not NULL); loss =
 * mean over rows of sum_c w_c (y_win,c - t_c)^2 / n_out, w = out_weight
 * (n_out floats, NULL = all 1); dy_h,c = 2 s_h w_c (y_h,c - t_c) / (rows
 * n_out) with s = 1 - eps for the winner and eps / (heads - 1) for the others
 * (1 with one head), zero in the padding columns. heads * n_out <= ld,
 * 1 <= n_select <= n_out, 0 <= eps < 1. */
int qssb_mse_heads(const float* y, const float* target, int32_t rows, int32_t n_out,
                   int32_t heads, int32_t ld, const float* out_weight, int32_t n_select,
                   float eps, float* dy, float* loss, int32_t* winner, void* stream);
/* Adam (bias-corrected, decoupled weight decay) on FP32 master weights; the
 * BF16 copy w_bf16 (may be NULL) is refreshed. step counts from 1. */
int qssb_adam(float* w, float* m, float* v, const float* grad, int64_t n, float lr, float beta1,
              float beta2, float eps, float weight_decay, int32_t step, void* w_bf16,
              void* stream);
/* The training schedule on the device, for graph-replayed steps: *step += 1,
 * then hyper[0..2] = {lr0 (1 + cos(pi (step - 1 - first_step) / total_steps))
 * / 2, 1 - beta1^step, 1 - beta2^step} (device float[3], device int32 step;
 * first_step: the step count when this cosine run began). */
int qssb_adam_schedule(float* hyper, int32_t* step, int32_t first_step, int32_t total_steps,
                       float lr0, float beta1, float beta2, void* stream);
/* qssb_adam with the learning rate and bias corrections read from hyper
 * (device {lr, c1, c2}, as qssb_adam_schedule writes them). */
int qssb_adam_dev(float* w, float* m, float* v, const float* grad, int64_t n, const float* hyper,
                  float beta1, float beta2, float eps, float weight_decay, void* w_bf16,
                  void* stream);
/* y = BF16(x), n elements. */
int qssb_to_bf16(const float* x, int64_t n, void* y, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* QSSB_H */
