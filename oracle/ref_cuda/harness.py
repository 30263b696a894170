"""Launch the reference's own 128x128 SSB object kernels (checker and baseline).

Test infrastructure: imported only by tests/ and by bench.py's baseline legs.
The kernels come from ``oracle/_ref/ssb_fft128.cubin`` (built by
``build_ref.py`` from the reference's sources); this file holds only the
launch sequence of ``SSBEngine._run_correction_pipeline`` (engine.py:934-971)
and ``CustomFFTBase.ifft2_inplace_fused_pk`` (common.py:768-816), and the
restated pk element-wise kernel (engine.py:217-231).
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from .build_ref import CUBIN, FULL_PROBE_NAME, KERNEL_NAMES, TWIDDLE_NAME, available

N = 128


def _check(res):
    err = res[0] if isinstance(res, tuple) else res
    if int(err) != 0:
        raise RuntimeError(f"CUDA driver call failed: {err}")
    return res[1:] if isinstance(res, tuple) and len(res) > 1 else None


class ReferenceObject128:
    """The reference's per-BF fused IFFT object path for 128x128 scans."""

    def __init__(self, device: torch.device | str = "cuda:0"):
        if not available():
            raise FileNotFoundError(f"{CUBIN} is missing: run python -m oracle.ref_cuda.build_ref")
        from cuda.bindings import driver as cu

        self.cu = cu
        self.device = torch.device(device)
        torch.cuda.set_device(self.device)
        torch.zeros(1, device=self.device)  # make torch's primary context current
        (self.module,) = _check(cu.cuModuleLoad(str(CUBIN).encode()))
        (self.rows,) = _check(cu.cuModuleGetFunction(self.module, KERNEL_NAMES[0].encode()))
        (self.cols,) = _check(cu.cuModuleGetFunction(self.module, KERNEL_NAMES[1].encode()))
        dptr, nbytes = _check(cu.cuModuleGetGlobal(self.module, TWIDDLE_NAME.encode()))
        # CustomFFTBase._init_twiddles (common.py:725-730): exp(+2 pi i n / N), complex64
        w = np.exp(2j * math.pi * np.arange(N) / N).astype(np.complex64)
        assert int(nbytes) == w.nbytes
        tw = torch.from_numpy(w.view(np.float32)).to(self.device)
        torch.cuda.synchronize(self.device)
        _check(cu.cuMemcpyDtoD(dptr, cu.CUdeviceptr(tw.data_ptr()), w.nbytes))
        self._buf: torch.Tensor | None = None

    @staticmethod
    def pk(geom: torch.Tensor, C10: float, C12: float, phi12: float, factor: float) -> torch.Tensor:
        """pk = A(k) exp(-i chi(k)) per BF pixel: the reference's _pk_kernel
        (engine.py:217-231) restated with torch float32 operations."""
        alpha2, c2, s2, ap = geom[2], geom[3], geom[4], geom[5]
        cos_term = c2 * np.float32(math.cos(2 * phi12)) + s2 * np.float32(math.sin(2 * phi12))
        chi = np.float32(factor) * alpha2 * (np.float32(C12) * cos_term + np.float32(C10))
        return torch.complex(ap * torch.cos(chi), -ap * torch.sin(chi))

    def _launch(self, fn, grid, block, args, stream) -> None:
        values = tuple(a[0] for a in args)
        types = tuple(a[1] for a in args)
        _check(self.cu.cuLaunchKernel(fn, *grid, *block, 0, stream, (values, types), 0))

    def corrected_images(self, g_half: torch.Tensor, geom: torch.Tensor, q_row: torch.Tensor,
                         q_col: torch.Tensor, wavelength: float, semiangle_rad: float,
                         ang_y_rad: float, ang_x_rad: float, C10: float, C12: float,
                         phi12: float, dc: complex) -> torch.Tensor:
        """[B, 128, 128] corrected BF images O_b (rows kernel + columns kernel)."""
        n_bf = int(g_half.shape[0])
        assert g_half.shape == (n_bf, N, N // 2 + 1) and g_half.dtype == torch.complex64
        assert geom.shape[0] >= 6 and geom.shape[1] == n_bf and n_bf * N * N < 2 ** 31
        g_half = g_half.contiguous()
        factor = math.pi / wavelength
        pk = self.pk(geom, C10, C12, phi12, factor).contiguous()
        kx = geom[0].contiguous()
        ky = geom[1].contiguous()
        if self._buf is None or self._buf.shape[0] != n_bf:
            self._buf = torch.empty((n_bf, N, N), dtype=torch.complex64, device=self.device)
        out = self._buf
        stream = self.cu.CUstream(torch.cuda.current_stream(self.device).cuda_stream)
        P, F, I = ctypes.c_void_p, ctypes.c_float, ctypes.c_int
        f32 = lambda x: float(np.float32(x))  # noqa: E731  (np.float32 kernel arguments)
        args = [(kx.data_ptr(), P), (ky.data_ptr(), P), (q_row.data_ptr(), P), (q_col.data_ptr(), P),
                (f32(wavelength), F), (f32(semiangle_rad), F), (f32(ang_y_rad), F),
                (f32(ang_x_rad), F), (f32(C10), F), (f32(C12), F),
                (f32(math.cos(2.0 * phi12)), F), (f32(math.sin(2.0 * phi12)), F), (f32(factor), F),
                (pk.data_ptr(), P), (g_half.data_ptr(), P), (out.data_ptr(), P),
                (f32(dc.real), F), (f32(dc.imag), F), (n_bf, I), (N // 2 + 1, I)]
        # grids of ifft2_inplace_fused_pk: (1, 16, B) x (32, 8, 1), both kernels
        self._launch(self.rows, (1, 16, n_bf), (32, 8, 1), args, stream)
        self._launch(self.cols, (1, 16, n_bf), (32, 8, 1),
                     [(out.data_ptr(), P), (n_bf, I), (f32(1.0 / (N * N)), F)], stream)
        return out

    def full_chi_probe(self, qx, qy, kx, ky, *, wavelength: float, semiangle_rad: float,
                       ang_y_rad: float, ang_x_rad: float, magnitudes, angles, pk, g):
        """The reference's chi_full(q - k) and gamma_mul_pk_onthefly_full
        (common.py:410-532) at n points (float32 CUDA [n] inputs; pk, g
        complex64 [n]). Coefficients packed as pack_aberration_coefs does
        (common.py:646-674): mag / (n+1), cos(m angle), sin(m angle) in float32."""
        nm = ((1, 0), (1, 2), (2, 1), (2, 3), (3, 0), (3, 2), (3, 4),
              (4, 1), (4, 3), (4, 5), (5, 0), (5, 2), (5, 4), (5, 6))
        mags = np.asarray(magnitudes, np.float32)
        angs = np.asarray(angles, np.float32)
        n1 = np.array([n + 1 for n, _ in nm], np.float32)
        m = np.array([m for _, m in nm], np.float32)
        packed = [torch.as_tensor(a, device=self.device) for a in
                  (mags * (np.float32(1.0) / n1), np.cos(m * angs, dtype=np.float32),
                   np.sin(m * angs, dtype=np.float32))]
        if not hasattr(self, "probe"):
            (self.probe,) = _check(self.cu.cuModuleGetFunction(self.module, FULL_PROBE_NAME.encode()))
        n = int(qx.numel())
        chi = torch.empty(n, dtype=torch.float32, device=self.device)
        out = torch.empty(n, dtype=torch.complex64, device=self.device)
        pk = pk.contiguous()
        g = g.contiguous()
        P, F, I = ctypes.c_void_p, ctypes.c_float, ctypes.c_int
        f32 = lambda x: float(np.float32(x))  # noqa: E731
        args = [(qx.data_ptr(), P), (qy.data_ptr(), P), (kx.data_ptr(), P), (ky.data_ptr(), P),
                (n, I), (f32(wavelength), F), (f32(semiangle_rad), F), (f32(ang_y_rad), F),
                (f32(ang_x_rad), F), *[(t.data_ptr(), P) for t in packed],
                (pk.data_ptr(), P), (g.data_ptr(), P), (chi.data_ptr(), P), (out.data_ptr(), P)]
        stream = self.cu.CUstream(torch.cuda.current_stream(self.device).cuda_stream)
        self._launch(self.probe, ((n + 255) // 256, 1, 1), (256, 1, 1), args, stream)
        torch.cuda.synchronize(self.device)
        return chi, out

    def object(self, *args, **kw) -> torch.Tensor:
        """reconstruct_object for B > 1024 (engine.py:1148-1151): mean over BF pixels."""
        return self.corrected_images(*args, **kw).mean(dim=0)


def reference_cold_object(counts: torch.Tensor, ref: ReferenceObject128, *, wavelength: float,
                          semiangle_mrad: float, det_sampling_mrad: float,
                          scan_sampling_A: float, C10: float, C12: float, phi12: float,
                          threshold: float = 0.0, bf_radius=None):
    """One cold reconstruction the way CudaSSBBackend + SSBEngine do it for a
    128^4 u16 device tensor: u64 frame sums and float32 mean
    (backend.py:432-441, torch.sum standing in for CuPy's reduction), the BF
    selection and the rotation cache (host restatements of backend.py:448-518
    and engine.py:784-830, which the reference evaluates with CuPy and host
    syncs), the gather / transpose / complex64 cast / cuFFT fft2 / half-plane
    slice / dc of _extract_gqk (backend.py:520-589) as torch library calls,
    then the reference's own object kernels. Returns (object, phase, n_bf)."""
    from quantem.gpu_b200.calibration import bf_geometry, scan_frequencies, select_bf

    r0, r1, k0, k1 = (int(s) for s in counts.shape)
    assert r0 == r1 == N
    frames = counts.reshape(-1, k0, k1)
    sums = frames.sum(dim=0, dtype=torch.int64)
    mean_dp = sums.to(torch.float32) / float(frames.shape[0])
    sel = select_bf(mean_dp.cpu().numpy(), threshold, bf_radius)
    rows = torch.as_tensor(sel.rows, device=counts.device, dtype=torch.int64)
    cols = torch.as_tensor(sel.cols, device=counts.device, dtype=torch.int64)
    n_bf = int(rows.numel())
    # torch's CUDA gather has no uint16 kernel: gather the same bits as int16
    vbf = frames.view(torch.int16)[:, rows, cols]                 # [N_R, B]
    vbf_int = vbf.T.reshape(n_bf, r0, r1).contiguous()
    vbf_c = (vbf_int.to(torch.int32) & 0xFFFF).to(torch.complex64)
    g_half = torch.fft.fft2(vbf_c)[:, :, : r1 // 2 + 1].contiguous()
    dc = complex(g_half[:, 0, 0].mean().item())
    recip = det_sampling_mrad * 1e-3 / wavelength
    sampling = (1.0 / (recip * k0), 1.0 / (recip * k1))
    geo = bf_geometry(sel.rows, sel.cols, sel.center, (k0, k1), sampling, wavelength,
                      semiangle_mrad, (det_sampling_mrad, det_sampling_mrad), 0.0)
    geom = torch.as_tensor(geo.stacked(), device=counts.device)
    q_row, q_col = (torch.as_tensor(q, device=counts.device)
                    for q in scan_frequencies((r0, r1), (scan_sampling_A, scan_sampling_A)))
    obj = ref.object(g_half, geom, q_row, q_col, wavelength, semiangle_mrad * 1e-3,
                     det_sampling_mrad * 1e-3, det_sampling_mrad * 1e-3, C10, C12, phi12, dc)
    return obj, torch.angle(obj), n_bf


class ReferenceLossBatch128:
    """The reference's batched phase-variance loss for 128x128 scans, replayed
    with its own kernels: ``SSBEngine.variance_loss_batch`` (engine.py:2120-2295)
    -> the pk element-wise kernel (restated, engine.py:217-231) ->
    ``ifft2_inplace_batch_fused_pk_variance`` streaming over BF chunks
    (common.py:1006-1092: K12 ``ifft128_rows_fused_pk_batch_t32_mr8_transpose_packed_b4``
    on grid (1, 8, quads * chunk) x (32, 16, 1) with 64 KB of dynamic shared
    memory, then K13 ``ifft128_rows_var_g32_t32_mr1_batch`` on grid
    (1, 128, ceil(chunk / 32) * batch) x (32, 1, 1) adding into the sums) ->
    K14 ``loss_from_sums_batch`` (engine.py:96-137) on (batch,) x (256,).

    The BF chunk is the engine's for 128x128 scans: every BF pixel at once when
    the staging planes (batch x B x 128 x 128 complex64) fit 2 GiB, else
    min(1024, B) (engine.py:2183-2200, with the memory-derived cap far above
    1024 on a B200). Batches below 4 are padded with copies of the last
    candidate (the reference loops them through its scalar path instead).
    """

    def __init__(self, device: torch.device | str = "cuda:0"):
        from .build_ref import LOSS_KERNEL_NAMES, SUMS_CUBIN, SUMS_KERNEL, sums_available

        if not (available() and sums_available()):
            raise FileNotFoundError("reference loss cubins missing: run python -m oracle.ref_cuda.build_ref")
        self.obj = ReferenceObject128(device)  # loads the module and its twiddles
        cu = self.obj.cu
        self.cu = cu
        self.device = self.obj.device
        (self.k12,) = _check(cu.cuModuleGetFunction(self.obj.module, LOSS_KERNEL_NAMES[0].encode()))
        (self.k13,) = _check(cu.cuModuleGetFunction(self.obj.module, LOSS_KERNEL_NAMES[1].encode()))
        _check(cu.cuFuncSetAttribute(
            self.k12, cu.CUfunction_attribute.CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, 65536))
        (self.sums_module,) = _check(cu.cuModuleLoad(str(SUMS_CUBIN).encode()))
        (self.k14,) = _check(cu.cuModuleGetFunction(self.sums_module, SUMS_KERNEL.encode()))
        self._bufs: dict = {}

    def _buffers(self, batch: int, n_bf: int, chunk: int) -> dict:
        key = (batch, n_bf, chunk)
        if key not in self._bufs:
            self._bufs.clear()
            tail = n_bf % chunk
            dev = self.device
            self._bufs[key] = {
                "staging": torch.empty((batch, chunk, N, N), dtype=torch.complex64, device=dev),
                "tail": (torch.empty((batch, tail, N, N), dtype=torch.complex64, device=dev)
                         if tail else None),
                "sum": torch.empty((batch, N, N), dtype=torch.float32, device=dev),
                "sumsq": torch.empty((batch, N, N), dtype=torch.float32, device=dev),
                "loss": torch.empty(batch, dtype=torch.float32, device=dev),
            }
        return self._bufs[key]

    def losses(self, g_half: torch.Tensor, geom: torch.Tensor, q_row: torch.Tensor,
               q_col: torch.Tensor, wavelength: float, semiangle_rad: float, ang_y_rad: float,
               ang_x_rad: float, C10, C12, phi12, dc: complex) -> torch.Tensor:
        """float32 CUDA [batch] losses of the candidates (C10, C12, phi12 arrays)."""
        n_bf = int(g_half.shape[0])
        assert g_half.shape == (n_bf, N, N // 2 + 1) and g_half.dtype == torch.complex64
        assert geom.shape[0] >= 6 and geom.shape[1] == n_bf
        c10 = np.atleast_1d(np.asarray(C10, np.float32))
        n = c10.size
        c12 = np.broadcast_to(np.asarray(C12, np.float32), (n,))
        phi = np.broadcast_to(np.asarray(phi12, np.float32), (n,))
        batch = max(n, 4)
        pad = lambda a: np.concatenate([a, np.repeat(a[-1:], batch - n)])  # noqa: E731
        c10, c12, phi = pad(c10), pad(np.array(c12)), pad(np.array(phi))
        dev = self.device
        cos2 = np.cos(2.0 * phi).astype(np.float32)
        sin2 = np.sin(2.0 * phi).astype(np.float32)
        params = [torch.as_tensor(a, device=dev) for a in (c10, c12, cos2, sin2)]
        factor = math.pi / wavelength
        # pk [batch, B] = A(k) exp(-i chi(k)) per candidate (engine.py:217-231)
        alpha2, c2k, s2k, ak = geom[2], geom[3], geom[4], geom[5]
        chi = np.float32(factor) * alpha2[None, :] * (
            params[1][:, None] * (c2k[None, :] * params[2][:, None] + s2k[None, :] * params[3][:, None])
            + params[0][:, None])
        pk = torch.complex(ak[None, :] * torch.cos(chi), -ak[None, :] * torch.sin(chi)).contiguous()
        staging_bytes = batch * n_bf * N * N * 8
        chunk = n_bf if staging_bytes <= 2 * 1024 ** 3 else min(1024, n_bf)
        bufs = self._buffers(batch, n_bf, chunk)
        bufs["sum"].zero_()
        bufs["sumsq"].zero_()
        g_half = g_half.contiguous()
        kx, ky = geom[0].contiguous(), geom[1].contiguous()
        stream = self.cu.CUstream(torch.cuda.current_stream(dev).cuda_stream)
        P, F, I = ctypes.c_void_p, ctypes.c_float, ctypes.c_int
        f32 = lambda x: float(np.float32(x))  # noqa: E731
        quads = (batch + 3) // 4
        for start in range(0, n_bf, chunk):
            cnt = min(chunk, n_bf - start)
            staging = bufs["staging"] if cnt == chunk else bufs["tail"]
            pk_group = pk[:, start:start + cnt].contiguous()
            args = [(kx.data_ptr() + 4 * start, P), (ky.data_ptr() + 4 * start, P),
                    (q_row.data_ptr(), P), (q_col.data_ptr(), P),
                    (f32(wavelength), F), (f32(semiangle_rad), F), (f32(ang_y_rad), F),
                    (f32(ang_x_rad), F), *[(t.data_ptr(), P) for t in params], (f32(factor), F),
                    (pk_group.data_ptr(), P), (g_half.data_ptr() + 8 * start * N * (N // 2 + 1), P),
                    (staging.data_ptr(), P), (f32(dc.real), F), (f32(dc.imag), F),
                    (cnt, I), (batch, I), (N // 2 + 1, I)]
            _check(self.cu.cuLaunchKernel(self.k12, 1, 8, quads * cnt, 32, 16, 1, 65536, stream,
                                          (tuple(a[0] for a in args), tuple(a[1] for a in args)), 0))
            groups = (cnt + 31) // 32
            args = [(staging.data_ptr(), P), (bufs["sum"].data_ptr(), P),
                    (bufs["sumsq"].data_ptr(), P), (cnt, I), (batch, I), (f32(1.0 / (N * N)), F),
                    (0, I)]
            _check(self.cu.cuLaunchKernel(self.k13, 1, 128, groups * batch, 32, 1, 1, 0, stream,
                                          (tuple(a[0] for a in args), tuple(a[1] for a in args)), 0))
        args = [(bufs["sum"].data_ptr(), P), (bufs["sumsq"].data_ptr(), P),
                (bufs["loss"].data_ptr(), P), (n_bf, I), (N, I), (N, I), (batch, I)]
        _check(self.cu.cuLaunchKernel(self.k14, batch, 1, 1, 256, 1, 1, 0, stream,
                                      (tuple(a[0] for a in args), tuple(a[1] for a in args)), 0))
        return bufs["loss"][:n]
