"""Learned aberration proposer: trotter-amplitude features, an MLP trained on
the SSB forward model with the library's own CUDA kernels, and the short
batched SSB refinement its proposal seeds.

No counterpart in the reference, whose fits search the whole prior box
(Optuna TPE + Nelder-Mead, backend.py:958-1374). The pieces:

* Features (``qssb_trotter_features`` / ``qssb_synth_features``): |G_b(Q)|
  at 16 fixed scan frequencies Q = (m, n) / 32 A^-1 on the reciprocal
  lattice of the synthetic 4 A square crystal (multiples of 1/4 A^-1 along
  eight directions, where its signal lies; on the fftfreq grid of every scan
  whose extent N d is a multiple of 32 A), resampled onto a 32x32 grid over
  the aperture disk with a tent of the training detector's pitch and
  normalised per Q: 16384 inputs, independent of dose and object contrast.
* Training data: the SSB forward model of a weak-phase object,
  G_b(Q) = Gamma(Q, k_b) Phi(Q) + noise, on a 64x64-scan x 64x64-detector
  lattice (300 kV, 20 mrad, 20/12 mrad per pixel), aberrations uniform in the
  sweep ranges (C1 +-50 nm, |A1| <= 10 nm, C3 <= 1 um), random Phi and noise;
  each sample leaves a random 0 .. 8 of its 16 maps noise-dominated.
* Network: 16384 -> 512 -> 512 -> 512 -> 4 heads x 4, GELU, BF16 weights
  and activations on the tensor cores with FP32 accumulation, FP32 master
  weights and Adam (``qssb_gemm_bf16_tc`` / ``qssb_gemm_bf16``,
  ``qssb_gelu_backward``, ``qssb_bias_grad``, ``qssb_mse_heads``,
  ``qssb_adam``). Each head outputs (C1, |A1| cos 2phi, |A1| sin 2phi, C3),
  C1 and A1 on one scale (an error of 1 A costs the same in either). The
  heads train winner-takes-all on (C1, A1): the amplitudes fix
  c(phi) = C1 + |A1| cos 2(phi - phi_A1) per direction only up to
  |sin(pi lambda |Q|^2 c)|, whose aliases differ by 16/lambda (812 A at
  300 kV) on this lattice, so one input can have several answers and each
  head learns one.
* Sign: trotter amplitudes are unchanged when every aberration flips sign
  (Gamma -> conj Gamma), so targets are canonical (C1 >= 0) and a proposal
  is eight hypotheses (four heads, each sign), scored together as the
  refinement's first 8-candidate batch.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib, ops
from ._lib import Calibration, check
from .calibration import bf_geometry
from .physics import electron_wavelength_angstrom
from .synthetic import SWEEP_RANGES

Q_UNITS = np.array([(8, 0), (16, 0), (24, 0), (0, 8), (0, 16), (0, 24), (8, 8), (16, 16),
                    (8, -8), (16, -16), (16, 8), (8, 16), (16, -8), (8, -16), (24, 8), (8, 24)],
                   dtype=np.int32)
Q_PERIOD_A = 32.0          # Q = units / 32 A^-1
GRID = 32
K_MAX_FACTOR = 1.05        # grid half-width in units of the aperture radius alpha/lambda
CELL_RADIUS_FACTOR = 0.9   # cells beyond 0.9 alpha/lambda stay empty: the BF sets of the
                           # training lattice and of a selected dataset differ at the rim
N_IN = len(Q_UNITS) * GRID * GRID
HIDDEN = 512
N_OUT = 4
HEADS = 4
N_OUT_PAD = 16             # HEADS x N_OUT
OUT_SCALE = np.array([200.0, 200.0, 200.0, 1.0e4], dtype=np.float32)
OUT_WEIGHT = np.array([1.0, 1.0, 1.0, 0.1], dtype=np.float32)  # C3 is barely visible
WTA_EPS = 0.05             # share of the gradient the losing heads keep
ADAM_BETAS = (0.9, 0.999)

# the training lattice (64x64 detector)
TRAIN_VOLTAGE_KV = 300.0
TRAIN_SEMIANGLE_MRAD = 20.0
TRAIN_DET_SAMPLING_MRAD = 20.0 / 12.0
TRAIN_DET = 64


def _ptr(t):
    return ctypes.c_void_p(0 if t is None else t.data_ptr())


def _stream(dev):
    return ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def _call(name, dev, *args):
    ops._call(name, dev, *args)


# --------------------------------------------------------------- features
def tent_half_width() -> float:
    """Tent half-width (1/A): the training detector's pixel pitch."""
    lam = electron_wavelength_angstrom(TRAIN_VOLTAGE_KV * 1e3)
    return TRAIN_DET_SAMPLING_MRAD * 1e-3 / lam


def k_max(semiangle_mrad: float, wavelength_A: float) -> float:
    return K_MAX_FACTOR * semiangle_mrad * 1e-3 / wavelength_A


def resample_table(kx: np.ndarray, ky: np.ndarray, kmax: float, h: float,
                   grid: int = GRID, cell_radius: float | None = None
                   ) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """CSR (cell -> BF pixels) tent weights, rows normalised to sum 1; cells whose
    centre lies beyond ``cell_radius`` (1/A) are left empty."""
    kx = np.asarray(kx, np.float64)
    ky = np.asarray(ky, np.float64)
    step = 2.0 * kmax / grid
    centres = -kmax + (np.arange(grid) + 0.5) * step
    rmax2 = np.inf if cell_radius is None else cell_radius * cell_radius
    wx = 1.0 - np.abs(kx[None, :] - centres[:, None]) / h          # [grid, B]
    wy = 1.0 - np.abs(ky[None, :] - centres[:, None]) / h
    wx = np.where(wx > 0, wx, 0.0)
    wy = np.where(wy > 0, wy, 0.0)
    # each tent spans a few cells per axis: (pixel, cell) pairs from the cells
    # near each pixel only, then ordered cell-major with pixels ascending
    reach = int(np.ceil(h / step)) + 1
    n_bf = kx.size
    base_i = np.floor((kx + kmax) / step).astype(np.int64)
    base_j = np.floor((ky + kmax) / step).astype(np.int64)
    d = np.arange(-reach, reach + 1)
    ci = base_i[:, None] + d[None, :]                                # [B, 2R+1]
    cj = base_j[:, None] + d[None, :]
    ok_i = (ci >= 0) & (ci < grid)
    ok_j = (cj >= 0) & (cj < grid)
    ci_c = np.clip(ci, 0, grid - 1)
    cj_c = np.clip(cj, 0, grid - 1)
    pix = np.arange(n_bf)[:, None]
    wxi = np.where(ok_i, wx[ci_c, pix], 0.0)
    wyj = np.where(ok_j, wy[cj_c, pix], 0.0)
    w = wxi[:, :, None] * wyj[:, None, :]                           # [B, 2R+1, 2R+1]
    cells = ci_c[:, :, None] * grid + cj_c[:, None, :]
    inside = (centres[:, None] ** 2 + centres[None, :] ** 2 <= rmax2).ravel()
    keep = (w > 0) & inside[cells]
    cell = cells[keep]
    b = np.broadcast_to(np.arange(n_bf)[:, None, None], w.shape)[keep]
    vals = w[keep]
    order = np.lexsort((b, cell))
    cell, b, vals = cell[order], b[order], vals[order]
    counts = np.bincount(cell, minlength=grid * grid)
    sums = np.bincount(cell, weights=vals, minlength=grid * grid)
    off = np.concatenate([[0], np.cumsum(counts)])
    wts = vals / sums[cell]
    return off.astype(np.int32), b.astype(np.int32), wts.astype(np.float32)


@dataclass
class Lattice:
    """Geometry of one feature source on the device: BF k-vectors and the CSR table."""

    n_bf: int
    off: torch.Tensor
    idx: torch.Tensor
    w: torch.Tensor


_LATTICES: dict = {}  # device CSR tables by (device, geometry): datasets share detectors


def _lattice(kx: np.ndarray, ky: np.ndarray, kmax: float, device) -> Lattice:
    key = (str(device), float(kmax), np.asarray(kx, np.float32).tobytes(),
           np.asarray(ky, np.float32).tobytes())
    hit = _LATTICES.get(key)
    if hit is not None:
        return hit
    off, idx, w = resample_table(kx, ky, kmax, tent_half_width(),
                                 cell_radius=CELL_RADIUS_FACTOR * kmax / K_MAX_FACTOR)
    if idx.size == 0:
        idx = np.zeros(1, np.int32)
        w = np.zeros(1, np.float32)
    t = lambda a: torch.as_tensor(a, device=device)  # noqa: E731
    lat = Lattice(int(len(kx)), t(off), t(idx), t(w))
    if len(_LATTICES) >= 8:
        _LATTICES.pop(next(iter(_LATTICES)))
    _LATTICES[key] = lat
    return lat


def backend_features(be) -> torch.Tensor:
    """Features [1, N_IN] (BF16) of a prepared ``B200SSBBackend`` dataset."""
    n = be.scan_shape[0]
    extent = n * be.scan_sampling[0]
    scale = extent / Q_PERIOD_A
    if abs(scale - round(scale)) > 1e-6 or abs(be.scan_sampling[0] - be.scan_sampling[1]) > 1e-12:
        raise ValueError("the proposer needs square scans whose extent is a multiple of 32 A")
    q_idx = torch.as_tensor((Q_UNITS * int(round(scale))).astype(np.int32), device=be.device)
    lat = getattr(be, "_proposer_lattice", None)
    if lat is None:
        geo = be._geom_dev[:2].cpu().numpy()
        lat = _lattice(geo[0], geo[1], k_max(be.semiangle_cutoff, be.wavelength), be.device)
        be._proposer_lattice = lat
    nq = len(Q_UNITS)
    scratch = torch.empty(nq * lat.n_bf, dtype=torch.float32, device=be.device)
    out = torch.empty((1, N_IN), dtype=torch.bfloat16, device=be.device)
    _call("qssb_trotter_features", be.device, _ptr(be.G_qk), lat.n_bf, n, _ptr(q_idx), nq,
          _ptr(lat.off), _ptr(lat.idx), _ptr(lat.w), GRID * GRID, _ptr(scratch), None, _ptr(out),
          _stream(be.device))
    return out


class TrainingLattice:
    """The 64x64-detector lattice of the forward-model training data."""

    def __init__(self, device):
        self.device = torch.device(device)
        lam = electron_wavelength_angstrom(TRAIN_VOLTAGE_KV * 1e3)
        self.wavelength = lam
        dk = TRAIN_DET_SAMPLING_MRAD * 1e-3 / lam
        c = TRAIN_DET / 2.0
        ii, jj = np.meshgrid(np.arange(TRAIN_DET), np.arange(TRAIN_DET), indexing="ij")
        kr = (ii - c) * dk
        kc = (jj - c) * dk
        edge = (TRAIN_SEMIANGLE_MRAD * 1e-3 + 0.5 * TRAIN_DET_SAMPLING_MRAD * 1e-3) / lam
        inside = (kr * kr + kc * kc) < edge * edge
        rows, cols = np.nonzero(inside)
        sampling = (1.0 / (dk * TRAIN_DET),) * 2
        geo = bf_geometry(rows.astype(np.int32), cols.astype(np.int32), (c, c),
                          (TRAIN_DET, TRAIN_DET), sampling, lam, TRAIN_SEMIANGLE_MRAD,
                          (TRAIN_DET_SAMPLING_MRAD,) * 2, 0.0)
        self.geom = torch.as_tensor(geo.stacked(), device=self.device).contiguous()
        self.lattice = _lattice(geo.kx_bf, geo.ky_bf, k_max(TRAIN_SEMIANGLE_MRAD, lam), self.device)
        self.q_vec = torch.as_tensor((Q_UNITS / Q_PERIOD_A).astype(np.float32), device=self.device)
        self.cal = Calibration(
            n_bf=self.lattice.n_bf, scan_rows=64, scan_cols=64, reserved=0, wavelength_A=lam,
            semiangle_rad=TRAIN_SEMIANGLE_MRAD * 1e-3,
            det_sampling_row_rad=TRAIN_DET_SAMPLING_MRAD * 1e-3,
            det_sampling_col_rad=TRAIN_DET_SAMPLING_MRAD * 1e-3,
            scan_sampling_row_A=0.5, scan_sampling_col_A=0.5, dc_re=1.0, dc_im=0.0)

    def features(self, aberrations: np.ndarray, rng: np.random.Generator,
                 sigma: tuple[float, float] = (0.02, 1.0), seed: int = 0,
                 chunk: int = 4096, informative: tuple[int, int] | None = None,
                 amplitude_contrast: tuple[float, float] = (0.0, 0.5)) -> torch.Tensor:
        """BF16 features [n, N_IN] of the forward model at ``aberrations`` [n, 4].
        Each sample keeps between ``informative`` = (lo, hi) of its maps at a
        noise level drawn log-uniformly in ``sigma`` (default half .. all of
        them: the crystal's reflections all carry signal, some weakly) and
        drowns the rest; its amplitude part is a fraction of the phase part
        drawn uniformly in ``amplitude_contrast``, with a random phase."""
        n = int(aberrations.shape[0])
        nq = len(Q_UNITS)
        out = torch.empty((n, N_IN), dtype=torch.bfloat16, device=self.device)
        lat = self.lattice
        for s in range(0, n, chunk):
            e = min(n, s + chunk)
            m = e - s
            ab = torch.as_tensor(np.ascontiguousarray(aberrations[s:e], np.float32), device=self.device)
            amp = np.exp(rng.uniform(np.log(0.2), np.log(5.0), size=(m, nq)))
            ph = rng.uniform(0, 2 * np.pi, size=(m, nq))
            amp_a = amp * rng.uniform(*amplitude_contrast, size=(m, nq))
            ph_a = rng.uniform(0, 2 * np.pi, size=(m, nq))
            phi = np.stack([np.stack([amp * np.cos(ph), amp * np.sin(ph)], axis=-1),
                            np.stack([amp_a * np.cos(ph_a), amp_a * np.sin(ph_a)], axis=-1)],
                           axis=2).astype(np.float32)     # [m, nq, 2, 2]
            # one noise level per map: a crystal's reflections differ in
            # strength, so each sample keeps a random number of informative
            # maps and drowns the rest
            lo_n, hi_n = (nq // 2, nq) if informative is None else informative
            n_good = rng.integers(lo_n, hi_n + 1, size=m)
            good = rng.random((m, nq)).argsort(axis=1) < n_good[:, None]
            lo = rng.uniform(np.log(sigma[0]), np.log(sigma[1]), size=(m, nq))
            hi = rng.uniform(np.log(2.0), np.log(50.0), size=(m, nq))
            sig = np.exp(np.where(good, lo, hi)).astype(np.float32)
            phi_d = torch.as_tensor(phi, device=self.device)
            sig_d = torch.as_tensor(sig, device=self.device)
            scratch = torch.empty(m * nq * lat.n_bf, dtype=torch.float32, device=self.device)
            _call("qssb_synth_features", self.device, _ptr(self.geom), lat.n_bf, _ptr(self.q_vec),
                  nq, _ptr(ab), _ptr(phi_d), _ptr(sig_d), m, ctypes.byref(self.cal),
                  ctypes.c_uint64(seed * 1_000_003 + s), _ptr(lat.off), _ptr(lat.idx), _ptr(lat.w),
                  GRID * GRID, _ptr(scratch), None, _ptr(out[s:e]), _stream(self.device))
        return out


# ---------------------------------------------------------------- targets
def canonical_targets(ab: np.ndarray) -> np.ndarray:
    """(C10, C12, phi12, C30) -> scaled (C1, A1 cos 2phi, A1 sin 2phi, C3), with
    every aberration's sign flipped where C1 < 0."""
    ab = np.asarray(ab, np.float64)
    s = np.where(ab[:, 0] < 0, -1.0, 1.0)
    t = np.stack([s * ab[:, 0], s * ab[:, 1] * np.cos(2 * ab[:, 2]),
                  s * ab[:, 1] * np.sin(2 * ab[:, 2]), s * ab[:, 3]], axis=1)
    return (t / OUT_SCALE).astype(np.float32)


def decode(pred: np.ndarray) -> np.ndarray:
    """Scaled outputs [n, 4] -> aberrations (C10, C12, phi12, C30) [n, 4]."""
    p = np.asarray(pred, np.float64) * OUT_SCALE
    c12 = np.hypot(p[:, 1], p[:, 2])
    phi = 0.5 * np.arctan2(p[:, 2], p[:, 1])
    return np.stack([p[:, 0], c12, np.mod(phi, np.pi), p[:, 3]], axis=1)


def flipped(ab: np.ndarray) -> np.ndarray:
    """Every aberration negated: C10 -> -C10, A1 -> -A1 (phi12 + pi/2), C30 -> -C30."""
    ab = np.array(ab, np.float64, ndmin=2)
    return np.stack([-ab[:, 0], ab[:, 1], np.mod(ab[:, 2] + np.pi / 2, np.pi), -ab[:, 3]], axis=1)


# -------------------------------------------------------------------- MLP
class MLP:
    """16384 -> 512 -> 512 -> 512 -> HEADS x 4, GELU, BF16 weights on the
    tensor cores, FP32 master weights and Adam; every step in the C ABI."""

    def __init__(self, device, seed: int = 0):
        self.device = torch.device(device)
        g = torch.Generator(device=self.device).manual_seed(seed)
        dims = [N_IN, HIDDEN, HIDDEN, HIDDEN, N_OUT_PAD]
        self.w, self.b = [], []
        for i in range(4):
            fan_in = dims[i]
            w = torch.randn((dims[i], dims[i + 1]), generator=g, device=self.device) * math.sqrt(2.0 / fan_in)
            b = torch.zeros(dims[i + 1], device=self.device)
            if i == 3:
                # small output weights; the heads start from spread biases so
                # that they split the winners from the first steps
                w *= 0.1
                b = torch.linspace(-0.5, 0.5, dims[i + 1], device=self.device)
            self.w.append(w.contiguous())
            self.b.append(b)
        self.dims = dims
        self.w_bf = [w.to(torch.bfloat16).contiguous() for w in self.w]
        self.m = [torch.zeros_like(t) for t in self.w + self.b]
        self.v = [torch.zeros_like(t) for t in self.w + self.b]
        self.t = 0
        self._bufs: dict = {}
        self._tc_ws: torch.Tensor | None = None
        self._out_weight = torch.as_tensor(OUT_WEIGHT, device=self.device)

    # buffers per batch size
    def _buf(self, m: int) -> dict:
        b = self._bufs.get(m)
        if b is None:
            dev = self.device
            b = {
                "z": [torch.empty((m, d), device=dev) for d in self.dims[1:]],
                "a": [torch.empty((m, d), dtype=torch.bfloat16, device=dev) for d in self.dims[1:4]],
                "dy": torch.empty((m, N_OUT_PAD), device=dev),
                "dy_bf": torch.empty((m, N_OUT_PAD), dtype=torch.bfloat16, device=dev),
                "da": [torch.empty((m, d), device=dev) for d in self.dims[1:4]],
                "dz": [torch.empty((m, d), device=dev) for d in self.dims[1:4]],
                "dz_bf": [torch.empty((m, d), dtype=torch.bfloat16, device=dev) for d in self.dims[1:4]],
                "gw": [torch.empty_like(w) for w in self.w],
                "gb": [torch.empty_like(x) for x in self.b],
                "loss": torch.empty(1, device=dev),
                "winner": torch.empty(m, dtype=torch.int32, device=dev),
            }
            self._bufs[m] = b
        return b

    # the large GEMMs (M, N multiples of 128, K of 64) run on the tcgen05
    # kernel, split over K until about two CTAs per SM; the rest on the warp MMA
    use_tc = True

    @staticmethod
    def _tc_splits(m: int, n: int, k: int) -> int:
        tiles = (m // 128) * (n // 128)
        splits = 1
        while tiles * splits * 2 <= 296 and k % (64 * splits * 2) == 0 and k // (splits * 2) >= 256:
            splits *= 2
        return splits

    def _gemm(self, a, lda, ta, bmat, ldb, tb, m, n, k, bias=None, c=None, ldc=0, act=None,
              ld_act=0, accumulate=False):
        if self.use_tc and m % 128 == 0 and n % 128 == 0 and k % 64 == 0:
            splits = self._tc_splits(m, n, k)
            need = ctypes.c_size_t(0)
            _lib.check(_lib.load().qssb_gemm_tc_workspace_bytes(m, n, k, splits, ctypes.byref(need)))
            if self._tc_ws is None or self._tc_ws.numel() < need.value:
                self._tc_ws = torch.empty(need.value, dtype=torch.uint8, device=self.device)
            _call("qssb_gemm_bf16_tc", self.device, _ptr(a), lda, int(ta), _ptr(bmat), ldb, int(tb),
                  m, n, k, splits, _ptr(bias), int(accumulate), _ptr(c), ldc, _ptr(act), ld_act,
                  _ptr(self._tc_ws), need.value, _stream(self.device))
            return
        _call("qssb_gemm_bf16", self.device, _ptr(a), lda, int(ta), _ptr(bmat), ldb, int(tb), m, n,
              k, _ptr(bias), int(accumulate), _ptr(c), ldc, _ptr(act), ld_act, _stream(self.device))

    def forward(self, x: torch.Tensor) -> torch.Tensor:
        """x: BF16 [m, N_IN] (m a multiple of 16) -> FP32 [m, N_OUT_PAD]."""
        m = int(x.shape[0])
        if m % 16 or x.dtype != torch.bfloat16 or x.shape[1] != N_IN:
            raise ValueError("x must be BF16 [m, 16384] with m a multiple of 16")
        bf = self._buf(m)
        inp = x
        for i in range(4):
            k, n = self.dims[i], self.dims[i + 1]
            act = bf["a"][i] if i < 3 else None
            self._gemm(inp, k, False, self.w_bf[i], n, False, m, n, k, bias=self.b[i],
                       c=bf["z"][i], ldc=n, act=act, ld_act=n)
            inp = act
        self._x = x
        return bf["z"][3]

    def backward_and_step(self, target: torch.Tensor, lr: float, wd: float = 1e-5,
                          hyper: torch.Tensor | None = None) -> torch.Tensor:
        """Winner-takes-all MSE of the heads against target [m, N_OUT] (FP32;
        winner by (C1, A1), C3 weighted by OUT_WEIGHT), gradients, one Adam
        step; returns the loss (device). With ``hyper`` (device {lr, c1, c2}
        from ``qssb_adam_schedule``) the step takes its learning rate and bias
        corrections from there, so that it can be replayed from a graph."""
        bf = self._buf(int(target.shape[0]))
        m = int(target.shape[0])
        dev = self.device
        _call("qssb_mse_heads", dev, _ptr(bf["z"][3]), _ptr(target), m, N_OUT, HEADS, N_OUT_PAD,
              _ptr(self._out_weight), 3, ctypes.c_float(WTA_EPS), _ptr(bf["dy"]), _ptr(bf["loss"]),
              _ptr(bf["winner"]), _stream(dev))
        _call("qssb_to_bf16", dev, _ptr(bf["dy"]), m * N_OUT_PAD, _ptr(bf["dy_bf"]), _stream(dev))
        grad_bf, grad_f = bf["dy_bf"], bf["dy"]
        for i in (3, 2, 1, 0):
            k, n = self.dims[i], self.dims[i + 1]
            a_in = self._x if i == 0 else bf["a"][i - 1]
            # dW_i = A_in^T dZ_i ; db_i = colsum dZ_i
            self._gemm(a_in, k, True, grad_bf, n, False, k, n, m, c=bf["gw"][i], ldc=n)
            _call("qssb_bias_grad", dev, _ptr(grad_f), m, n, _ptr(bf["gb"][i]), _stream(dev))
            if i > 0:
                # dA_{i-1} = dZ_i W_i^T, then through GELU'
                self._gemm(grad_bf, n, False, self.w_bf[i], n, True, m, k, n, c=bf["da"][i - 1], ldc=k)
                _call("qssb_gelu_backward", dev, _ptr(bf["da"][i - 1]), _ptr(bf["z"][i - 1]), m * k,
                      _ptr(bf["dz_bf"][i - 1]), _ptr(bf["dz"][i - 1]), _stream(dev))
                grad_bf, grad_f = bf["dz_bf"][i - 1], bf["dz"][i - 1]
        self.t += 1
        params = self.w + self.b
        grads = bf["gw"] + bf["gb"]
        for j, (p, gr) in enumerate(zip(params, grads)):
            wbf = self.w_bf[j] if j < 4 else None
            if hyper is None:
                _call("qssb_adam", dev, _ptr(p), _ptr(self.m[j]), _ptr(self.v[j]), _ptr(gr),
                      p.numel(), ctypes.c_float(lr), ctypes.c_float(ADAM_BETAS[0]),
                      ctypes.c_float(ADAM_BETAS[1]), ctypes.c_float(1e-8),
                      ctypes.c_float(wd if j < 4 else 0.0), self.t, _ptr(wbf), _stream(dev))
            else:
                _call("qssb_adam_dev", dev, _ptr(p), _ptr(self.m[j]), _ptr(self.v[j]), _ptr(gr),
                      p.numel(), _ptr(hyper), ctypes.c_float(ADAM_BETAS[0]),
                      ctypes.c_float(ADAM_BETAS[1]), ctypes.c_float(1e-8),
                      ctypes.c_float(wd if j < 4 else 0.0), _ptr(wbf), _stream(dev))
        return bf["loss"]

    def predict(self, x: torch.Tensor) -> np.ndarray:
        """Scaled outputs [m, HEADS, N_OUT] of x [m, N_IN]. The rows are padded
        with zeros to a multiple of 128 (each row's outputs depend on that row
        only) so that the large layers run on the tcgen05 kernel: one proposal
        (16 rows on the warp MMA) took 0.66 ms, 8 CTAs for the 16384-wide layer."""
        m = int(x.shape[0])
        pad = (-m) % (128 if self.use_tc else 16)
        if pad:
            x = torch.cat([x, torch.zeros((pad, N_IN), dtype=x.dtype, device=x.device)])
        return self.forward(x)[:m, :HEADS * N_OUT].cpu().numpy().reshape(m, HEADS, N_OUT)


class Proposer:
    """Trains the MLP on forward-model features and proposes aberrations."""

    def __init__(self, device, seed: int = 0):
        self.device = torch.device(device)
        self.lattice = TrainingLattice(self.device)
        self.mlp = MLP(self.device, seed)
        self.seed = seed
        self.history: list[float] = []

    def make_data(self, n: int, seed: int) -> tuple[torch.Tensor, torch.Tensor, np.ndarray]:
        from .synthetic import draw_aberrations

        rng = np.random.default_rng(seed)
        ab = draw_aberrations(rng, n)
        x = self.lattice.features(ab, rng, seed=seed)
        t = torch.as_tensor(canonical_targets(ab), device=self.device)
        return x, t, ab

    def train(self, n_samples: int = 50_000, epochs: int = 40, batch: int = 256,
              lr: float = 1e-3, use_graph: bool = True) -> dict:
        """Adam with a cosine learning rate over ``epochs`` shuffled passes.

        Every step gathers its batch through a device index (this epoch's
        permutation at a device cursor), runs forward, the winner-takes-all
        loss, backward and the Adam update with the schedule computed on the
        device (``qssb_adam_schedule``). The first step runs eagerly; the
        rest replay it as one CUDA graph (``use_graph``), so the ~45 launches
        of a step cost one host call. The per-epoch losses are read after
        each epoch's last step."""
        x, t, _ = self.make_data(n_samples, self.seed)
        dev = self.device
        steps_per_epoch = n_samples // batch
        total = epochs * steps_per_epoch
        g = torch.Generator(device=dev).manual_seed(self.seed + 1)
        perm = torch.empty(n_samples, dtype=torch.int64, device=dev)
        base = torch.arange(batch, dtype=torch.int64, device=dev)
        pos = torch.empty_like(base)
        idx = torch.empty_like(base)
        xb = torch.empty((batch, N_IN), dtype=x.dtype, device=dev)
        tb = torch.empty((batch, N_OUT), dtype=t.dtype, device=dev)
        hyper = torch.zeros(4, device=dev)
        step_ctr = torch.zeros(1, dtype=torch.int32, device=dev)
        mlp = self.mlp
        t0 = mlp.t
        step_ctr.fill_(t0)

        def one_step() -> torch.Tensor:
            torch.index_select(perm, 0, pos, out=idx)
            torch.index_select(x, 0, idx, out=xb)
            torch.index_select(t, 0, idx, out=tb)
            pos.add_(batch)
            _call("qssb_adam_schedule", dev, _ptr(hyper), _ptr(step_ctr), t0, total,
                  ctypes.c_float(lr), ctypes.c_float(ADAM_BETAS[0]), ctypes.c_float(ADAM_BETAS[1]),
                  _stream(dev))
            mlp.forward(xb)
            return mlp.backward_and_step(tb, lr, hyper=hyper)

        graph = None
        loss_t = None
        losses = []
        for _ in range(epochs):
            perm.copy_(torch.randperm(n_samples, generator=g, device=dev))
            pos.copy_(base)
            for _s in range(steps_per_epoch):
                if graph is not None:
                    graph.replay()
                    continue
                loss_t = one_step()
                if use_graph:
                    torch.cuda.synchronize(dev)
                    graph = torch.cuda.CUDAGraph()
                    with torch.cuda.graph(graph, capture_error_mode="relaxed"):
                        loss_t = one_step()
            losses.append(float(loss_t.item()))
        mlp.t = int(step_ctr.item())
        self.history = losses
        return {"epochs": epochs, "steps": mlp.t - t0, "graph": graph is not None,
                "final_train_mse": losses[-1] if losses else None}

    def validate(self, n: int = 2048, seed: int = 12345) -> dict:
        """Errors of the best head per sample (the head nearest the target in
        (C1, A1), as the refinement's first batch picks it by loss) on fresh
        forward-model samples: RMS and median, scaled and in A."""
        x, t, _ = self.make_data(n, seed)
        pred = self.mlp.predict(x)
        tt = t.cpu().numpy()
        d = pred - tt[:, None, :]
        win = np.argmin(np.sum(d[..., :3] ** 2, axis=-1), axis=1)
        err = d[np.arange(len(d)), win]
        rmse = np.sqrt(np.mean(err ** 2, axis=0))
        return {"rmse_scaled": rmse.tolist(), "rmse_units": (rmse * OUT_SCALE).tolist(),
                "median_abs_units": (np.median(np.abs(err), axis=0) * OUT_SCALE).tolist()}

    def propose(self, be) -> np.ndarray:
        """2 x HEADS hypotheses [8, 4] (C10, C12, phi12, C30): each head's
        canonical proposal followed by its sign flip."""
        z = self.mlp.predict(backend_features(be))[0]
        out = []
        for h in range(HEADS):
            p = decode(z[h][None])
            out += [p[0], flipped(p)[0]]
        return np.stack(out)


# ------------------------------------------------------------- refinement
# Searches move in x = (C10, a, b, C30) with the astigmatism in Cartesian form
# (a, b) = C12 (cos 2 phi12, sin 2 phi12), so a box around a point is a box.
BOX_LO = np.array([SWEEP_RANGES["C10"][0], -SWEEP_RANGES["C12"][1], -SWEEP_RANGES["C12"][1],
                   SWEEP_RANGES["C30"][0]])
BOX_HI = np.array([SWEEP_RANGES["C10"][1], SWEEP_RANGES["C12"][1], SWEEP_RANGES["C12"][1],
                   SWEEP_RANGES["C30"][1]])


def to_x(ab: np.ndarray) -> np.ndarray:
    ab = np.array(ab, np.float64, ndmin=2)
    return np.stack([ab[:, 0], ab[:, 1] * np.cos(2 * ab[:, 2]), ab[:, 1] * np.sin(2 * ab[:, 2]),
                     ab[:, 3]], axis=1)


def from_x(x: np.ndarray) -> np.ndarray:
    x = np.array(x, np.float64, ndmin=2)
    return np.stack([x[:, 0], np.hypot(x[:, 1], x[:, 2]),
                     np.mod(0.5 * np.arctan2(x[:, 2], x[:, 1]), np.pi), x[:, 3]], axis=1)


def zoom_search(be, centres: np.ndarray | None, half_widths: np.ndarray, batch: int, rounds: int,
                shrink: float, rng: np.random.Generator, done=None, lo=None, hi=None,
                history: tuple[list, list] | None = None):
    """Batched zoom search on the phase-variance loss in x = (C10, a, b, C30):
    each round scores ``batch`` candidates in one ``qssb_loss_batch`` call (the
    current best plus uniform draws in a box around it; the first round splits
    them over ``centres``), keeps the best and shrinks the box by ``shrink``.
    ``done(best_aberrations)`` ends it early. Returns (best (C10, C12, phi12,
    C30), SSB evaluations, rounds)."""
    lo = BOX_LO if lo is None else np.asarray(lo, np.float64)
    hi = BOX_HI if hi is None else np.asarray(hi, np.float64)
    w = np.asarray(half_widths, np.float64).copy()
    if centres is None:  # no prior point: the first round spreads over the whole box
        centres = np.empty((0, 4))
    centres = np.clip(np.array(centres, np.float64, ndmin=2).reshape(-1, 4), lo, hi)
    best_x, best_loss = (centres[0].copy() if len(centres) else (lo + hi) / 2), np.inf
    evals = 0
    for r in range(rounds):
        if r == 0 and len(centres) == 0:
            cand = lo + rng.random((batch, 4)) * (hi - lo)
        elif r == 0:
            per = max(1, batch // len(centres))
            cand = []
            for c in centres:
                cand.append(c)
                cand.extend(c + rng.uniform(-1, 1, size=(per - 1, 4)) * w)
            cand = np.array(cand[:batch])
            if len(cand) < batch:
                cand = np.vstack([cand, centres[0] + rng.uniform(-1, 1, size=(batch - len(cand), 4)) * w])
        else:
            cand = np.vstack([best_x, best_x + rng.uniform(-1, 1, size=(batch - 1, 4)) * w])
        cand = np.clip(cand, lo, hi)
        ab = from_x(cand)
        losses = be.variance_loss_batch(ab[:, 0], ab[:, 1], ab[:, 2], ab[:, 3]).cpu().numpy()
        evals += batch
        if history is not None:
            history[0].extend(cand)
            history[1].extend(float(v) for v in losses)
        j = int(np.argmin(losses))
        if losses[j] < best_loss:
            best_x, best_loss = cand[j].copy(), float(losses[j])
        w *= shrink
        if done is not None and done(from_x(best_x)[0]):
            return from_x(best_x)[0], evals, r + 1
    return from_x(best_x)[0], evals, rounds


def compass_search(be, start: np.ndarray, steps: np.ndarray, rounds: int, done=None,
                   lo=None, hi=None, grow: float = 1.0, shrink: float = 0.5):
    """Batched pattern search for the 8-candidate refinement: each round scores
    the 8 points x +- s_i e_i (one ``qssb_loss_batch`` call); the best point
    becomes the centre if it beats it, otherwise every step halves. The start
    points (the proposal's two sign hypotheses) are scored first in one batch.
    Returns (best (C10, C12, phi12, C30), SSB evaluations, rounds)."""
    lo = BOX_LO if lo is None else np.asarray(lo, np.float64)
    hi = BOX_HI if hi is None else np.asarray(hi, np.float64)
    starts = np.clip(np.array(start, np.float64, ndmin=2).reshape(-1, 4), lo, hi)
    ab = from_x(starts)
    losses = be.variance_loss_batch(ab[:, 0], ab[:, 1], ab[:, 2], ab[:, 3]).cpu().numpy()
    evals = len(starts)
    j = int(np.argmin(losses))
    x, fx = starts[j].copy(), float(losses[j])
    s = np.asarray(steps, np.float64).copy()
    if done is not None and done(from_x(x)[0]):
        return from_x(x)[0], evals, 0
    eye = np.eye(4)
    for r in range(rounds):
        cand = np.clip(np.vstack([x + s * eye, x - s * eye]), lo, hi)
        ab = from_x(cand)
        losses = be.variance_loss_batch(ab[:, 0], ab[:, 1], ab[:, 2], ab[:, 3]).cpu().numpy()
        evals += len(cand)
        j = int(np.argmin(losses))
        if losses[j] < fx:
            x, fx = cand[j].copy(), float(losses[j])
            s *= grow
        else:
            s *= shrink
        if done is not None and done(from_x(x)[0]):
            return from_x(x)[0], evals, r + 1
    return from_x(x)[0], evals, rounds


def _quadratic_design(u: np.ndarray, kind: str) -> np.ndarray:
    """Columns of a quadratic model in u [n, d]: 1, u_i, then u_i u_j (i <= j,
    kind "full") or u_i^2 (kind "diag"); kind "linear" stops after u_i."""
    n, d = u.shape
    cols = [np.ones(n), *u.T]
    if kind == "full":
        cols += [u[:, i] * u[:, j] for i in range(d) for j in range(i, d)]
    elif kind == "diag":
        cols += [u[:, i] * u[:, i] for i in range(d)]
    return np.stack(cols, axis=1)


def _model_step(coef: np.ndarray, d: int, kind: str, radius: float) -> np.ndarray:
    """Minimiser of the fitted quadratic within |u| <= radius: the Newton step
    when the Hessian is positive definite and the step fits, else the
    trust-region step (H + lambda I) u = -g with lambda found by bisection."""
    g = coef[1:1 + d]
    h = np.zeros((d, d))
    if kind == "full":
        k = 1 + d
        for i in range(d):
            for j in range(i, d):
                if i == j:
                    h[i, i] = 2.0 * coef[k]
                else:
                    h[i, j] = h[j, i] = coef[k]
                k += 1
    elif kind == "diag":
        h = np.diag(2.0 * coef[1 + d:1 + 2 * d])
    gn = float(np.linalg.norm(g))
    if kind == "linear" or gn == 0.0:
        return -radius * g / gn if gn > 0 else np.zeros(d)
    lam_min = float(np.linalg.eigvalsh(h).min())
    if lam_min > 0:
        u = np.linalg.solve(h, -g)
        if np.linalg.norm(u) <= radius:
            return u
    lo_l, hi_l = max(0.0, -lam_min) + 1e-12, max(0.0, -lam_min) + gn / radius + 1.0
    for _ in range(60):
        lam = 0.5 * (lo_l + hi_l)
        u = np.linalg.solve(h + lam * np.eye(d), -g)
        if np.linalg.norm(u) > radius:
            lo_l = lam
        else:
            hi_l = lam
    return np.linalg.solve(h + hi_l * np.eye(d), -g)


def surrogate_search(be, starts: np.ndarray, widths: np.ndarray, batch: int, rounds: int,
                     rng: np.random.Generator, done=None, lo=None, hi=None,
                     radius0: float = 0.5, min_radius: float = 1e-4, history=None):
    """Trust-region refinement with a quadratic surrogate of the
    phase-variance loss, ``batch`` SSB evaluations per round (one
    ``qssb_loss_batch`` call), in x = (C10, a, b, C30) scaled by ``widths``.

    Round 0 scores the start points (a proposal's two sign hypotheses) and
    draws around the first. Each later round fits a weighted least-squares
    quadratic (full, then diagonal, then linear as the points allow) to the
    scored points nearest the incumbent, takes its minimiser within the trust
    radius, and scores it, half of that step, and points at half the radius
    around it (which keep the next fit well posed). The radius doubles when
    the full step hits the boundary and wins, and halves when nothing beats
    the incumbent. ``done(best_aberrations)`` ends it early. Returns
    (best (C10, C12, phi12, C30), SSB evaluations, rounds). ``history``
    (scored points (xs, losses) of an earlier search on the same data) seeds
    the fits; its evaluations are not counted again."""
    lo = BOX_LO if lo is None else np.asarray(lo, np.float64)
    hi = BOX_HI if hi is None else np.asarray(hi, np.float64)
    w = np.asarray(widths, np.float64)
    d = 4
    xs: list[np.ndarray] = [] if history is None else [np.asarray(x, np.float64) for x in history[0]]
    fs: list[float] = [] if history is None else [float(f) for f in history[1]]
    n_prior = len(fs)

    def score(cand: np.ndarray) -> None:
        cand = np.clip(cand, lo, hi)
        ab = from_x(cand)
        losses = be.variance_loss_batch(ab[:, 0], ab[:, 1], ab[:, 2], ab[:, 3]).cpu().numpy()
        xs.extend(cand)
        fs.extend(float(v) for v in losses)

    starts = np.clip(np.array(starts, np.float64, ndmin=2).reshape(-1, d), lo, hi)[:batch]
    extra = batch - len(starts)
    cand = starts
    if extra > 0:
        cand = np.vstack([starts, starts[0] + rng.normal(0.0, radius0, (extra, d)) * w])
    score(cand)
    best = int(np.argmin(fs))
    c, fc = xs[best].copy(), fs[best]
    radius = radius0
    if done is not None and done(from_x(c)[0]):
        return from_x(c)[0], len(fs) - n_prior, 0
    for r in range(1, rounds):
        X = np.asarray(xs)
        F = np.asarray(fs)
        U = (X - c) / w
        dist = np.linalg.norm(U, axis=1)
        order = np.argsort(dist)
        near = order[dist[order] <= 2.0 * radius]
        if len(near) < 24:
            near = order[:min(len(order), 24)]
        n = len(near)
        kind = "full" if n >= 18 else ("diag" if n >= 11 else "linear")
        A = _quadratic_design(U[near], kind)
        wt = 1.0 / (1.0 + (dist[near] / radius) ** 2)
        coef = np.linalg.lstsq(A * wt[:, None], (F[near] - fc) * wt, rcond=None)[0]
        u = _model_step(coef, d, kind, radius)
        step = c + u * w
        v = rng.normal(size=(batch - 2, d))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        cand = np.vstack([step, c + 0.5 * u * w, step + 0.5 * radius * v * w])
        n0 = len(fs)
        score(cand)
        j = n0 + int(np.argmin(fs[n0:]))
        if fs[j] < fc:
            moved = float(np.linalg.norm((xs[j] - c) / w))
            c, fc = xs[j].copy(), fs[j]
            # the radius follows the step: doubled when a full step to the
            # boundary won, else twice the distance moved (at most a quarter
            # of the old radius less)
            if j == n0 and np.linalg.norm(u) >= 0.9 * radius:
                radius = min(2.0 * radius, 2.0)
            else:
                radius = min(radius, max(2.0 * moved, 0.25 * radius))
        else:
            radius *= 0.5
        if done is not None and done(from_x(c)[0]):
            return from_x(c)[0], len(fs) - n_prior, r + 1
        if radius < min_radius:
            break
    return from_x(c)[0], len(fs) - n_prior, rounds


REFINE_MARGIN = 0.1  # the refinement may step this share of each range beyond the sweep box


def refine_box() -> tuple[np.ndarray, np.ndarray]:
    """Bounds of the refinement: the sweep box widened by REFINE_MARGIN of its
    span on each side (a truth on the box's edge stays inside the designs)."""
    span = BOX_HI - BOX_LO
    return BOX_LO - REFINE_MARGIN * span, BOX_HI + REFINE_MARGIN * span


def _local_design(centre: np.ndarray, r: float, dims: int, batch: int,
                  with_centre: bool) -> np.ndarray:
    """The centre (optional), centre +- r e_i (i < dims), then centre + r (e_i +- e_k)/sqrt 2
    until ``batch`` points."""
    eye = np.eye(4)[:dims]
    pts = [centre] if with_centre else []
    pts += [centre + s * r * e for e in eye for s in (1.0, -1.0)]
    pairs = [(i, k) for i in range(dims) for k in range(i + 1, dims)]
    for sign in (1.0, -1.0):
        for i, k in pairs:
            pts.append(centre + r * (eye[i] + sign * eye[k]) / math.sqrt(2.0))
    while len(pts) < batch:  # more points than the patterns: a wider axial ring
        j = len(pts)
        pts.append(centre + 2.0 * r * (1.0 if j % 2 else -1.0) * eye[(j // 2) % dims])
    return np.asarray(pts[:batch])


def quadratic_refine(be, hypotheses: np.ndarray, step: float, batch: int, rounds: int,
                     done=None, lo=None, hi=None, dims: int = 3, min_step: float = 0.05):
    """The short refinement a proposal seeds: ``batch`` SSB evaluations per
    round, each round one ``qssb_loss_batch`` call, in x = (C10, a, b, C30).

    Round 0 scores the hypotheses (the proposal's heads and signs; spare
    slots take the design below around the first) and keeps the best as the
    centre c. Later rounds move the first ``dims`` coordinates
    (C1, A1; C3 stays at the hypothesis's value - it shifts the phase by about
    1e-5 rad per 1000 A on the 64^2 test scans): while fewer than 1 + 2 dims
    scored points lie within 3 rho of c, a round scores the design
    c +- rho e_i plus diagonals; after that it fits a quadratic in (x - c) /
    rho (diagonal Hessian below 1 + dims + dims (dims + 1) / 2 + 2 points,
    full above; weights 1 / (1 + d^2)) to those points, steps to the model's
    minimiser within 2 rho and scores that point with a design of radius
    rho / 2 around it (which keeps the next fit posed). rho starts at
    ``step`` (A), follows accepted moves (twice the move, at least half the
    old rho, never more) and halves when a round finds nothing better.
    Returns (best (C10, C12, phi12, C30), SSB evaluations, rounds, ok): ok
    means ``done(best)`` held, or, without ``done``, that rho fell below
    ``min_step`` within ``rounds``."""
    if lo is None or hi is None:
        lo, hi = refine_box()
    xs: list[np.ndarray] = []
    fs: list[float] = []

    def score(cand: np.ndarray) -> None:
        cand = np.clip(np.asarray(cand, np.float64), lo, hi)
        ab = from_x(cand)
        losses = be.variance_loss_batch(ab[:, 0], ab[:, 1], ab[:, 2], ab[:, 3]).cpu().numpy()
        xs.extend(cand)
        fs.extend(float(v) for v in losses)

    rho = float(step)
    hyp = np.array(hypotheses, np.float64, ndmin=2).reshape(-1, 4)[:batch]
    if len(hyp) < batch:  # spare slots: the design around the first hypothesis
        hyp = np.vstack([hyp, _local_design(hyp[0], rho, dims, batch - len(hyp), False)])
    score(hyp)
    j = int(np.argmin(fs))
    c, fc = xs[j].copy(), fs[j]
    if done is not None and done(from_x(c)[0]):
        return from_x(c)[0], len(fs), 1, True
    n_diag = 1 + 2 * dims
    n_full = 1 + dims + dims * (dims + 1) // 2
    for r in range(1, rounds):
        X = np.asarray(xs)
        F = np.asarray(fs)
        U = (X[:, :dims] - c[:dims]) / rho
        dist = np.linalg.norm(U, axis=1)
        near = np.nonzero(dist <= 3.0)[0]
        if len(near) >= n_diag:
            kind = "full" if len(near) >= n_full + 2 else "diag"
            A = _quadratic_design(U[near], kind)
            wt = 1.0 / (1.0 + dist[near] ** 2)
            coef = np.linalg.lstsq(A * wt[:, None], (F[near] - fc) * wt, rcond=None)[0]
            u = np.zeros(4)
            u[:dims] = _model_step(coef, dims, kind, 2.0) * rho
            cand = _local_design(c + u, 0.5 * rho, dims, batch, with_centre=True)
        else:
            cand = _local_design(c, rho, dims, batch, with_centre=False)
        n0 = len(fs)
        score(cand)
        k = n0 + int(np.argmin(fs[n0:]))
        if fs[k] < fc:
            moved = float(np.linalg.norm(xs[k][:dims] - c[:dims]))
            c, fc = xs[k].copy(), fs[k]
            rho = min(rho, max(2.0 * moved, 0.5 * rho))
        else:
            rho *= 0.5
        if done is not None and done(from_x(c)[0]):
            return from_x(c)[0], len(fs), r + 1, True
        if rho < min_step:
            return from_x(c)[0], len(fs), r + 1, done is None
    return from_x(c)[0], len(fs), rounds, False


def learned_refine(be, hypotheses: np.ndarray, step: float = 8.0, batch: int = 8,
                   rounds: int = 12, rng: np.random.Generator | None = None, done=None,
                   fallback_rounds: int = 200):
    """Proposal + refinement with the plain sweep as the fallback:
    ``quadratic_refine`` from the hypotheses, and when it does not end ok
    (``done`` unmet, or no convergence within ``rounds``) the plain
    64-candidate zoom sweep over the whole box, whose evaluations are added.
    Returns (best (C10, C12, phi12, C30), SSB evaluations, rounds,
    fell_back)."""
    best, ev, r, ok = quadratic_refine(be, hypotheses, step, batch, rounds, done=done)
    if ok:
        return best, ev, r, False
    rng = np.random.default_rng(0) if rng is None else rng
    best2, ev2, r2 = zoom_search(be, None, (BOX_HI - BOX_LO) / 2, 64, fallback_rounds, 0.75, rng,
                                 done=done)
    return best2, ev + ev2, r + r2, True
