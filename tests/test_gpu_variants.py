"""Tile and launch shapes the autotuner chooses between: every BF-gather
variant (``qssb_gather_bf_columns_2d_ex``) and every scan-FFT variant
(``qssb_scan_fft_half_ex``) gives the same bits as the built-in choice; the
trotter tile variants (2, 4, 8 frequencies per thread) agree with it to
float32 rounding and each repeats its own bits; the autotuner returns a
valid choice and caches it; and a tuned cold reconstruction matches an
untuned one."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from quantem.gpu_b200 import _lib, autotune, ops
from quantem.gpu_b200.pipeline import ColdReconstructor
from quantem.gpu_b200.synthetic import CONFIGS, generate

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
KW = dict(semiangle=20.0, scan_sampling=0.5, det_sampling=20.0 / 24.0, voltage_kV=300)


@pytest.fixture(scope="module")
def counts128():
    return generate(CONFIGS["plain_128x128_det128"], device=DEV).counts.contiguous()


def _disk(det, radius):
    rr, cc = np.meshgrid(np.arange(det), np.arange(det), indexing="ij")
    lin = np.nonzero(((rr - det / 2) ** 2 + (cc - det / 2) ** 2).ravel() <= radius ** 2)[0]
    return torch.as_tensor(lin.astype(np.int32), device=DEV)


@pytest.mark.parametrize("frames,det,radius,shuffle", [
    (4096, 128, 26.0, False),   # the 128^2-detector disk
    (1000, 128, 26.0, False),   # frames not a multiple of 8: the 64-frame tiles fall back
    (2048, 192, 60.0, True),    # a wide disk, unsorted BF order
])
def test_every_gather_variant_copies_the_same_bits(frames, det, radius, shuffle):
    g = torch.Generator(device=DEV).manual_seed(frames + det)
    counts = torch.randint(0, 65535, (frames, det, det), generator=g, device=DEV,
                           dtype=torch.int32).to(torch.uint16)
    lin = _disk(det, radius)
    if shuffle:
        lin = lin[torch.randperm(lin.numel(), generator=g, device=DEV)].contiguous()
    want = ops.gather_bf_columns(counts, lin, variant=0)
    ref = counts.view(frames, -1).view(torch.int16)[:, lin.long()].T
    assert torch.equal(want.view(torch.int16), ref)
    for v in range(1, _lib.GATHER_VARIANTS + 1):
        got = ops.gather_bf_columns(counts, lin, validate=False, variant=v)
        assert torch.equal(got.view(torch.int16), want.view(torch.int16)), v
    with pytest.raises(RuntimeError):
        ops.gather_bf_columns(counts, lin, variant=_lib.GATHER_VARIANTS + 1)


@pytest.mark.parametrize("n,n_bf", [(128, 300), (256, 60), (512, 12), (1024, 3)])
def test_every_scan_fft_variant_gives_the_same_bits(n, n_bf):
    g = torch.Generator(device=DEV).manual_seed(n)
    cols = torch.randint(0, 4000, (n_bf, n * n), generator=g, device=DEV,
                         dtype=torch.int32).to(torch.uint16)
    want = ops.scan_fft_half(cols, (n, n), variant=0)
    ref = torch.fft.rfft2(cols.to(torch.float64).view(n_bf, n, n))
    err = (want.to(torch.complex128) - ref).abs().max().item()
    assert err <= 2e-6 * ref.abs().max().item()
    n_var = ops.scan_fft_variants(n)
    assert n_var >= 2
    for v in range(1, n_var + 1):
        got = ops.scan_fft_half(cols, (n, n), variant=v)
        assert torch.equal(got.view(torch.float32), want.view(torch.float32)), (n, v)


def test_trotter_tile_variants_agree(counts128):
    from quantem.gpu_b200 import B200SSBBackend

    be = B200SSBBackend(counts128, device=DEV, **KW)
    cal = be._calibration()
    ab = _lib.Aberrations(-60.0, 20.0, 0.4, 0.0)
    base, _ = ops.object_wave(be.G_qk, be._geom_dev, be._q_row, be._q_col, cal, ab)
    scale = base.abs().max().item()
    for v in (1, 2, 3):
        f = _lib.flag_variant(v)
        a, _ = ops.object_wave(be.G_qk, be._geom_dev, be._q_row, be._q_col, cal, ab, flags=f)
        b, _ = ops.object_wave(be.G_qk, be._geom_dev, be._q_row, be._q_col, cal, ab, flags=f)
        assert torch.equal(a, b), v
        assert (a - base).abs().max().item() <= 2e-6 * scale, v
    be.close()


def test_autotuner_picks_and_caches_shapes(counts128, tmp_path, monkeypatch):
    monkeypatch.setenv("QSSB_TUNING_CACHE", str(tmp_path / "tuning.json"))
    monkeypatch.setattr(autotune, "_CACHE", None)
    lin = _disk(128, 26.0)
    v = autotune.tune_gather(counts128, lin)
    assert 0 <= v <= _lib.GATHER_VARIANTS
    assert autotune.tune_gather(counts128, lin) == v  # a cache hit
    cols = ops.gather_bf_columns(counts128, lin, variant=v)
    f = autotune.tune_scan_fft(cols, (128, 128))
    assert 0 <= f <= ops.scan_fft_variants(128)
    assert (tmp_path / "tuning.json").exists()


def test_tuned_cold_reconstruction_matches_untuned(counts128):
    tuned = ColdReconstructor(counts128, tune=True, **KW)
    plain = ColdReconstructor(counts128, tune=False, **KW)
    a = tuned.run().clone()
    b = plain.run().clone()
    assert (a - b).abs().max().item() <= 1e-5
    st = tuned._b[(tuned.last_info.n_bf, False)]
    assert 0 <= st["gather_variant"] <= _lib.GATHER_VARIANTS
    assert torch.equal(tuned.run(), a)


def test_library_counts_its_own_kernel_launches(counts128):
    """``qssb_kernel_launches``: one launch for a gather, two for a fused 128^2
    loss batch (the phase table and the pair kernel, whose last CTA folds),
    four for an object (trotter, fold, row and column inverse FFTs)."""
    from quantem.gpu_b200 import B200SSBBackend

    lib = _lib.load()
    lin = _disk(128, 26.0)
    n0 = lib.qssb_kernel_launches()
    ops.gather_bf_columns(counts128, lin, validate=False)
    assert lib.qssb_kernel_launches() - n0 == 1
    be = B200SSBBackend(counts128, device=DEV, **KW)
    be.variance_loss_batch([0.0] * 64, [0.0] * 64, [0.0] * 64)  # builds the overlap table
    n0, c0 = lib.qssb_kernel_launches(), ops.LAUNCH_COUNT
    be.variance_loss_batch(list(np.linspace(-50, 50, 64)), [0.0] * 64, [0.0] * 64)
    assert lib.qssb_kernel_launches() - n0 == 2
    assert ops.LAUNCH_COUNT - c0 == 2
    n0 = lib.qssb_kernel_launches()
    be.object_and_phase(10.0, 5.0, 0.1)
    assert lib.qssb_kernel_launches() - n0 == 4
    be.close()
