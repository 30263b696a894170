"""Pin the FP64 oracle against outputs of the reference itself (CPU only).

Fixtures in ``tests/golden/`` were produced by ``tests/golden/make_golden.py``,
which executes the reference's own host code and test restatement (see that
script's docstring). Tolerances follow the reference's precision contract
(``tests/ssb_precision.py:7-10``: phase 2e-4, loss rel 1e-5 / abs 1e-6) except
where the comparison is FP64 oracle vs the reference's float32 arithmetic.
"""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np
import pytest

from oracle import ssb_oracle as so
from recipes import digest, disk_input, synthetic_plain_32

GOLDEN = Path(__file__).resolve().parent / "golden"
PHASE_ATOL = 2.0e-4
LOSS_RTOL = 1.0e-5
LOSS_ATOL = 1.0e-6


def _load(name: str) -> dict:
    with np.load(GOLDEN / f"{name}.npz") as z:
        return {k: z[k] for k in z.files}


CASES = {
    "ref_disk128_bfr3": lambda: disk_input(123),
    "ref_disk96_padded": lambda: disk_input(124, scan=(96, 96)),
    "ref_plain32_auto": synthetic_plain_32,
    # det_sampling=None: BF radius detected from the mean DP (probe.py:12-119)
    "ref_plain32_detect": synthetic_plain_32,
    "ref_disk128_detect": lambda: disk_input(123),
}


def _prepare(name: str):
    gold = _load(name)
    data = CASES[name]()
    assert digest(data) == str(gold["input_sha256"]), "input recipe drifted"
    kw = dict(
        voltage_kV=float(gold["kw_voltage_kV"]),
        semiangle_mrad=float(gold["kw_semiangle"]),
        scan_sampling=float(gold["kw_scan_sampling"]),
        det_sampling=float(gold["kw_det_sampling"]) if "kw_det_sampling" in gold else None,
        bf_radius=float(gold["kw_bf_radius"]) if "kw_bf_radius" in gold else None,
    )
    return gold, data, so.prepare(data, **kw)


@pytest.mark.parametrize("name", sorted(CASES))
def test_selection_and_calibration_match_reference_exactly(name):
    gold, _data, prep = _prepare(name)
    np.testing.assert_array_equal(prep.bf.rows, gold["rows"])
    np.testing.assert_array_equal(prep.bf.cols, gold["cols"])
    assert prep.bf.center == tuple(gold["center"])
    assert prep.wavelength == float(gold["wavelength"])
    np.testing.assert_allclose(prep.sampling, gold["sampling"], rtol=1e-14)
    assert prep.scan_shape == tuple(gold["scan_shape"])
    assert prep.g_half.shape == tuple(gold["g_shape"])


@pytest.mark.parametrize("name", sorted(CASES))
def test_scan_fft_matches_reference_to_float32(name):
    gold, _data, prep = _prepare(name)
    scale = np.abs(prep.g_half).max()
    np.testing.assert_allclose(prep.g_half[:, :4, :4], gold["g_corner"], rtol=0, atol=2e-6 * scale)
    np.testing.assert_allclose(
        (np.abs(prep.g_half) ** 2).sum(axis=(1, 2)), gold["g_abs2_per_bf"], rtol=2e-6
    )
    # The oracle's dc is exact (integer sums); the reference's is a float32 FFT mean.
    assert abs(prep.dc - complex(gold["dc"])) <= 1e-6 * abs(prep.dc)
    if "g_half_first3" in gold:
        np.testing.assert_allclose(prep.g_half[:3], gold["g_half_first3"], rtol=0, atol=2e-6 * scale)


@pytest.mark.parametrize("name", sorted(CASES))
def test_geometry_matches_reference_cache_rotation(name):
    gold, _data, prep = _prepare(name)
    g = prep.geo
    kscale = max(np.abs(g.kx).max(), np.abs(g.ky).max())
    np.testing.assert_allclose(g.kx, gold["kx_bf"], rtol=0, atol=1e-6 * kscale)
    np.testing.assert_allclose(g.ky, gold["ky_bf"], rtol=0, atol=1e-6 * kscale)
    np.testing.assert_allclose(g.alpha_k2, gold["alpha_k2"], rtol=1e-5, atol=1e-12)
    np.testing.assert_allclose(g.cos2phi_k, gold["cos2phi_k"], rtol=0, atol=2e-6)
    np.testing.assert_allclose(g.sin2phi_k, gold["sin2phi_k"], rtol=0, atol=2e-6)
    np.testing.assert_allclose(g.aperture_k, gold["aperture_k"], rtol=0, atol=2e-5)
    np.testing.assert_allclose(g.q_row, gold["qx_1d"], rtol=1e-7)
    np.testing.assert_allclose(g.q_col, gold["qy_1d"], rtol=1e-7)


@pytest.mark.parametrize("name", sorted(CASES))
def test_loss_and_object_match_reference_restatement(name):
    gold, _data, prep = _prepare(name)
    c10, c12, phi12 = (float(v) for v in gold["aberrations"])
    ab = so.Aberrations(C10=c10, C12=c12, phi12=phi12)
    loss, mean_phase = so.phase_variance_loss(prep.g_half, prep.geo, ab, prep.dc)
    assert loss == pytest.approx(float(gold["loss"]), rel=LOSS_RTOL, abs=LOSS_ATOL)
    # Mean of per-BF atan2: a pixel whose phase crosses the branch cut differently
    # shifts the mean by 2 pi / B, so compare the 99.9th percentile like the
    # reference's own chunked tests (test_ssb_cuda_128.py:378-384).
    err = np.abs(so.wrapped_phase_error(mean_phase, gold["mean_phase"]))
    assert np.percentile(err, 99.9) < PHASE_ATOL
    obj, ph = so.reconstruct(prep, ab)
    ref_obj = gold["object"].astype(np.complex128)
    # the detected 8.56 mrad/px sampling of the 16x16 disk puts most (q, k) pairs
    # on the aperture's soft edge, where the reference's float32 arithmetic
    # departs furthest from FP64 (1.2e-5 of max here; 1.3e-6 on the other cases)
    rel = 2e-5 if name == "ref_disk128_detect" else 1e-5
    assert np.abs(obj - ref_obj).max() <= rel * np.abs(obj).max()
    np.testing.assert_array_less(np.abs(so.wrapped_phase_error(ph, np.angle(ref_obj))), 1e-4)


def test_oracle_matches_executable_specification():
    gold, _data, prep = _prepare("ref_disk128_bfr3")
    c10, c12, phi12 = (float(v) for v in gold["aberrations"])
    ab = so.Aberrations(C10=c10, C12=c12, phi12=phi12)
    loss, _ = so.phase_variance_loss(prep.g_half, prep.geo, ab, prep.dc)
    obj, _ = so.reconstruct(prep, ab)
    # The spec ran in FP64 on the reference's float32 G and geometry.
    assert loss == pytest.approx(float(gold["spec_loss"]), rel=1e-5)
    assert np.abs(obj - gold["spec_object"]).max() <= 1e-5 * np.abs(obj).max()


def test_hermitian_extraction_matches_reference():
    gold = _load("ref_arange_hermitian")
    data = np.arange(8 * 8 * 6 * 6, dtype=np.uint16).reshape(8, 8, 6, 6)
    g, dc = so.scan_fft_half(data, gold["rows"], gold["cols"])
    assert g.shape == (4, 8, 5)
    np.testing.assert_allclose(g, gold["g_half"], rtol=1e-6, atol=1e-6 * np.abs(g).max())
    assert dc == pytest.approx(complex(gold["dc"]), rel=1e-7)
    full = so.expand_hermitian(g, 8)
    images = data.reshape(64, 6, 6)[:, gold["rows"], gold["cols"]].T.reshape(4, 8, 8)
    np.testing.assert_allclose(full, np.fft.fft2(images), atol=1e-9)


def test_integer_sums_are_exact_u64():
    """Large uint16 detector sums match an integer reference exactly
    (tests/test_integer_detector_products.py:9-38 pattern)."""
    rng = np.random.default_rng(7)
    data = rng.integers(0, 65536, size=(6, 7, 24, 20), dtype=np.uint16)
    sums, mean_dp = so.mean_dp_u64(data)
    expected = data.reshape(-1, 24, 20).astype(np.uint64).sum(axis=0)
    np.testing.assert_array_equal(sums, expected)
    np.testing.assert_array_equal(mean_dp, expected.astype(np.float32) / np.float32(42))


def test_zero_input_known_answer():
    """Zero spectrum, one BF pixel, dc = 1: the Fourier sum is a delta at DC,
    the object is uniformly 1/N^2 and the loss is 0
    (MetalSSBKernelsTests.swift:35-82)."""
    n = 32
    g = np.zeros((1, n, n // 2 + 1), dtype=np.complex128)
    geo = so.geometry(
        np.asarray([16], np.int32), np.asarray([17], np.int32), (16.0, 16.0), (n, n),
        (0.5, 0.5), (1.0, 1.0), so.wavelength_angstrom(300), 21.4,
    )
    ab = so.Aberrations(C10=0.0, C12=0.0, phi12=0.0)
    fsum = so.fourier_sum(g, geo, ab, 1.0 + 0j)
    assert fsum[0, 0] == 1.0
    assert np.count_nonzero(fsum) == 1
    obj = so.object_wave(g, geo, ab, 1.0 + 0j)
    np.testing.assert_allclose(obj, np.full((n, n), 1.0 / (n * n)), atol=1e-15)
    loss, _ = so.phase_variance_loss(g, geo, ab, 1.0 + 0j)
    assert loss == 0.0


def test_fourier_sum_equals_mean_of_per_bf_objects():
    """IFFT linearity: ifft2(mean_b C_b) == mean_b ifft2(C_b) (engine.py:1047-1107)."""
    gold, _data, prep = _prepare("ref_disk128_bfr3")
    ab = so.Aberrations(C10=-120.0, C12=55.0, phi12=math.radians(17.0))
    direct = np.fft.ifft2(
        so.corrected_spectra(prep.g_half, prep.geo, ab, prep.dc, slice(None))
    ).mean(axis=0)
    obj, _ = so.reconstruct(prep, ab)
    np.testing.assert_allclose(obj, direct, atol=1e-12 * np.abs(obj).max())


def test_padding_rule_targets():
    """Scan padding/cropping targets (backend.py:229-269)."""
    d = np.ones((96, 96, 2, 2), np.uint16)
    assert so.pad_or_crop_scan(d).shape[:2] == (128, 128)
    d = np.ones((160, 120, 2, 2), np.uint16)
    assert so.pad_or_crop_scan(d).shape[:2] == (256, 256)
    d = np.ones((300, 40, 2, 2), np.uint16)
    assert so.pad_or_crop_scan(d).shape[:2] == (512, 512)
    d = np.ones((1100, 8, 1, 1), np.uint16)
    assert so.pad_or_crop_scan(d).shape[:2] == (1024, 1024)
    d = np.ones((128, 128, 2, 2), np.uint16)
    assert so.pad_or_crop_scan(d) is d


def test_bf_companion_matches_reference_writer():
    """The oracle's exact BF companion (suffix and bytes) equals the file the
    reference's own writer produced, on u16 counts that fit u8, the same with
    one hot pixel outside the disk (whole-block rule: stays u16), and u8."""
    import hashlib

    from recipes import export_cases

    gold = _load("ref_bf_export")
    ref = _load("ref_disk128_bfr3")
    for name, data in export_cases().items():
        assert digest(data) == str(gold[name + "_input_sha256"])
        suffix, raw = so.bf_companion(data, ref["rows"], ref["cols"])
        assert suffix == str(gold[name + "_suffix"]), name
        assert len(raw) == int(gold[name + "_bytes"])
        assert hashlib.sha256(raw).hexdigest() == str(gold[name + "_sha256"]), name
    with pytest.raises(TypeError):
        so.bf_companion(disk_input(123).astype(np.float32), ref["rows"], ref["cols"])


@pytest.mark.parametrize("name", ["ref_plain32_detect", "ref_disk128_detect"])
def test_detected_radius_gives_reference_det_sampling(name):
    """det_sampling=None: the detected half-max radius reproduces the
    reference's 2 alpha / r angular sampling exactly (its factor 2 included)."""
    gold = _load(name)
    data = CASES[name]()
    _, mean_dp = so.mean_dp_u64(so.pad_or_crop_scan(data))
    _, r = so.detect_bf_radius(mean_dp)
    want = np.asarray(gold["angular_sampling"], dtype=np.float64)
    assert 2.0 * float(gold["kw_semiangle"]) / r == want[0] == want[1]
