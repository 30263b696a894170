"""End-to-end: u16 counts -> B200SSBBackend / SSB -> object phase, vs the oracle.

Covers the CPU-runnable plain workload (32x32 scan, 64x64 detector, padded
to 128 by the reference rule) and the production workload (128x128 scan,
128x128 detector, ~1800 BF pixels) with the north-star bar of 1e-4 rad RMS
phase error against the FP64 oracle, exact integer selection and an exact dc.
"""
from __future__ import annotations

import math

import numpy as np
import pytest
import torch

from oracle import ssb_oracle as so
from quantem.gpu_b200 import SSB, B200SSBBackend, SSBProtocol
from quantem.gpu_b200.synthetic import CONFIGS, generate
from recipes import disk_input

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


def _compare(backend: B200SSBBackend, host: np.ndarray, kw: dict, ab: so.Aberrations,
             check_loss: bool = True):
    prep = so.prepare(host, **kw)
    np.testing.assert_array_equal(backend.bf_inds_row, prep.bf.rows)
    np.testing.assert_array_equal(backend.bf_inds_col, prep.bf.cols)
    if kw.get("bf_radius") is None:  # centroid of integer indices: exact
        assert backend.bf_center == prep.bf.center
    else:
        # intensity-weighted float32 centroid: the oracle sums in numpy's pairwise
        # float32 order, the reference's CuPy in its tree order, the device in FP64
        # rounded once; they agree to a few float32 ulps
        np.testing.assert_allclose(backend.bf_center, prep.bf.center, rtol=5e-7)
    # both are means of exact integer sums; only the summation order differs
    assert abs(backend.dc_value - prep.dc) <= 1e-14 * abs(prep.dc)
    g = backend.G_qk.cpu().numpy()
    assert np.abs(g - prep.g_half).max() <= 2e-6 * np.abs(prep.g_half).max()
    obj, ph = backend.object_and_phase(ab.C10, ab.C12, ab.phi12, ab.C30)
    ref_obj, ref_ph = so.reconstruct(prep, ab)
    err = so.wrapped_phase_error(ph.cpu().numpy(), ref_ph)
    rms = float(np.sqrt(np.mean(err ** 2)))
    assert rms < 1e-4, rms
    if check_loss:
        ref_loss, _ = so.phase_variance_loss(prep.g_half, prep.geo, ab, prep.dc)
        c30 = None if ab.C30 == 0.0 else [ab.C30]
        loss = float(backend.variance_loss_batch([ab.C10], [ab.C12], [ab.phi12], C30=c30)[0])
        assert loss == pytest.approx(ref_loss, rel=1e-5, abs=1e-6)
    return rms


def test_plain_32x32_det64_end_to_end():
    spec = CONFIGS["plain_32x32_det64"]
    counts = generate(spec, device="cpu").counts.numpy()
    kw = dict(voltage_kV=300, semiangle_mrad=20.0, scan_sampling=0.5, det_sampling=20.0 / 12.0)
    backend = B200SSBBackend(counts, semiangle=20.0, scan_sampling=0.5, det_sampling=20.0 / 12.0,
                             voltage_kV=300)
    assert isinstance(backend, SSBProtocol)
    assert backend.scan_shape == (128, 128)
    _compare(backend, counts, kw, so.Aberrations(50.0, 20.0, 0.3))
    backend.close()


def test_disk_case_matches_reference_golden():
    """The reference test's own end-to-end input, bf_radius=3."""
    counts = disk_input(123)
    kw = dict(voltage_kV=300, semiangle_mrad=21.4, scan_sampling=0.5, det_sampling=1.0, bf_radius=3)
    backend = B200SSBBackend(torch.as_tensor(counts, device=DEV), semiangle=21.4, scan_sampling=0.5,
                             det_sampling=1.0, voltage_kV=300, bf_radius=3,
                             aberrations={"C10": -120.0, "C12": 55.0, "phi12": math.radians(17.0)})
    _compare(backend, counts, kw, so.Aberrations(-120.0, 55.0, math.radians(17.0)))
    with np.load("tests/golden/ref_disk128_bfr3.npz") as z:
        ref_obj = z["object"].astype(np.complex128)
        ref_loss = float(z["loss"])
    res = backend.result()
    obj = res.object_wave.cpu().numpy()
    assert np.abs(obj - ref_obj).max() <= 1e-5 * np.abs(ref_obj).max()
    assert res.loss == pytest.approx(ref_loss, rel=1e-4, abs=1e-6)
    assert res.num_bf == 27


@pytest.mark.parametrize("name", ["ref_plain32_detect", "ref_disk128_detect"])
def test_detected_bf_radius_matches_reference(name):
    """det_sampling=None: the backend detects the BF radius from the mean DP
    (probe.py:12-119) and sets det_sampling = 2 alpha / r as the reference
    does (backend.py:276-285, its factor 2 included); angular sampling,
    selection, G and the reconstruction then follow the reference's golden
    outputs and the FP64 oracle."""
    from recipes import synthetic_plain_32

    with np.load(f"tests/golden/{name}.npz") as z:
        gold = {k: z[k] for k in z.files}
    counts = synthetic_plain_32() if name == "ref_plain32_detect" else disk_input(123)
    semi = float(gold["kw_semiangle"])
    bf_radius = float(gold["kw_bf_radius"]) if "kw_bf_radius" in gold else None
    backend = B200SSBBackend(torch.as_tensor(counts, device=DEV), semiangle=semi,
                             scan_sampling=0.5, det_sampling=None, voltage_kV=300,
                             bf_radius=bf_radius)
    assert backend.angular_sampling == tuple(gold["angular_sampling"])
    np.testing.assert_array_equal(backend.bf_inds_row, gold["rows"])
    np.testing.assert_array_equal(backend.bf_inds_col, gold["cols"])
    kw = dict(voltage_kV=300, semiangle_mrad=semi, scan_sampling=0.5, det_sampling=None,
              bf_radius=bf_radius)
    _compare(backend, counts, kw, so.Aberrations(*map(float, gold["aberrations"])))
    c10, c12, phi12 = map(float, gold["aberrations"])
    assert backend.variance_loss(c10, c12, phi12) == pytest.approx(float(gold["loss"]), rel=1e-4,
                                                                   abs=1e-6)
    backend.close()


def test_uneven_96_scan_is_padded_like_the_reference():
    counts = disk_input(124, scan=(96, 96))
    kw = dict(voltage_kV=300, semiangle_mrad=21.4, scan_sampling=0.5, det_sampling=1.0, bf_radius=3)
    backend = B200SSBBackend(counts, semiangle=21.4, scan_sampling=0.5, det_sampling=1.0,
                             voltage_kV=300, bf_radius=3)
    assert backend.scan_shape == (128, 128)
    _compare(backend, counts, kw, so.Aberrations(10.0, 5.0, 0.1))


@pytest.fixture(scope="module")
def production_128():
    """The 128x128 scan x 128x128 detector workload (537 MB u16), its backend
    and the FP64 oracle's preparation of the same counts, shared by the cases
    below."""
    spec = CONFIGS["plain_128x128_det128"]
    counts = generate(spec, device=DEV).counts
    host = counts.cpu().numpy()
    kw = dict(voltage_kV=300, semiangle_mrad=20.0, scan_sampling=0.5, det_sampling=20.0 / 24.0)
    backend = B200SSBBackend(counts, semiangle=20.0, scan_sampling=0.5, det_sampling=20.0 / 24.0,
                             voltage_kV=300)
    yield backend, host, kw
    backend.close()


@pytest.mark.parametrize("ab", [
    so.Aberrations(0.0, 0.0, 0.0),
    so.Aberrations(-120.0, 55.0, math.radians(17.0)),
    so.Aberrations(80.0, 30.0, 1.1, C30=3.0e4),
], ids=["aberration_free", "C10_C12", "C10_C12_C30"])
def test_production_128x128_det128_end_to_end(production_128, ab):
    """Selection, G, dc, object phase (1e-4 rad RMS) and the phase-variance
    loss (1e-5 relative) at 128^4 against the FP64 oracle, with and without
    aberrations; the C30 case takes the direct (non-factorised) overlap."""
    backend, host, kw = production_128
    assert 1700 <= backend.num_bf <= 1900
    rms = _compare(backend, host, kw, ab, check_loss=True)
    assert rms < 1e-4


def test_ssb_session_fit_recovers_defocus():
    """A short sweep + Nelder-Mead on data made with C10 = 100 A finds it.

    1e6 e per position: at 1000 e on a 32x32 scan the phase-variance
    objective is noise-dominated and its global minimum is the degenerate
    C10 ~ 0 (Gamma vanishes where both q-k and q+k are inside the aperture)."""
    spec = CONFIGS["plain_32x32_det64"]
    from dataclasses import replace

    counts = generate(replace(spec, C10=100.0, dose=1e6, seed=3), device="cpu").counts.numpy()
    with SSB.from_array(counts, voltage_kV=300, semiangle_mrad=20.0, scan_sampling_A=0.5,
                        det_sampling=20.0 / 12.0) as ssb:
        res = ssb.fit(trials=64, search_ranges={"C10_nm": (-200.0, 200.0), "C12_nm": 0.0,
                                                "phi12_deg": 0.0}, verbose=False)
    assert abs(res.aberrations["C10"] - 100.0) < 15.0
    assert res.refine_method == "nelder-mead"
    assert res.loss is not None


@pytest.mark.parametrize("dose", [50.0, 1000.0, 20000.0])
def test_stress_256_matches_fp64_gpu_path(dose):
    """256^2 scan x 128^2 detector (2.1 GB u16), defocus 20 nm: the float32
    kernels (Kahan trotter sum) against the FP64 GPU restatement of the oracle,
    target 1e-4 rad RMS."""
    from dataclasses import replace

    from oracle import ssb_torch_fp64 as tf

    spec = replace(CONFIGS["stress_256x256_det128"], dose=dose)
    counts = generate(spec, DEV).counts
    kw = dict(voltage_kV=spec.voltage_kV, semiangle_mrad=spec.semiangle_mrad,
              scan_sampling=spec.scan_step_A, det_sampling=spec.det_sampling_mrad)
    backend = B200SSBBackend(counts, semiangle=spec.semiangle_mrad, scan_sampling=spec.scan_step_A,
                             det_sampling=spec.det_sampling_mrad, voltage_kV=spec.voltage_kV,
                             device=DEV)
    assert backend.G_qk.shape[1:] == (256, 129)
    _, ph = backend.object_and_phase(spec.C10, 0.0, 0.0)
    prep = tf.prepare(counts, **kw)
    np.testing.assert_array_equal(backend.bf_inds_row, prep.bf.rows)
    _, ref = tf.reconstruct(prep, so.Aberrations(spec.C10, 0.0, 0.0))
    err = so.wrapped_phase_error(ph.cpu().numpy(), ref.cpu().numpy())
    rms = float(np.sqrt(np.mean(err ** 2)))
    assert rms <= 1e-4, rms
    # phase-variance loss at 256^2 (the staged-rows kernel), quadratic and C30 paths
    c10 = np.asarray([spec.C10, spec.C10 - 40.0, spec.C10 + 25.0])
    losses = backend.variance_loss_batch(c10, 0.0, 0.0).cpu().numpy()
    for c, got in zip(c10, losses):
        want, _ = tf.phase_variance_loss(prep, so.Aberrations(float(c), 0.0, 0.0))
        assert abs(got - want) <= 1e-5 * abs(want) + 1e-6, (c, got, want)
    got = backend.variance_loss_batch([spec.C10], [5.0], [0.3], C30=[2e4]).cpu().numpy()[0]
    want, _ = tf.phase_variance_loss(prep, so.Aberrations(spec.C10, 5.0, 0.3, C30=2e4))
    assert abs(got - want) <= 1e-5 * abs(want) + 1e-6, (got, want)
