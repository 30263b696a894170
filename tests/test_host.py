"""Host-side tests that need no GPU: the C ABI library, calibration logic,
optimizer, contract types and the synthetic generator."""
from __future__ import annotations

import ctypes
import math
import re
import sys
from pathlib import Path

import numpy as np
import pytest

from oracle import ssb_oracle as so
from quantem.gpu_b200 import _lib
from quantem.gpu_b200.backend import B200SSBBackend
from quantem.gpu_b200.calibration import bf_geometry, detect_bf_radius, pad_target, select_bf
from quantem.gpu_b200.optimizer import batch_nelder_mead, batch_sweep, halton, search_box
from quantem.gpu_b200.protocol import BrightfieldDisk, SSBProtocol, SSBResult
from quantem.gpu_b200.workflow import SSB, _validate_aberrations

REPO = Path(__file__).resolve().parent.parent
GOLDEN = REPO / "tests" / "golden"


# ------------------------------------------------------------------ C ABI
def _declared_symbols() -> list[str]:
    text = (REPO / "include" / "qssb.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:int|int64_t|const char\*)\s+(qssb_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    declared = _declared_symbols()
    assert len(declared) >= 9
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(_lib.SIGNATURES), "ctypes signatures out of sync with qssb.h"


def test_version_and_error_reporting_without_gpu():
    lib = _lib.load()
    assert lib.qssb_version() == 1
    size = ctypes.c_size_t(0)
    rc = lib.qssb_object_workspace_bytes(None, 0, ctypes.byref(size))
    assert rc == _lib.QSSB_ERR_INVALID
    assert lib.qssb_last_error()
    cal = _lib.Calibration(n_bf=1810, scan_rows=96, scan_cols=96, reserved=0, wavelength_A=0.0197,
                           semiangle_rad=0.02, det_sampling_row_rad=1e-3,
                           det_sampling_col_rad=1e-3, scan_sampling_row_A=0.5,
                           scan_sampling_col_A=0.5, dc_re=1.0, dc_im=0.0)
    assert lib.qssb_object_workspace_bytes(ctypes.byref(cal), 0, ctypes.byref(size)) == _lib.QSSB_ERR_UNSUPPORTED
    cal.scan_rows = cal.scan_cols = 128
    assert lib.qssb_object_workspace_bytes(ctypes.byref(cal), 0, ctypes.byref(size)) == 0
    assert size.value > 128 * 128 * 8
    assert lib.qssb_loss_workspace_bytes(ctypes.byref(cal), 64, 0, ctypes.byref(size)) == 0
    assert lib.qssb_loss_workspace_bytes(ctypes.byref(cal), 0, 0, ctypes.byref(size)) == _lib.QSSB_ERR_INVALID
    # null device pointers are rejected before any launch
    assert lib.qssb_mean_dp_u64(None, 10, 10, None, None, None) == _lib.QSSB_ERR_INVALID
    assert lib.qssb_gather_bf_columns(None, 1, 1, None, 1, None, None) == _lib.QSSB_ERR_INVALID
    assert lib.qssb_scan_fft_half(None, 1, 128, 128, None, None) == _lib.QSSB_ERR_INVALID
    assert lib.qssb_select_bf(None, 128, 128, 10, 0.0, 0.0, None, None, None, None) == _lib.QSSB_ERR_INVALID
    gp = _lib.GeometryParams(1.0, 1.0, 1.0, 0.0, 0.0197, 0.02, 1e-3, 1e-3)
    assert lib.qssb_bf_geometry(None, None, 128, 128, 10, ctypes.byref(gp), None, None) == _lib.QSSB_ERR_INVALID


def test_check_raises_with_message():
    with pytest.raises(_lib.QssbError) as exc:
        _lib.load().qssb_mean_dp_u64(None, 1, 1, None, None, None)
        _lib.check(_lib.QSSB_ERR_INVALID)
    assert exc.value.code == _lib.QSSB_ERR_INVALID


# ------------------------------------------------------------ calibration
@pytest.mark.parametrize("name", ["ref_disk128_bfr3", "ref_disk96_padded", "ref_plain32_auto"])
def test_selection_and_geometry_match_reference(name):
    from recipes import disk_input, synthetic_plain_32

    data = {"ref_disk128_bfr3": lambda: disk_input(123),
            "ref_disk96_padded": lambda: disk_input(124, scan=(96, 96)),
            "ref_plain32_auto": synthetic_plain_32}[name]()
    with np.load(GOLDEN / f"{name}.npz") as z:
        gold = {k: z[k] for k in z.files}
    data = so.pad_or_crop_scan(data)
    _, mean_dp = so.mean_dp_u64(data)
    bf_radius = float(gold["kw_bf_radius"]) if "kw_bf_radius" in gold else None
    sel = select_bf(mean_dp, 0.0, bf_radius)
    np.testing.assert_array_equal(sel.rows, gold["rows"])
    np.testing.assert_array_equal(sel.cols, gold["cols"])
    assert sel.center == tuple(gold["center"])
    det = float(gold["kw_det_sampling"])
    geo = bf_geometry(sel.rows, sel.cols, sel.center, data.shape[2:], tuple(gold["sampling"]),
                      float(gold["wavelength"]), float(gold["kw_semiangle"]), (det, det), 0.0)
    # float32 arithmetic mirroring the reference's CuPy cache: equal to rounding
    np.testing.assert_allclose(geo.kx_bf, gold["kx_bf"], rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(geo.ky_bf, gold["ky_bf"], rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(geo.alpha_k2, gold["alpha_k2"], rtol=1e-5, atol=1e-12)
    np.testing.assert_allclose(geo.aperture_k, gold["aperture_k"], atol=1e-6)
    np.testing.assert_allclose(geo.cos2phi_k, gold["cos2phi_k"], atol=1e-6)
    np.testing.assert_allclose(geo.sin2phi_k, gold["sin2phi_k"], atol=1e-6)


def test_pad_target_rule():
    assert pad_target(128, 128) is None
    assert pad_target(96, 96) == (128, 128)
    assert pad_target(160, 120) == (256, 256)
    assert pad_target(32, 32) == (128, 128)
    assert pad_target(2000, 5) == (1024, 1024)


def test_selection_errors():
    with pytest.raises(ValueError, match="No bright-field pixels found"):
        select_bf(np.zeros((8, 8), np.float32), threshold=0.5)
    dp = np.zeros((16, 16), np.float32)
    dp[0, 0] = dp[0, 2] = 1.0  # weighted centre (0, 1): no pixel within 0.1 px
    with pytest.raises(ValueError, match="within bf_radius"):
        select_bf(dp, threshold=0.5, bf_radius=0.1)


def test_detect_bf_radius_on_disk():
    yy, xx = np.mgrid[:64, :64]
    dp = ((yy - 32) ** 2 + (xx - 31) ** 2 <= 12 ** 2).astype(np.float32) * 100 + 1
    (r0, c0), r = detect_bf_radius(dp)
    assert (r0, c0) == (32, 31)
    assert abs(r - 12) <= 2


# -------------------------------------------------------------- optimizer
def test_nelder_mead_converges_on_quadratic():
    target = np.array([100.0, 20.0, 0.4])

    def f(x):
        x = np.atleast_2d(x)
        return ((x - target) ** 2 * np.array([1.0, 2.0, 50.0])).sum(axis=1)

    x, fx, n = batch_nelder_mead(f, np.array([50.0, 10.0, 0.1]), xatol=1e-3, fatol=1e-10)
    np.testing.assert_allclose(x, target, atol=1e-2)
    assert n < 400


def test_nelder_mead_keeps_first_vertex_for_tied_losses():
    """Stable tie ordering (tests/test_ssb_batch_optuna.py:39-69 pattern)."""
    x0 = np.asarray([-20.0, 22.0, 0.46])
    flat = lambda x: np.ones(len(np.atleast_2d(x)))  # noqa: E731
    first = batch_nelder_mead(flat, x0, max_iter=4)
    second = batch_nelder_mead(flat, x0, max_iter=4)
    np.testing.assert_array_equal(first[0], x0)
    np.testing.assert_array_equal(second[0], first[0])
    assert first[1:] == second[1:]


def test_sweep_is_seeded_and_takes_minimum():
    lo, hi = np.array([-400.0, 0.0, -1.5]), np.array([400.0, 100.0, 1.5])
    f = lambda x: np.abs(np.atleast_2d(x)[:, 0] - 123.0)  # noqa: E731
    a = batch_sweep(f, lo, hi, 200, seed=42)
    b = batch_sweep(f, lo, hi, 200, seed=42)
    np.testing.assert_array_equal(a[2], b[2])
    assert a[1] == a[3].min()
    assert halton(5, 3, 0).shape == (5, 3)
    keys, lo2, hi2 = search_box({"C10_nm": (-10, 10), "C12_nm": 3.0}, {"C10": 0, "C12": 0, "phi12": 0.5})
    assert keys == ["C10", "C12", "phi12"]
    np.testing.assert_allclose(lo2, [-10, 3.0, 0.5])
    np.testing.assert_allclose(hi2, [10, 3.0, 0.5])


# --------------------------------------------------------------- contract
def test_backend_class_has_every_protocol_member():
    members = [m for m in dir(SSBProtocol) if not m.startswith("_")]
    for m in ("fit", "reconstruct_result", "cache_rotation", "preview", "preview_context",
              "browser_state", "export_brightfield", "close", "scan_shape", "detector_shape",
              "num_bf", "backend", "precision"):
        assert m in members or m in ("backend", "precision")
        assert hasattr(B200SSBBackend, m), m
    assert B200SSBBackend.backend == "cuda"
    assert B200SSBBackend.precision.real_dtype == "float32"
    assert B200SSBBackend.precision.complex_dtype == "complex64"


def test_reference_protocol_members_match_when_reference_is_present():
    from oracle.ref_cuda.build_ref import reference_root

    ref = reference_root() / "src"
    if not ref.exists():
        pytest.skip("reference checkout not present")
    sys.path.insert(0, str(ref))
    try:
        from quantem.gpu.ssb.compute.protocol import SSBProtocol as RefProtocol
        from quantem.gpu.ssb.results import SSBResult as RefResult
    finally:
        sys.path.remove(str(ref))
    ref_members = {m for m in dir(RefProtocol) if not m.startswith("_")}
    for m in ref_members:
        assert hasattr(B200SSBBackend, m), m
    import dataclasses

    assert [f.name for f in dataclasses.fields(RefResult)] == [f.name for f in dataclasses.fields(SSBResult)]


def test_brightfield_disk_validation():
    disk = BrightfieldDisk(rows=[1, 2], cols=[3, 4], center_row_col=(1.5, 3.5), radius_px=2.0,
                           detected_radius_px=2.0, detector_shape=(8, 8))
    assert disk.size == 2
    assert not disk.rows.flags.writeable
    with pytest.raises(ValueError, match="duplicates"):
        BrightfieldDisk(rows=[1, 1], cols=[3, 3], center_row_col=(1, 3), radius_px=1,
                        detected_radius_px=1, detector_shape=(8, 8))
    with pytest.raises(ValueError, match="outside"):
        BrightfieldDisk(rows=[9], cols=[3], center_row_col=(1, 3), radius_px=1,
                        detected_radius_px=1, detector_shape=(8, 8))


def test_workflow_validation_without_gpu():
    assert _validate_aberrations(None) == {"C10": 0.0, "C12": 0.0, "phi12": 0.0}
    with pytest.raises(ValueError, match="missing"):
        _validate_aberrations({"C10": 1.0})
    with pytest.raises(ValueError, match="unknown"):
        _validate_aberrations({"C10": 1.0, "C12": 0.0, "phi12": 0.0, "C30": 1.0})
    with pytest.raises(RuntimeError):
        SSB(np.zeros((4, 4, 2, 2), np.uint16), backend="mps", voltage_kV=300, semiangle_mrad=20,
            scan_sampling_A=0.5)
    with pytest.raises(ValueError):
        SSB(np.zeros((4, 4, 2, 2), np.uint16), backend="tpu", voltage_kV=300, semiangle_mrad=20,
            scan_sampling_A=0.5)
    ssb = SSB(np.zeros((4, 4, 2, 2), np.uint16), voltage_kV=300, semiangle_mrad=20, scan_sampling_A=0.5)
    with pytest.raises(ValueError, match="trials"):
        ssb.fit(trials=-1)
    with pytest.raises(NotImplementedError):
        SSB.open("x.h5")


def test_result_phase_from_numpy_object():
    obj = np.exp(1j * np.linspace(-1, 1, 16)).reshape(4, 4).astype(np.complex64)
    res = SSBResult(object_wave=obj, backend="cuda")
    np.testing.assert_allclose(res.phase, np.angle(obj))
    assert "SSB Result" in repr(res)


# -------------------------------------------------------------- generator
def test_synthetic_generator_dose_and_bf_radius():
    from quantem.gpu_b200.synthetic import CONFIGS, generate

    spec = CONFIGS["plain_32x32_det64"]
    data = generate(spec, device="cpu")
    counts = data.counts.numpy()
    assert counts.dtype == np.uint16 and counts.shape == (32, 32, 64, 64)
    per_position = counts.reshape(1024, -1).sum(axis=1)
    assert abs(per_position.mean() - spec.dose) < 0.05 * spec.dose
    _, mean_dp = so.mean_dp_u64(counts)
    sel = select_bf(mean_dp)
    assert abs(sel.radius - 12.0) < 1.0
    again = generate(spec, device="cpu").counts.numpy()
    np.testing.assert_array_equal(counts, again)


def test_persistent_loss_plan_without_gpu():
    """The workspace query is host arithmetic: at 256^2 (float32 chi)
    QSSB_FLAG_PERSISTENT adds two more staging slots (three in all) and the
    queue words (ticket, abort word, two counts per BF chunk); elsewhere the
    flag changes nothing. The sizes follow the plan: 27-candidate groups
    (444 column CTA slots / 16 strips), 4 BF pixels per chunk in the 32 MB
    staging budget, 10 for the last group of 10 candidates."""
    cal = _lib.Calibration(n_bf=1783, scan_rows=256, scan_cols=256, reserved=0,
                           wavelength_A=0.0197, semiangle_rad=0.02, det_sampling_row_rad=1e-3,
                           det_sampling_col_rad=1e-3, scan_sampling_row_A=0.5,
                           scan_sampling_col_A=0.5, dc_re=1.0, dc_im=0.0)
    q, per, f64 = _lib.QSSB_FLAG_QUADRATIC, _lib.QSSB_FLAG_PERSISTENT, _lib.QSSB_FLAG_CHI_FP64
    from quantem.gpu_b200 import ops
    seq = ops.loss_workspace_bytes(cal, 64, q)
    pst = ops.loss_workspace_bytes(cal, 64, q | per)
    slot = 8 * 129 * 256 * 4 * 27          # staged half rows of a chunk
    dslot = 8 * 128 * 4 * 27               # its Nyquist-column deviations
    chunks = 2 * -(-1783 // 4) + -(-1783 // 10)
    words = (4 * (2 + 2 * chunks) + 255) // 256 * 256
    assert chunks == 1071
    assert pst - seq == 2 * slot + 2 * dslot + words
    assert ops.loss_workspace_bytes(cal, 64, q | per | f64) == ops.loss_workspace_bytes(cal, 64, q | f64)
    for n in (128, 512):
        cal.scan_rows = cal.scan_cols = n
        assert ops.loss_workspace_bytes(cal, 64, q | per) == ops.loss_workspace_bytes(cal, 64, q)
