"""ctypes binding of ``libqssb.so`` (the C ABI declared in ``include/qssb.h``).

The shared library is built in-tree by ``quantem.gpu_b200.build`` (nvcc,
sm_100a). There is no fallback: if the library is missing or a symbol is
absent, loading raises, and every entry point's nonzero status becomes a
Python exception carrying ``qssb_last_error()``.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libqssb.so"

QSSB_OK = 0
QSSB_ERR_INVALID = -1
QSSB_ERR_CUDA = -2
QSSB_ERR_UNSUPPORTED = -3
QSSB_ERR_WORKSPACE = -4
QSSB_FLAG_CHI_FP64 = 1
QSSB_FLAG_FULL_PLANE = 2
QSSB_FLAG_QUADRATIC = 4
QSSB_FLAG_PERSISTENT = 8
QSSB_NOALLOC_SCRATCH_BYTES = 16 << 20
QSSB_FLAG_CHUNKS_SHIFT = 16
QSSB_FLAG_CHUNKS_MAX = 32767
QSSB_FLAG_VARIANT_SHIFT = 8
QSSB_FLAG_VARIANT_MAX = 15
GATHER_VARIANTS = 6  # qssb_gather_bf_columns_2d_ex: 1..6 (0 = built-in rule)
OBJECT_VARIANTS = 3  # QSSB_FLAG_VARIANT on qssb_object: 1..3 (0 = built-in)


def flag_chunks(n: int) -> int:
    """``QSSB_FLAG_CHUNKS(n)``: the work partition knob (0 = built-in plan)."""
    if not 0 <= int(n) <= QSSB_FLAG_CHUNKS_MAX:
        raise ValueError(f"chunk count must be in [0, {QSSB_FLAG_CHUNKS_MAX}]")
    return int(n) << QSSB_FLAG_CHUNKS_SHIFT


def flag_variant(v: int) -> int:
    """``QSSB_FLAG_VARIANT(v)``: the tile-shape knob (0 = built-in shape)."""
    if not 0 <= int(v) <= QSSB_FLAG_VARIANT_MAX:
        raise ValueError(f"variant must be in [0, {QSSB_FLAG_VARIANT_MAX}]")
    return int(v) << QSSB_FLAG_VARIANT_SHIFT


class Calibration(ctypes.Structure):
    """``qssb_calibration_t``."""

    _fields_ = [
        ("n_bf", ctypes.c_int32),
        ("scan_rows", ctypes.c_int32),
        ("scan_cols", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("wavelength_A", ctypes.c_double),
        ("semiangle_rad", ctypes.c_double),
        ("det_sampling_row_rad", ctypes.c_double),
        ("det_sampling_col_rad", ctypes.c_double),
        ("scan_sampling_row_A", ctypes.c_double),
        ("scan_sampling_col_A", ctypes.c_double),
        ("dc_re", ctypes.c_double),
        ("dc_im", ctypes.c_double),
    ]


GEOM_ROWS = 8
FULL_TERMS = 14  # QSSB_FULL_TERMS
# slot order of qssb_full_aberrations_t (aberration.py:63 of the reference)
FULL_TERM_NAMES = ("C10", "C12", "C21", "C23", "C30", "C32", "C34", "C41", "C43", "C45", "C50",
                   "C52", "C54", "C56")


class Aberrations(ctypes.Structure):
    """``qssb_aberrations_t`` (reference numeric convention: Angstrom, rad)."""

    _fields_ = [
        ("C10", ctypes.c_float),
        ("C12", ctypes.c_float),
        ("phi12", ctypes.c_float),
        ("C30", ctypes.c_float),
    ]


class BFInfo(ctypes.Structure):
    """``qssb_bf_info_t`` (written on the device by ``qssb_select_bf``)."""

    _fields_ = [
        ("n_bf", ctypes.c_int32),
        ("n_mask", ctypes.c_int32),
        ("center_row", ctypes.c_double),
        ("center_col", ctypes.c_double),
        ("radius", ctypes.c_double),
        ("dc_re", ctypes.c_double),
        ("dc_im", ctypes.c_double),
    ]


class GeometryParams(ctypes.Structure):
    """``qssb_geometry_params_t``."""

    _fields_ = [
        ("k_step_row_inv_A", ctypes.c_double),
        ("k_step_col_inv_A", ctypes.c_double),
        ("rot_cos", ctypes.c_double),
        ("rot_sin", ctypes.c_double),
        ("wavelength_A", ctypes.c_double),
        ("semiangle_rad", ctypes.c_double),
        ("det_sampling_row_rad", ctypes.c_double),
        ("det_sampling_col_rad", ctypes.c_double),
    ]


_P = ctypes.c_void_p
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
_SZ = ctypes.c_size_t

# name -> (restype, argtypes); must match include/qssb.h exactly.
SIGNATURES = {
    "qssb_version": (ctypes.c_int, []),
    "qssb_last_error": (ctypes.c_char_p, []),
    "qssb_mean_dp_u64": (ctypes.c_int, [_P, _I64, _I32, _P, _P, _P]),
    "qssb_gather_bf_columns": (ctypes.c_int, [_P, _I64, _I32, _P, _I32, _P, _P]),
    "qssb_gather_bf_columns_2d": (ctypes.c_int, [_P, _I64, _I32, _I32, _P, _I32, _P, _P]),
    "qssb_gather_bf_columns_2d_ex": (ctypes.c_int, [_P, _I64, _I32, _I32, _P, _I32, _P, _I32, _P]),
    "qssb_select_bf": (ctypes.c_int, [_P, _I32, _I32, _I64, ctypes.c_float, ctypes.c_float,
                                      _P, _P, _P, _P]),
    "qssb_bf_geometry": (ctypes.c_int, [_P, _P, _I32, _I32, _I32, ctypes.POINTER(GeometryParams),
                                        _P, _P]),
    "qssb_scan_fft_half": (ctypes.c_int, [_P, _I32, _I32, _I32, _P, _P]),
    "qssb_scan_fft_half_ex": (ctypes.c_int, [_P, _I32, _I32, _I32, _P, _I32, _P]),
    "qssb_scan_fft_variants": (ctypes.c_int, [_I32, _P]),
    "qssb_count_max": (ctypes.c_int, [_P, _I32, _I64, _P, _P]),
    "qssb_bf_box_estimate": (ctypes.c_int, [_P, _I32, _I32, ctypes.c_float, _I32, _I64, _P, _P]),
    "qssb_mean_dp_u64_box": (ctypes.c_int, [_P, _I64, _I32, _I32, _P, _P, _I64, _P, _P]),
    "qssb_bf_box_map": (ctypes.c_int, [_P, _P, _I32, _I32, _I32, _I64, _P, _P, _P, _P]),
    "qssb_scan_fft_half_mapped": (ctypes.c_int, [_P, _I64, _P, _I32, _I32, _I32, _P, _P]),
    "qssb_export_bf_columns": (ctypes.c_int, [_P, _I32, _I64, _I64, _P, _I32, _P, _I32, _P]),
    "qssb_object_workspace_bytes": (
        ctypes.c_int, [ctypes.POINTER(Calibration), _I32, ctypes.POINTER(_SZ)]),
    "qssb_object": (ctypes.c_int, [
        _P, _P, _P, _P, ctypes.POINTER(Calibration), ctypes.POINTER(Aberrations), _I32, _P, _SZ,
        _P, _P, _P]),
    "qssb_object_ex": (ctypes.c_int, [
        _P, _P, _P, _P, ctypes.POINTER(Calibration), ctypes.POINTER(Aberrations), _I32, _P, _P, _SZ,
        _P, _P, _P]),
    "qssb_object_noalloc": (ctypes.c_int, [
        _P, _P, _P, _P, ctypes.POINTER(Calibration), ctypes.POINTER(Aberrations), _I32, _P, _P, _P]),
    "qssb_loss_workspace_bytes": (
        ctypes.c_int, [ctypes.POINTER(Calibration), _I32, _I32, ctypes.POINTER(_SZ)]),
    "qssb_trotter_features": (ctypes.c_int, [_P, _I32, _I32, _P, _I32, _P, _P, _P, _I32, _P, _P,
                                             _P, _P]),
    "qssb_synth_features": (ctypes.c_int, [_P, _I32, _P, _I32, _P, _P, _P, _I32,
                                           ctypes.POINTER(Calibration), ctypes.c_uint64, _P, _P,
                                           _P, _I32, _P, _P, _P, _P]),
    "qssb_gemm_bf16": (ctypes.c_int, [_P, _I32, _I32, _P, _I32, _I32, _I32, _I32, _I32, _P, _I32,
                                      _P, _I32, _P, _I32, _P]),
    "qssb_gelu_backward": (ctypes.c_int, [_P, _P, _I64, _P, _P, _P]),
    "qssb_bias_grad": (ctypes.c_int, [_P, _I32, _I32, _P, _P]),
    "qssb_kernel_launches": (ctypes.c_int64, []),
    "qssb_mse": (ctypes.c_int, [_P, _P, _I32, _I32, _I32, _P, _P, _P]),
    "qssb_mse_heads": (ctypes.c_int, [_P, _P, _I32, _I32, _I32, _I32, _P, _I32, ctypes.c_float,
                                      _P, _P, _P, _P]),
    "qssb_adam": (ctypes.c_int, [_P, _P, _P, _P, _I64, ctypes.c_float, ctypes.c_float,
                                 ctypes.c_float, ctypes.c_float, ctypes.c_float, _I32, _P, _P]),
    "qssb_adam_schedule": (ctypes.c_int, [_P, _P, _I32, _I32, ctypes.c_float, ctypes.c_float,
                                          ctypes.c_float, _P]),
    "qssb_adam_dev": (ctypes.c_int, [_P, _P, _P, _P, _I64, _P, ctypes.c_float, ctypes.c_float,
                                     ctypes.c_float, ctypes.c_float, _P, _P]),
    "qssb_to_bf16": (ctypes.c_int, [_P, _I64, _P, _P]),
    "qssb_loss_batch": (ctypes.c_int, [
        _P, _P, _P, _P, ctypes.POINTER(Calibration), _P, _I32, _I32, _P, _SZ, _P, _P, _P]),
    "qssb_loss_batch_ex": (ctypes.c_int, [
        _P, _P, _P, _P, ctypes.POINTER(Calibration), _P, _I32, _I32, _P, _P, _SZ, _P, _P, _P]),
    "qssb_set_cancel": (ctypes.c_int, [_P]),
    "qssb_gemm_tc_workspace_bytes": (ctypes.c_int, [_I32, _I32, _I32, _I32, ctypes.POINTER(_SZ)]),
    "qssb_gemm_bf16_tc": (ctypes.c_int, [_P, _I32, _I32, _P, _I32, _I32, _I32, _I32, _I32, _I32, _P,
                                         _I32, _P, _I32, _P, _I32, _P, _SZ, _P]),
    "qssb_overlap_table_bytes": (ctypes.c_int, [ctypes.POINTER(Calibration), ctypes.POINTER(_SZ)]),
    "qssb_overlap_table": (ctypes.c_int, [_P, _P, _P, ctypes.POINTER(Calibration), _P, _P]),
    "qssb_decode_bslz4_u16": (ctypes.c_int, [_P, ctypes.c_int64, _P, _I32, ctypes.c_int64, _P, _P,
                                             _P]),
    "qssb_encode_bslz4_scratch_bytes": (ctypes.c_int, [_I32, ctypes.c_int64, ctypes.POINTER(_SZ)]),
    "qssb_encode_bslz4_u16": (ctypes.c_int, [_P, _I32, ctypes.c_int64, _P, _P, _P]),
    "qssb_pack_bslz4": (ctypes.c_int, [_P, _P, _I32, ctypes.c_int64, _P, _P, _P]),
    "qssb_fourier_shift": (ctypes.c_int, [_P, _P, _I32, _I32, _I32, _P, _P]),
    "qssb_join_workspace_bytes": (ctypes.c_int, [_I32, ctypes.POINTER(_SZ)]),
    "qssb_join_object_waves": (ctypes.c_int, [_P, _P, _I32, ctypes.c_int64, _I32, _P, _SZ, _P,
                                              _I32, _P]),
    "qssb_loss_full_workspace_bytes": (
        ctypes.c_int, [ctypes.POINTER(Calibration), _I32, _I32, ctypes.POINTER(_SZ)]),
    "qssb_loss_batch_full": (ctypes.c_int, [
        _P, _P, _P, _P, ctypes.POINTER(Calibration), _P, _I32, _I32, _P, _SZ, _P, _P, _P]),
    "qssb_phase_atan2": (ctypes.c_int, [_P, _P, _P, ctypes.c_int64, _P]),
}

_lib = None


class QssbError(RuntimeError):
    """A nonzero status from the native library."""

    def __init__(self, code: int, message: str):
        super().__init__(f"qssb error {code}: {message}")
        self.code = code


def load() -> ctypes.CDLL:
    """Load ``libqssb.so`` once; raise if it is missing (no CPU fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    path = Path(os.environ.get("QSSB_LIBRARY", LIB_PATH))
    if not path.exists():
        raise ImportError(
            f"{path} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
            "or `python -m quantem.gpu_b200.build`. The SSB engine has no CPU fallback."
        )
    lib = ctypes.CDLL(str(path))
    for name, (restype, argtypes) in SIGNATURES.items():
        fn = getattr(lib, name)  # AttributeError if a symbol is absent
        fn.restype = restype
        fn.argtypes = argtypes
    _lib = lib
    return lib


def check(code: int) -> None:
    """Raise :class:`QssbError` for a nonzero status."""
    if code != QSSB_OK:
        msg = load().qssb_last_error()
        raise QssbError(code, msg.decode() if msg else "")
