"""B200-native single-sideband (SSB) ptychography engine.

A drop-in for the SSB path of bobleesj/quantem.gpu: the ``SSB`` session and
the ``SSBProtocol`` backend contract, computed by hand-written sm_100a CUDA
kernels in ``libqssb.so`` (C ABI: ``include/qssb.h``). Importing the package
does not load the library; the first device call does, and fails loudly if
it is missing.
"""
from __future__ import annotations

from .protocol import BrightfieldDisk, SSBExportState, SSBPrecision, SSBProtocol, SSBResult

__all__ = [
    "SSB",
    "B200SSBBackend",
    "BrightfieldDisk",
    "SSBExportState",
    "SSBPrecision",
    "SSBProtocol",
    "SSBResult",
]


def __getattr__(name: str):
    if name == "SSB":
        from .workflow import SSB

        return SSB
    if name == "B200SSBBackend":
        from .backend import B200SSBBackend

        return B200SSBBackend
    raise AttributeError(name)
