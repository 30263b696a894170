"""FP64 restatement of the reference's temporal joining (TEST INFRASTRUCTURE).

Follows ssb/temporal.py of bobleesj/quantem.gpu: ``fourier_shift_2d``
(:77-107), the global-phase alignment to frame 0 (:154-180) and the weighted
complex mean of ``join_object_waves`` (:183-257), in numpy complex128.
"""
from __future__ import annotations

import numpy as np


def fourier_shift_2d(image: np.ndarray, shift) -> np.ndarray:
    """ifft2(fft2(image) exp(-2 pi i (f_r s_r + f_c s_c))), f = fftfreq(n, 1)."""
    arr = np.asarray(image)
    n_row, n_col = arr.shape
    fr = np.fft.fftfreq(n_row, d=1.0).reshape(-1, 1)
    fc = np.fft.fftfreq(n_col, d=1.0).reshape(1, -1)
    phase = np.exp(-2j * np.pi * (fr * float(shift[0]) + fc * float(shift[1])))
    return np.fft.ifft2(np.fft.fft2(arr.astype(np.complex128)) * phase)


def join_object_waves(stack: np.ndarray, shifts=None, weights=None, phase_reference: str = "first"):
    """(joined, aligned stack) in complex128."""
    stack = np.asarray(stack, dtype=np.complex128)
    n = stack.shape[0]
    shifts = np.zeros((n, 2)) if shifts is None else np.asarray(shifts, dtype=np.float64)
    w = np.full(n, 1.0 / n) if weights is None else np.asarray(weights, dtype=np.float64)
    w = w / w.sum()
    aligned = np.empty_like(stack)
    for i in range(n):
        shifted = fourier_shift_2d(stack[i], shifts[i])
        if i > 0 and phase_reference == "first":
            overlap = np.sum(shifted * np.conj(aligned[0]))
            shifted = shifted * np.exp(-1j * np.angle(overlap))
        aligned[i] = shifted
    return np.tensordot(w, aligned, axes=(0, 0)), aligned
