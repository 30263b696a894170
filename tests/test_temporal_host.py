"""The temporal oracle on the CPU: integer Fourier shifts are rolls, shifts
compose and invert, and phase referencing removes a global phase offset."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import temporal_oracle as to


def _wave(rng, shape=(32, 48)):
    amp = 1.0 + 0.05 * rng.standard_normal(shape)
    return amp * np.exp(1j * 0.2 * rng.standard_normal(shape))


def test_integer_shift_is_a_roll():
    rng = np.random.default_rng(0)
    w = _wave(rng)
    np.testing.assert_allclose(to.fourier_shift_2d(w, (3, -5)), np.roll(w, (3, -5), axis=(0, 1)),
                               atol=1e-12)


def test_shifts_compose_and_invert():
    rng = np.random.default_rng(1)
    w = _wave(rng)
    a = to.fourier_shift_2d(to.fourier_shift_2d(w, (1.25, -0.5)), (0.5, 2.0))
    np.testing.assert_allclose(a, to.fourier_shift_2d(w, (1.75, 1.5)), atol=1e-12)
    np.testing.assert_allclose(to.fourier_shift_2d(to.fourier_shift_2d(w, (2.3, -1.7)), (-2.3, 1.7)),
                               w, atol=1e-12)


def test_phase_reference_removes_global_offset():
    rng = np.random.default_rng(2)
    w = _wave(rng)
    stack = np.stack([w, w * np.exp(0.7j)])
    joined, aligned = to.join_object_waves(stack, phase_reference="first")
    np.testing.assert_allclose(joined, w, atol=1e-12)
    literal, _ = to.join_object_waves(stack, phase_reference="none")
    assert np.abs(literal - w).mean() > 0.1


def test_weights_are_normalised():
    rng = np.random.default_rng(3)
    a, b = _wave(rng), _wave(rng)
    joined, _ = to.join_object_waves(np.stack([a, b]), weights=[3.0, 1.0], phase_reference="none")
    np.testing.assert_allclose(joined, 0.75 * a + 0.25 * b, atol=1e-12)
