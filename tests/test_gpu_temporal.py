"""Temporal joining on the GPU (qssb_fourier_shift, qssb_join_object_waves):
the reference's own temporal tests (tests/test_ssb_temporal.py of
bobleesj/quantem.gpu) restated on torch tensors, parity with the FP64 oracle
over sizes, shifts, weights and both phase references, and a time series
through real SSB sessions."""
from __future__ import annotations

import math
from types import SimpleNamespace

import numpy as np
import pytest
import torch

from oracle import temporal_oracle as to
from quantem.gpu_b200 import SSB
from quantem.gpu_b200.synthetic import CONFIGS, generate
from quantem.gpu_b200.temporal import (fourier_shift_2d, join_object_waves, ssb_time_average,
                                       ssb_time_series)

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


def _object_wave(shape=(64, 64), seed=123):
    g = torch.Generator(device=DEV).manual_seed(seed)
    amp = 1.0 + 0.05 * torch.randn(shape, generator=g, device=DEV)
    phase = 0.2 * torch.randn(shape, generator=g, device=DEV)
    return torch.polar(amp, phase).to(torch.complex64)


def test_join_undoes_known_fourier_shift():
    base = _object_wave()
    shift = (2.25, -1.5)
    shifted = fourier_shift_2d(base, shift)
    result = join_object_waves(torch.stack([base, shifted]),
                               shifts=[(0.0, 0.0), (-shift[0], -shift[1])], phase_reference="none")
    assert float((result.object_wave - base).abs().max()) < 2e-5
    assert result.join_mode == "drift_corrected_complex_mean"
    assert result.num_frames == 2


def test_join_aligns_global_phase_offsets():
    base = _object_wave()
    offset = complex(math.cos(0.7), math.sin(0.7))
    stack = torch.stack([base, base * offset])
    aligned = join_object_waves(stack, phase_reference="first")
    literal = join_object_waves(stack, phase_reference="none")
    assert float((aligned.object_wave - base).abs().max()) < 2e-6
    assert float((literal.object_wave - base).abs().mean()) > 0.1


class _FakeSSB:
    def __init__(self, wave):
        self.wave = wave
        self.aberrations = {"C10": 1.0, "C12": 2.0, "phi12": 0.0}
        self.rotation_angle_deg = 0.0
        self.voltage_kV = 300
        self.semiangle_mrad = 21.4
        self.scan_sampling_A = (0.5, 0.5)
        self.calls = []

    def set_rotation(self, rotation_angle_deg):
        self.rotation_angle_deg = rotation_angle_deg

    def reconstruct(self, aberrations):
        self.calls.append((aberrations["C10"], aberrations["C12"], aberrations["phi12"],
                           math.radians(self.rotation_angle_deg)))
        return SimpleNamespace(object_wave=self.wave)


def test_time_average_with_shared_calibration():
    base = _object_wave()
    shift = (1.5, -0.75)
    frames = [_FakeSSB(base), _FakeSSB(fourier_shift_2d(base, shift))]
    result = ssb_time_average(frames, shifts=[(0.0, 0.0), (-shift[0], -shift[1])],
                              aberrations={"C10": 10.0, "C12": 4.0, "phi12": math.radians(12.0)},
                              rotation_angle_deg=5.0, phase_reference="none")
    assert float((result.object_wave - base).abs().max()) < 2e-5
    assert result.join_mode == "ssb_time_average"
    assert (result.voltage_kV, result.semiangle_mrad, result.scan_sampling_A) == (300, 21.4, 0.5)
    np.testing.assert_allclose(np.asarray(frames[0].calls[0], dtype=float),
                               [10.0, 4.0, math.radians(12.0), math.radians(5.0)])


def test_time_series_preserves_frames_and_can_average():
    base = _object_wave()
    changed = base * complex(math.cos(0.03), math.sin(0.03))
    frames = [_FakeSSB(base), _FakeSSB(fourier_shift_2d(changed, (1.0, -0.5)))]
    shifts = [(0.0, 0.0), (-1.0, 0.5)]
    series = ssb_time_series(frames, shifts=shifts, phase_reference="none")
    joined = ssb_time_average(frames, shifts=shifts, phase_reference="none")
    avg = series.time_average()
    assert tuple(series.object_waves.shape) == (2, *base.shape)
    assert series.mode == "shared_calibration_time_series"
    assert avg.join_mode == "shared_calibration_time_series_average"
    assert float((series.object_waves[1] - series.object_waves[0]).abs().mean()) > 0.01
    assert float((avg.object_wave - joined.object_wave).abs().max()) < 2e-6


@pytest.mark.parametrize("shape", [(64, 64), (128, 128), (256, 256), (512, 512), (128, 256),
                                   (1024, 64)])
@pytest.mark.parametrize("ref", ["first", "none"])
def test_matches_fp64_oracle(shape, ref):
    rng = np.random.default_rng(shape[0] + shape[1])
    n = 5
    amp = 1.0 + 0.05 * rng.standard_normal((n, *shape))
    waves = amp * np.exp(1j * (0.2 * rng.standard_normal((n, *shape)) + rng.uniform(-3, 3, (n, 1, 1))))
    shifts = rng.uniform(-6.0, 6.0, (n, 2))
    weights = rng.uniform(0.2, 1.0, n)
    want_joined, want_aligned = to.join_object_waves(waves, shifts, weights, ref)
    stack = torch.as_tensor(waves.astype(np.complex64), device=DEV)
    res, aligned = join_object_waves(stack, shifts=shifts, weights=weights, phase_reference=ref,
                                     return_aligned_stack=True)
    scale = np.abs(want_aligned).max()
    assert np.abs(aligned.cpu().numpy() - want_aligned).max() < 3e-6 * scale
    assert np.abs(res.object_wave.cpu().numpy() - want_joined).max() < 3e-6 * scale
    # real input keeps its dtype; integer shifts are exact rolls up to float32 rounding
    real = torch.as_tensor(rng.standard_normal(shape).astype(np.float32), device=DEV)
    rolled = fourier_shift_2d(real, (3, -2))
    assert rolled.dtype == torch.float32
    np.testing.assert_allclose(rolled.cpu().numpy(), np.roll(real.cpu().numpy(), (3, -2), axis=(0, 1)),
                               atol=2e-5)


def test_time_series_through_ssb_sessions():
    spec = CONFIGS["plain_128x128_det128"]
    kw = dict(voltage_kV=spec.voltage_kV, semiangle_mrad=spec.semiangle_mrad,
              scan_sampling_A=spec.scan_step_A, det_sampling=spec.det_sampling_mrad)
    sessions = []
    for seed in (3, 4, 5):
        from dataclasses import replace
        counts = generate(replace(spec, seed=seed), DEV).counts
        sessions.append(SSB.from_array(counts, **kw))
    ab = {"C10": 0.0, "C12": 0.0, "phi12": 0.0}
    shifts = [(0.0, 0.0), (0.5, -0.25), (-1.0, 2.0)]
    series = ssb_time_series(sessions, shifts=shifts, aberrations=ab)
    waves = [s.reconstruct(ab).object_wave.cpu().numpy() for s in sessions]
    _, want_aligned = to.join_object_waves(np.stack(waves), shifts, None, "first")
    got = series.object_waves.cpu().numpy()
    assert np.abs(got - want_aligned).max() < 3e-6 * np.abs(want_aligned).max()
    avg = ssb_time_average(sessions, shifts=shifts, aberrations=ab)
    assert avg.object_wave.shape == (128, 128)
    for s in sessions:
        s.close()
