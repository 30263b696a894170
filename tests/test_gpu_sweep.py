"""Batched aberration sweep over three uneven scans in one CUDA-graph launch.

Scans of 96x96, 128x128 and 160x120 positions (128^2 detector) are padded by
the reference's rule (backend.py:229-269) to 128^2, 128^2 and 256^2, and
scored with candidates that include C3 (C30). Checks: the graph replay gives
the same bits as direct calls with the same (autotuned) partition and on
every replay; the losses match the FP64 GPU restatement of the oracle within
the reference's loss tolerance (tests/ssb_precision.py:7-10 of
bobleesj/quantem.gpu: rel 1e-5, abs 1e-6); the true aberrations, hidden among
random candidates, give the lowest loss of each scan.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import ssb_oracle as so
from oracle import ssb_torch_fp64 as tf
from quantem.gpu_b200 import B200SSBBackend, _lib, ops
from quantem.gpu_b200.sweep import MultiScanSweep
from quantem.gpu_b200.synthetic import draw_aberrations, generate, sweep_specs

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
N_CAND = 8


@pytest.fixture(scope="module")
def scans():
    out = []
    for spec in sweep_specs():
        counts = generate(spec, DEV).counts
        be = B200SSBBackend(counts, semiangle=spec.semiangle_mrad, scan_sampling=spec.scan_step_A,
                            det_sampling=spec.det_sampling_mrad, voltage_kV=spec.voltage_kV,
                            device=DEV)
        out.append((spec, counts, be))
    return out


@pytest.fixture(scope="module")
def candidates(scans):
    rng = np.random.default_rng(11)
    cands = []
    for i, (spec, _, _) in enumerate(scans):
        c = draw_aberrations(rng, N_CAND)
        c[i % N_CAND] = (spec.C10, spec.C12, spec.phi12, spec.C30)  # hide the truth
        cands.append(c)
    return cands


def test_reference_padding_of_uneven_scans(scans):
    assert [be.scan_shape for _, _, be in scans] == [(128, 128), (128, 128), (256, 256)]


def test_graph_sweep_matches_direct_calls_and_repeats(scans, candidates):
    sw = MultiScanSweep([be for _, _, be in scans], N_CAND)
    first = sw(candidates)
    second = sw(candidates)
    for a, b in zip(first, second):
        np.testing.assert_array_equal(a, b)
    # the graph holds exactly the kernels the direct calls launch (the library
    # counts every launch): at 128^2 the phase table and the pair kernel, at
    # 256^2 the table and a row and a column pass per L2-sized BF chunk, then
    # the fold
    lib = _lib.load()
    direct_launches = 0
    for (_, _, be), slot, c, got in zip(scans, sw._slots, candidates, first):
        n0 = lib.qssb_kernel_launches()
        ops.loss_batch(be.G_qk, be._geom_dev, be._q_row, be._q_col, slot["cal"],
                       torch.as_tensor(c, device=DEV), flags=slot["flags"],
                       overlap=slot["overlap"])
        direct_launches += lib.qssb_kernel_launches() - n0
        direct, _ = ops.loss_batch(be.G_qk, be._geom_dev, be._q_row, be._q_col, slot["cal"],
                                   torch.as_tensor(c, device=DEV), flags=slot["flags"])
        np.testing.assert_array_equal(direct.cpu().numpy(), got)
    assert sw.launches_per_replay == direct_launches
    assert sw._slots[0]["overlap"] is not None  # 128^2: two launches
    assert direct_launches > 2 * 2


def test_sweep_losses_match_fp64_and_find_the_truth(scans, candidates):
    sw = MultiScanSweep([be for _, _, be in scans], N_CAND)
    got = sw(candidates)
    for i, ((spec, counts, be), c, losses) in enumerate(zip(scans, candidates, got)):
        assert int(np.argmin(losses)) == i % N_CAND, (spec.scan_shape, losses)
        padded = torch.as_tensor(so.pad_or_crop_scan(counts.cpu().numpy()), device=DEV)
        prep = tf.prepare(padded, voltage_kV=spec.voltage_kV, semiangle_mrad=spec.semiangle_mrad,
                          scan_sampling=spec.scan_step_A, det_sampling=spec.det_sampling_mrad)
        for j in (i % N_CAND, (i + 3) % N_CAND):
            want, _ = tf.phase_variance_loss(prep, so.Aberrations(*map(float, c[j])))
            assert abs(losses[j] - want) <= 1e-5 * abs(want) + 1e-6, (spec.scan_shape, j, losses[j], want)


def test_persistent_sweep_is_a_few_kernels_per_scan(scans, candidates):
    """By default the 256^2 scan's row and column passes run in one launch.
    With C30 candidates there is no quadratic phase table, so the graph holds
    one kernel per 128^2 scan (the pair kernel, which folds in its last CTA)
    and four for the 256^2 scan (setup, queue, reduce, final); the losses
    agree with the launch-sequence sweep to float32 rounding (the C30 path)
    and still rank the truth first."""
    seq = MultiScanSweep([be for _, _, be in scans], N_CAND, tune=False, persistent=False)
    per = MultiScanSweep([be for _, _, be in scans], N_CAND, tune=False)
    want = seq(candidates)
    got = per(candidates)
    assert per.launches_per_replay == 1 + 1 + 4
    assert seq.launches_per_replay > per.launches_per_replay
    for i, (w, g) in enumerate(zip(want, got)):
        np.testing.assert_allclose(g, w, rtol=1e-6, atol=0)
        assert int(np.argmin(g)) == i % N_CAND


def test_cancel_flag_registered_before_capture_stops_a_replay(scans, candidates):
    """The graph captures the registered flag's address: set, a replay ends
    with NaN losses for every scan (the 128^2 pair kernels and the 256^2
    persistent kernel both poll it) and no hang; cleared, the losses return."""
    flag = torch.zeros(1, dtype=torch.int32, device=DEV)
    try:
        ops.set_cancel_flag(flag)
        sw = MultiScanSweep([be for _, _, be in scans], N_CAND, tune=False)
        want = sw(candidates)
        flag.fill_(1)
        got = sw(candidates)
        assert all(np.all(np.isnan(g)) for g in got)
        flag.fill_(0)
        for w, g in zip(want, sw(candidates)):
            np.testing.assert_array_equal(g, w)
    finally:
        ops.set_cancel_flag(None)
