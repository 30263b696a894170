"""The table-driven 128x128 phase-variance loss (``qssb_overlap_table`` +
``qssb_loss_batch_ex``): two BF pixels per inverse 2D FFT, their
anti-Hermitian parts packed into one complex plane and the Hermitian DC and
Nyquist-line parts transformed on their own.

Checked against the FP64 oracle (loss 1e-5 relative, mean phase 2e-4 rad at
the 99.9th percentile, as the other loss tests) and against the table-free
kernel (float32 rounding only), on the reference test's 27-pixel disk case
and on the CPU-runnable workload padded to 128^2 (437 pixels: an odd count,
so the last pixel of a chunk is transformed alone); plus the table itself
against an FP64 evaluation of the apertures, repeatability, and the
single-candidate, three-candidate and 64-candidate plans.

At 256^2 and 512^2 the two-pass loss reads the same apertures from its own
table order; there the table layout, the losses against the oracle and the
table-free kernel, and the backend's table switch are checked.
"""
from __future__ import annotations

import math

import numpy as np
import pytest
import torch

from oracle import ssb_oracle as so
from quantem.gpu_b200 import B200SSBBackend, ops
from quantem.gpu_b200._lib import (QSSB_FLAG_CHI_FP64, QSSB_FLAG_PERSISTENT,
                                   QSSB_FLAG_QUADRATIC)
from recipes import disk_input, synthetic_plain_32
from test_gpu_parity import DISK_KW, _prep_case

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
LOSS_RTOL, LOSS_ATOL, PHASE_ATOL = 1e-5, 1e-6, 2e-4
CANDS = [(-120.0, 55.0, math.radians(17.0)), (-80.0, 30.0, math.radians(-5.0)),
         (20.0, 40.0, math.radians(11.0)), (100.0, 10.0, math.radians(43.0)),
         (0.0, 0.0, 0.0)]


@pytest.fixture(scope="module", params=["disk27", "plain437"])
def case(request):
    if request.param == "disk27":
        return _prep_case(disk_input(123), **DISK_KW)
    kw = dict(voltage_kV=300, semiangle_mrad=20.0, scan_sampling=0.5, det_sampling=20.0 / 12.0)
    return _prep_case(synthetic_plain_32(), **kw)


def _cands(rows) -> torch.Tensor:
    return torch.tensor([[a, b, c, 0.0] for a, b, c in rows], dtype=torch.float32, device=DEV)


@pytest.mark.parametrize("flags", [QSSB_FLAG_QUADRATIC, QSSB_FLAG_QUADRATIC | QSSB_FLAG_CHI_FP64])
def test_table_loss_matches_oracle_and_table_free_kernel(case, flags):
    prep, cal, d = case
    table = ops.overlap_table(d["geom"], d["q_row"], d["q_col"], cal)
    cands = _cands(CANDS)
    losses, mp = ops.loss_batch(d["g"], d["geom"], d["q_row"], d["q_col"], cal, cands,
                                flags=flags, want_mean_phase=True, overlap=table)
    plain, mp_plain = ops.loss_batch(d["g"], d["geom"], d["q_row"], d["q_col"], cal, cands,
                                     flags=flags, want_mean_phase=True)
    losses, mp, plain = losses.cpu().numpy(), mp.cpu().numpy(), plain.cpu().numpy()
    for i, (a, b, c) in enumerate(CANDS):
        ref_loss, ref_mean = so.phase_variance_loss(prep.g_half, prep.geo, so.Aberrations(a, b, c),
                                                    prep.dc)
        assert losses[i] == pytest.approx(ref_loss, rel=LOSS_RTOL, abs=LOSS_ATOL), (i, flags)
        assert losses[i] == pytest.approx(plain[i], rel=2e-6, abs=1e-7)
        err = np.abs(so.wrapped_phase_error(mp[i], ref_mean))
        assert np.percentile(err, 99.9) < PHASE_ATOL
    np.testing.assert_allclose(mp, mp_plain.cpu().numpy(), rtol=0, atol=2e-5)


def test_table_matches_fp64_apertures(case):
    """table[b][e] = (A(q-k), A(q+k)) on the evaluated half set: the float32
    fast aperture with the FP64 tie rule, within float32 rounding of an FP64
    evaluation except where the rule itself switched to FP64."""
    prep, cal, d = case
    table = ops.overlap_table(d["geom"], d["q_row"], d["q_col"], cal).cpu().numpy().astype(np.float64)
    n = prep.scan_shape[0]
    rows = np.concatenate([np.repeat(np.arange(65), n), np.arange(127, 64, -1)])
    cols = np.concatenate([np.tile(np.arange(n), 65), np.full(63, 64)])
    geo = prep.geo
    qx = geo.q_row.astype(np.float64)[rows][None, :]
    qy = geo.q_col.astype(np.float64)[cols][None, :]
    kx = geo.kx[:, None].astype(np.float64)
    ky = geo.ky[:, None].astype(np.float64)
    am = so._aperture_and_angles(qx - kx, qy - ky, geo)[3]
    ap = so._aperture_and_angles(qx + kx, qy + ky, geo)[3]
    want = np.stack([am, ap], axis=-1)
    assert table.shape == want.shape
    assert np.abs(table - want).max() <= 2e-5


def test_table_loss_plans_and_repeatability(case):
    """One, three and 64 candidates (different chunk plans) agree per
    candidate with each other within float32 rounding; a call repeated gives
    identical bits."""
    prep, cal, d = case
    table = ops.overlap_table(d["geom"], d["q_row"], d["q_col"], cal)
    rng = np.random.default_rng(9)
    rows = [(float(a), float(b), float(c)) for a, b, c in
            zip(rng.uniform(-150, 150, 64), rng.uniform(0, 60, 64), rng.uniform(-1.5, 1.5, 64))]
    run = lambda r: ops.loss_batch(d["g"], d["geom"], d["q_row"], d["q_col"], cal, _cands(r),  # noqa: E731
                                   flags=QSSB_FLAG_QUADRATIC, overlap=table)[0]
    big = run(rows)
    assert torch.equal(big, run(rows))
    big = big.cpu().numpy()
    three = run(rows[:3]).cpu().numpy()
    one = run(rows[:1]).cpu().numpy()
    np.testing.assert_allclose(three, big[:3], rtol=2e-6)
    np.testing.assert_allclose(one, big[:1], rtol=2e-6)
    for i in (0, 37):
        ref, _ = so.phase_variance_loss(prep.g_half, prep.geo, so.Aberrations(*rows[i]), prep.dc)
        assert big[i] == pytest.approx(ref, rel=LOSS_RTOL, abs=LOSS_ATOL)


@pytest.mark.parametrize("flags", [0, QSSB_FLAG_CHI_FP64])
def test_table_loss_with_spherical_aberration(case, flags):
    """C30 != 0 (no quadratic factorisation): the pair kernel takes the probe
    phases directly and only the apertures from the table; against the FP64
    oracle and the table-free kernel."""
    prep, cal, d = case
    table = ops.overlap_table(d["geom"], d["q_row"], d["q_col"], cal)
    # (C10 = C12 = 0 with a small C30 is left out: there chi(q -+ k) - chi(k)
    # vanishes near q = 0 and the float32 displacements decide the overlap's
    # sign, the zero-aberration degeneracy that only the quadratic path's
    # factorised form avoids; the table-free kernel has it too)
    rows = [(-120.0, 55.0, math.radians(17.0), 3.0e4), (40.0, 20.0, 0.4, 8.0e4),
            (25.0, 5.0, 0.2, 1.0e4)]
    cands = torch.tensor(rows, dtype=torch.float32, device=DEV)
    losses, mp = ops.loss_batch(d["g"], d["geom"], d["q_row"], d["q_col"], cal, cands,
                                flags=flags, want_mean_phase=True, overlap=table)
    plain, _ = ops.loss_batch(d["g"], d["geom"], d["q_row"], d["q_col"], cal, cands, flags=flags)
    losses, mp, plain = losses.cpu().numpy(), mp.cpu().numpy(), plain.cpu().numpy()
    for i, (a, b, c, c30) in enumerate(rows):
        ref_loss, ref_mean = so.phase_variance_loss(prep.g_half, prep.geo,
                                                    so.Aberrations(a, b, c, C30=c30), prep.dc)
        assert losses[i] == pytest.approx(ref_loss, rel=LOSS_RTOL, abs=LOSS_ATOL), (i, flags)
        assert losses[i] == pytest.approx(plain[i], rel=5e-6, abs=1e-7)
        err = np.abs(so.wrapped_phase_error(mp[i], ref_mean))
        assert np.percentile(err, 99.9) < PHASE_ATOL


def test_cancel_flag_stops_a_batch_without_hanging(case):
    """A registered cancel flag that is already set stops every CTA of the
    table kernel at its first BF-pixel pair: the call returns (no hang) with
    NaN losses; cleared, the next call gives the normal losses again; a flag
    that is never set changes nothing."""
    prep, cal, d = case
    table = ops.overlap_table(d["geom"], d["q_row"], d["q_col"], cal)
    cands = _cands(CANDS * 8)  # 40 candidates: the one-launch fold
    run = lambda: ops.loss_batch(d["g"], d["geom"], d["q_row"], d["q_col"], cal, cands,  # noqa: E731
                                 flags=QSSB_FLAG_QUADRATIC, overlap=table)[0].cpu().numpy()
    want = run()
    flag = torch.zeros(1, dtype=torch.int32, device=DEV)
    try:
        ops.set_cancel_flag(flag)
        np.testing.assert_array_equal(run(), want)
        flag.fill_(1)
        got = run()
        assert np.all(np.isnan(got))
        flag.fill_(0)
        np.testing.assert_array_equal(run(), want)
    finally:
        ops.set_cancel_flag(None)
    np.testing.assert_array_equal(run(), want)


# ---------------------------------------------------------------- 256^2 .. 1024^2
# The two-pass loss (row pass, then column pass) reads the same apertures from
# a per-geometry table in its own order: rows 0 .. N/2 of the scan-frequency
# plane over all N columns, then the partner (N - r, N/2) of each row r of the
# Nyquist-column relation at index (N/2 + 1) N + r.


@pytest.fixture(scope="module", params=[256, 512])
def big_case(request):
    n = request.param
    return _prep_case(disk_input(123, scan=(n, n)), **DISK_KW)


def test_two_pass_table_layout_matches_fp64_apertures(big_case):
    prep, cal, d = big_case
    n = prep.scan_shape[0]
    table = ops.overlap_table(d["geom"], d["q_row"], d["q_col"], cal)
    assert ops.overlap_table_bytes(cal) == 8 * cal.n_bf * ((n // 2 + 1) * n + n // 2)
    table = table.cpu().numpy().astype(np.float64)
    assert table.shape == (cal.n_bf, (n // 2 + 1) * n + n // 2, 2)
    main = (n // 2 + 1) * n
    np.testing.assert_array_equal(table[:, main], 0.0)  # index r = 0 of the partners: unused
    rows = np.concatenate([np.repeat(np.arange(n // 2 + 1), n), np.arange(n - 1, n // 2, -1)])
    cols = np.concatenate([np.tile(np.arange(n), n // 2 + 1), np.full(n // 2 - 1, n // 2)])
    geo = prep.geo
    qx = geo.q_row.astype(np.float64)[rows][None, :]
    qy = geo.q_col.astype(np.float64)[cols][None, :]
    kx = geo.kx[:, None].astype(np.float64)
    ky = geo.ky[:, None].astype(np.float64)
    am = so._aperture_and_angles(qx - kx, qy - ky, geo)[3]
    ap = so._aperture_and_angles(qx + kx, qy + ky, geo)[3]
    got = np.delete(table, main, axis=1)
    assert np.abs(got - np.stack([am, ap], axis=-1)).max() <= 2e-5


@pytest.mark.parametrize("flags", [QSSB_FLAG_QUADRATIC, QSSB_FLAG_QUADRATIC | QSSB_FLAG_CHI_FP64, 0])
def test_two_pass_table_loss_matches_oracle_and_table_free_kernel(big_case, flags):
    """The quadratic float32 path reads the table; the FP64-chi and C30 paths
    accept it and evaluate as before. Losses against the FP64 oracle and the
    table-free kernel, mean phases against the table-free kernel."""
    prep, cal, d = big_case
    table = ops.overlap_table(d["geom"], d["q_row"], d["q_col"], cal)
    rows = CANDS if flags else [(-120.0, 55.0, math.radians(17.0)), (40.0, 20.0, 0.4)]
    c30 = 0.0 if flags else 3.0e4
    cands = torch.tensor([[a, b, c, c30] for a, b, c in rows], dtype=torch.float32, device=DEV)
    losses, mp = ops.loss_batch(d["g"], d["geom"], d["q_row"], d["q_col"], cal, cands,
                                flags=flags, want_mean_phase=True, overlap=table)
    plain, mp_plain = ops.loss_batch(d["g"], d["geom"], d["q_row"], d["q_col"], cal, cands,
                                     flags=flags, want_mean_phase=True)
    losses, mp, plain = losses.cpu().numpy(), mp.cpu().numpy(), plain.cpu().numpy()
    for i, (a, b, c) in enumerate(rows):
        ref_loss, _ = so.phase_variance_loss(prep.g_half, prep.geo,
                                             so.Aberrations(a, b, c, C30=c30), prep.dc)
        assert losses[i] == pytest.approx(ref_loss, rel=LOSS_RTOL, abs=LOSS_ATOL), (i, flags)
        assert losses[i] == pytest.approx(plain[i], rel=2e-6, abs=1e-7)
    np.testing.assert_allclose(mp, mp_plain.cpu().numpy(), rtol=0, atol=2e-5)


def test_two_pass_table_rejects_a_wrong_size(big_case):
    prep, cal, d = big_case
    table = ops.overlap_table(d["geom"], d["q_row"], d["q_col"], cal)
    cands = _cands(CANDS[:1])
    with pytest.raises(ValueError):
        ops.loss_batch(d["g"], d["geom"], d["q_row"], d["q_col"], cal, cands,
                       flags=QSSB_FLAG_QUADRATIC, overlap=table[:, :-1].contiguous())


def test_backend_builds_the_256_table_and_agrees_without_it():
    counts = disk_input(123, scan=(256, 256))
    be = B200SSBBackend(torch.as_tensor(counts, device=DEV), semiangle=21.4, scan_sampling=0.5,
                        det_sampling=1.0, voltage_kV=300, bf_radius=3)
    c1 = np.linspace(-100.0, 100.0, 9)
    with_table = be.variance_loss_batch(c1, 20.0, 0.3).cpu().numpy()
    assert be._overlap_table() is not None
    be.use_overlap_table = False
    assert be._overlap_table() is None
    without = be.variance_loss_batch(c1, 20.0, 0.3).cpu().numpy()
    np.testing.assert_allclose(with_table, without, rtol=2e-6, atol=1e-7)
    be.close()


# ------------------------------------------- the persistent one-launch loss
# At 256^2 (half set, float32 chi) QSSB_FLAG_PERSISTENT runs every row and
# column item of the batch in one k_loss_queue launch from a ticket queue,
# with bounded waits on per-chunk completion counts, instead of a row and a
# column launch per BF chunk. Same plan, so the same bits on the quadratic
# path (float32 rounding on the C30 path).


@pytest.fixture(scope="module")
def case256():
    return _prep_case(disk_input(123, scan=(256, 256)), **DISK_KW)


def _rows(n, seed=3, c30=False):
    rng = np.random.default_rng(seed)
    out = np.stack([rng.uniform(-150, 150, n), rng.uniform(0, 60, n), rng.uniform(-1.5, 1.5, n),
                    rng.uniform(0.0, 5e4, n) if c30 else np.zeros(n)], axis=1)
    return torch.tensor(out, dtype=torch.float32, device=DEV)


@pytest.mark.parametrize("n_cand,c30", [(1, False), (5, True), (27, False), (64, False),
                                        (64, True), (70, False)])
def test_persistent_launch_matches_the_launch_sequence(case256, n_cand, c30):
    """1 .. 70 candidates: one group, a full group of 27, 64 = 27 + 27 + 10
    and 70 = 27 + 27 + 16 (a last group with larger chunks); quadratic and C30."""
    prep, cal, d = case256
    table = ops.overlap_table(d["geom"], d["q_row"], d["q_col"], cal)
    cands = _rows(n_cand, seed=n_cand, c30=c30)
    fl = 0 if c30 else QSSB_FLAG_QUADRATIC
    n0 = ops.LAUNCH_COUNT
    q, mq = ops.loss_batch(d["g"], d["geom"], d["q_row"], d["q_col"], cal, cands,
                           flags=fl | QSSB_FLAG_PERSISTENT, want_mean_phase=True, overlap=table)
    launches = ops.LAUNCH_COUNT - n0
    seq, ms = ops.loss_batch(d["g"], d["geom"], d["q_row"], d["q_col"], cal, cands, flags=fl,
                             want_mean_phase=True, overlap=table)
    if c30:
        # the general-chi arithmetic, inlined into two different kernels, is
        # contracted into FMAs differently: float32 rounding, not the plan
        torch.testing.assert_close(q, seq, rtol=1e-6, atol=0)
        torch.testing.assert_close(mq, ms, rtol=0, atol=2e-6)
    else:
        assert torch.equal(q, seq)
        assert torch.equal(mq, ms)
    # eq table (quadratic), setup, the queue kernel, reduce, final
    assert launches == (4 if c30 else 5)
    # the sequence: the same plus a row and a column launch per BF chunk
    assert ops.LAUNCH_COUNT - n0 - launches > launches
    if n_cand <= 5:
        for i in range(n_cand):
            a, b, c, c3 = (float(v) for v in cands[i].cpu())
            ref, _ = so.phase_variance_loss(prep.g_half, prep.geo, so.Aberrations(a, b, c, C30=c3),
                                            prep.dc)
            assert float(q[i]) == pytest.approx(ref, rel=LOSS_RTOL, abs=LOSS_ATOL)


def test_persistent_launch_repeats_its_bits_without_the_table(case256):
    prep, cal, d = case256
    cands = _rows(30)
    run = lambda fl: ops.loss_batch(d["g"], d["geom"], d["q_row"], d["q_col"], cal, cands,  # noqa: E731
                                    flags=fl)[0]
    a = run(QSSB_FLAG_QUADRATIC | QSSB_FLAG_PERSISTENT)
    assert torch.equal(a, run(QSSB_FLAG_QUADRATIC | QSSB_FLAG_PERSISTENT))
    assert torch.equal(a, run(QSSB_FLAG_QUADRATIC))


def test_persistent_launch_cancel_flag_gives_nan_without_hanging(case256):
    """A set cancel flag makes every queue wait give up at once: the launch
    drains (no hang) and the losses are NaN; cleared, the losses come back."""
    prep, cal, d = case256
    table = ops.overlap_table(d["geom"], d["q_row"], d["q_col"], cal)
    cands = _rows(40)
    run = lambda: ops.loss_batch(d["g"], d["geom"], d["q_row"], d["q_col"], cal, cands,  # noqa: E731
                                 flags=QSSB_FLAG_QUADRATIC | QSSB_FLAG_PERSISTENT,
                                 overlap=table)[0].cpu().numpy()
    want = run()
    flag = torch.zeros(1, dtype=torch.int32, device=DEV)
    try:
        ops.set_cancel_flag(flag)
        np.testing.assert_array_equal(run(), want)
        flag.fill_(1)
        assert np.all(np.isnan(run()))
        flag.fill_(0)
        np.testing.assert_array_equal(run(), want)
    finally:
        ops.set_cancel_flag(None)
