"""BF columns written by the frame-sum pass (``qssb_bf_box_estimate``,
``qssb_mean_dp_u64_box``, ``qssb_bf_box_map``, ``qssb_scan_fft_half_mapped``)
and the cold reconstructor that uses them.

Integer work, so bit-exact: the sums equal ``qssb_mean_dp_u64``'s, every box
column equals the gathered column of its pixel, and a cold reconstruction
through the box gives the same phase bits as through the gather. When the
estimate misses part of the disk the map's ok flag is 0 and the reconstructor
gathers instead (same bits again).
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from quantem.gpu_b200 import ops
from quantem.gpu_b200.pipeline import ColdReconstructor
from quantem.gpu_b200.synthetic import CONFIGS, generate

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
KW = dict(semiangle=20.0, scan_sampling=0.5, det_sampling=20.0 / 24.0, voltage_kV=300)


@pytest.fixture(scope="module")
def counts128():
    return generate(CONFIGS["plain_128x128_det128"], device=DEV).counts.contiguous()


def test_box_sums_and_columns_are_exact(counts128):
    frames = counts128.view(-1, 128, 128)
    cap = 8192
    sample, _ = ops.mean_dp_u64(frames[:512], want_mean=False)
    box = ops.bf_box_estimate(sample, (128, 128), cap)
    r0, r1, c0, c1, width, npix, valid, _ = box.cpu().numpy().tolist()
    assert valid == 1 and width == c1 - c0 and npix == (r1 - r0) * width
    assert c0 % 8 == 0 and c1 % 8 == 0 and 1500 < npix < 4000
    cols = torch.zeros((cap, frames.shape[0]), dtype=torch.uint16, device=DEV)
    sums = ops.mean_dp_u64_box(counts128, box, cols)
    ref, _ = ops.mean_dp_u64(counts128, want_mean=False)
    assert torch.equal(sums, ref)
    lin = torch.tensor([(r * 128 + c) for r in range(r0, r1) for c in range(c0, c1)],
                       dtype=torch.int32, device=DEV)
    want = ops.gather_bf_columns(counts128, lin)
    assert torch.equal(cols[:npix].view(torch.int16), want.view(torch.int16))
    # the selection's pixels all map into the box, to their own columns
    sel = ops.select_bf(sums, (128, 128), frames.shape[0])
    n_bf = ops.read_bf_info(sel).n_bf
    bmap, ok = ops.bf_box_map(sel, (128, 128), box, cap)
    assert int(ok[0]) == 1
    m = bmap[:n_bf].cpu().numpy()
    p = sel.bf_linear[:n_bf].cpu().numpy()
    np.testing.assert_array_equal(m, (p // 128 - r0) * width + (p % 128 - c0))
    g_box = ops.scan_fft_half_mapped(cols, bmap, n_bf, (128, 128))
    g_ref = ops.scan_fft_half(ops.gather_bf_columns(counts128, sel.bf_linear[:n_bf]), (128, 128))
    assert torch.equal(g_box.view(torch.float32), g_ref.view(torch.float32))


def test_cold_reconstruction_through_the_box_is_bit_identical(counts128):
    boxed = ColdReconstructor(counts128, use_box=True, **KW)
    plain = ColdReconstructor(counts128, use_box=False, **KW)
    assert boxed.use_box and not plain.use_box
    for _ in range(2):
        a = boxed.run().clone()
        b = plain.run().clone()
        assert torch.equal(a, b)
    assert boxed.box_runs == 2


def test_missed_disk_falls_back_to_the_gather(counts128):
    """The first 512 frames see the disk 12 detector columns to the right of
    where the whole scan puts it: the box from their sums misses the selected
    disk's left side, the ok flag is 0, the run gathers, and the phase equals
    the gathering reconstructor's."""
    shifted = counts128.clone()
    frames = shifted.view(-1, 128, 128)
    f16 = shifted.view(torch.int16).view(-1, 128, 128)
    f16[:512] = torch.roll(f16[:512], 12, dims=2)
    boxed = ColdReconstructor(shifted, use_box=True, **KW)
    plain = ColdReconstructor(shifted, use_box=False, **KW)
    a = boxed.run().clone()
    b = plain.run().clone()
    assert boxed.box_runs == 0
    assert torch.equal(a, b)
    # a box record that is not valid (too small a capacity) maps nothing
    box = ops.bf_box_estimate(ops.mean_dp_u64(frames[:512], want_mean=False)[0], (128, 128), 16)
    assert int(box[6]) == 0
    cols = torch.zeros((16, frames.shape[0]), dtype=torch.uint16, device=DEV)
    sums = ops.mean_dp_u64_box(shifted, box, cols)
    assert int(cols.view(torch.int16).abs().sum()) == 0
    sel = ops.select_bf(sums, (128, 128), frames.shape[0])
    _, ok = ops.bf_box_map(sel, (128, 128), box, 16)
    assert int(ok[0]) == 0
