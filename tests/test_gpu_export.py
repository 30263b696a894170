"""The exact bright-field companion (``export_brightfield``) against the file
the reference's own writer produced (engine.py:577-701, fixtures from
``tests/golden/make_golden.py``): same suffix, same bytes, on u16 counts that
fit u8, the same block with one hot pixel outside the BF disk (the whole
block decides: u16), and u8 counts; plus the reference's error rules.
"""
from __future__ import annotations

import hashlib
from pathlib import Path

import numpy as np
import pytest
import torch

from quantem.gpu_b200 import B200SSBBackend, ops
from recipes import disk_input, export_cases

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def disk_backend():
    be = B200SSBBackend(torch.as_tensor(disk_input(123), device=DEV), semiangle=21.4,
                        scan_sampling=0.5, det_sampling=1.0, voltage_kV=300, bf_radius=3)
    yield be
    be.close()


@pytest.mark.parametrize("name", ["u16_fits_u8", "u16_hot_pixel_outside_bf", "u8"])
@pytest.mark.parametrize("host_input", [False, True], ids=["device", "host"])
def test_export_matches_reference_writer(disk_backend, tmp_path, name, host_input):
    with np.load(GOLDEN / "ref_bf_export.npz") as z:
        gold = {k: z[k] for k in z.files}
    data = export_cases()[name]
    arg = data if host_input else torch.as_tensor(data, device=DEV)
    path, seconds = disk_backend.export_brightfield(arg, tmp_path / name)
    assert path.suffix == str(gold[name + "_suffix"])
    raw = path.read_bytes()
    assert len(raw) == int(gold[name + "_bytes"])
    assert hashlib.sha256(raw).hexdigest() == str(gold[name + "_sha256"])
    assert seconds >= 0.0


def test_export_chunks_and_rules(tmp_path):
    """More BF pixels than one 256-pixel chunk (two pinned buffers in turn),
    against a direct numpy gather; a stale file of the other suffix is left
    alone and one of the same name is replaced; float counts and a wrong
    scan shape raise as in the reference."""
    rng = np.random.default_rng(3)
    data = rng.integers(0, 4000, size=(32, 32, 48, 48), dtype=np.uint16)
    be = B200SSBBackend(torch.as_tensor(data, device=DEV), semiangle=20.0, scan_sampling=0.5,
                        det_sampling=1.0, voltage_kV=300, bf_radius=18)
    padded = torch.as_tensor(data, device=DEV)
    assert be.num_bf > 600
    # the backend pads 32^2 scans to 128^2: export takes data of the engine's scan shape
    with pytest.raises(ValueError):
        be.export_brightfield(padded, tmp_path / "bad")
    full = rng.integers(0, 4000, size=be.scan_shape + (48, 48), dtype=np.uint16)
    (tmp_path / "bf.u16").write_bytes(b"stale")
    path, _ = be.export_brightfield(full, tmp_path / "bf")
    lin = be.bf_inds_row.astype(np.int64) * 48 + be.bf_inds_col
    want = np.ascontiguousarray(full.reshape(-1, 48 * 48)[:, lin].T)
    assert path.name == "bf.u16"
    assert path.read_bytes() == want.tobytes()
    with pytest.raises(TypeError):
        be.export_brightfield(full.astype(np.float32), tmp_path / "f")
    with pytest.raises(TypeError):
        be.export_brightfield(torch.as_tensor(full.astype(np.int32), device=DEV), tmp_path / "i")
    be.close()


@pytest.mark.parametrize("dtype,n,offset", [(np.uint16, 1_000_003, 0), (np.uint16, 37, 3),
                                           (np.uint8, 999_999, 5), (np.uint8, 7, 1),
                                           (np.uint16, 0, 0)])
def test_count_max(dtype, n, offset):
    """The whole-block maximum behind the u8 narrowing, with unaligned heads
    and tails (a view that starts ``offset`` elements in)."""
    rng = np.random.default_rng(n)
    top = 256 if dtype == np.uint8 else 65536
    host = rng.integers(0, top // 2, size=n + offset, dtype=dtype)
    if n:
        host[offset + n // 2] = top - 1 - (n % 3)
    t = torch.as_tensor(host, device=DEV)[offset:]
    got = int(ops.count_max(t).cpu()[0]) & 0xFFFFFFFF
    assert got == (int(host[offset:].max()) if n else 0)
