"""The graph-launched cold pipeline (quantem.gpu_b200.pipeline) gives the same
bits as the backend's own launch sequence, for two different acquisitions
loaded into the same input buffer (dc and BF count change between them)."""
from __future__ import annotations

from dataclasses import replace

import numpy as np
import pytest
import torch

from quantem.gpu_b200 import B200SSBBackend
from quantem.gpu_b200.pipeline import ColdReconstructor
from quantem.gpu_b200.synthetic import CONFIGS, generate

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


@pytest.mark.parametrize("graphs", [True, False])
def test_pipeline_matches_backend_bitwise(graphs):
    spec = CONFIGS["plain_128x128_det128"]
    kw = dict(semiangle=spec.semiangle_mrad, scan_sampling=spec.scan_step_A,
              det_sampling=spec.det_sampling_mrad, voltage_kV=spec.voltage_kV)
    first = generate(spec, DEV).counts
    second = generate(replace(spec, seed=9, dose=3000.0, C10=40.0), DEV).counts
    buf = first.clone()
    rec = ColdReconstructor(buf, use_graphs=graphs, **kw)
    for data in (first, second, first):
        rec.load(data)
        ph = rec.run().clone()
        be = B200SSBBackend(data, device=DEV, **kw)
        _, want = be.object_and_phase(0.0, 0.0, 0.0)
        assert rec.last_info.n_bf == be.num_bf
        np.testing.assert_array_equal(ph.cpu().numpy(), want.cpu().numpy())
