"""The proposer MLP's GEMM on the tcgen05 tensor cores (``qssb_gemm_bf16_tc``)
against an FP32 product of the same BF16 operands: all four transpose
combinations, one and several K splits, the bias / accumulate / GELU
epilogue (in the reduce pass with split K, in the MMA kernel without), and
the training step's shapes. BF16 products are exact in FP32;
only the summation order differs (FP32 accumulation in the tensor core, the
splits added in order), hence the 1e-5 relative bound on the largest
element, and two calls give identical bits."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from quantem.gpu_b200 import _lib

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


def _gemm_tc(a, ta, b, tb, m, n, k, splits, bias=None, c=None, accumulate=False, act=None):
    lib = _lib.load()
    nbytes = ctypes.c_size_t(0)
    _lib.check(lib.qssb_gemm_tc_workspace_bytes(m, n, k, splits, ctypes.byref(nbytes)))
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device=DEV)
    p = lambda t: ctypes.c_void_p(0 if t is None else t.data_ptr())  # noqa: E731
    _lib.check(lib.qssb_gemm_bf16_tc(p(a), a.shape[1], int(ta), p(b), b.shape[1], int(tb), m, n, k,
                                     splits, p(bias), int(accumulate), p(c), n, p(act), n, p(ws),
                                     ws.numel(), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    status = int(ws[-256:].view(torch.int32)[0])
    assert status == 0, "a bounded wait in the kernel gave up"


@pytest.mark.parametrize("ta,tb", [(False, False), (False, True), (True, False), (True, True)])
@pytest.mark.parametrize("m,n,k,splits", [(128, 128, 64, 1), (256, 384, 512, 1), (256, 256, 1024, 4)])
def test_gemm_tc_matches_fp32_product(ta, tb, m, n, k, splits):
    g = torch.Generator(device=DEV).manual_seed(m + n + k + 2 * ta + tb)
    a = torch.randn((k, m) if ta else (m, k), generator=g, device=DEV).to(torch.bfloat16)
    b = torch.randn((n, k) if tb else (k, n), generator=g, device=DEV).to(torch.bfloat16)
    ref = (a.float().T if ta else a.float()) @ (b.float().T if tb else b.float())
    c = torch.empty((m, n), device=DEV)
    _gemm_tc(a, ta, b, tb, m, n, k, splits, c=c)
    err = (c - ref).abs().max().item()
    assert err <= 1e-5 * ref.abs().max().item() + 1e-6, err
    again = torch.empty_like(c)
    _gemm_tc(a, ta, b, tb, m, n, k, splits, c=again)
    assert torch.equal(c, again)


def test_gemm_tc_epilogue_and_training_shapes():
    """Forward layer 1 of the MLP (256 x 16384 @ 16384 x 512, 32 K splits)
    with bias and GELU; the first-layer weight gradient (16384 x 256 @ 256 x
    512, A transposed) accumulated into an existing C."""
    g = torch.Generator(device=DEV).manual_seed(3)
    x = (0.1 * torch.randn((256, 16384), generator=g, device=DEV)).to(torch.bfloat16)
    w = (0.01 * torch.randn((16384, 512), generator=g, device=DEV)).to(torch.bfloat16)
    bias = torch.randn(512, generator=g, device=DEV)
    z = torch.empty((256, 512), device=DEV)
    act = torch.empty((256, 512), dtype=torch.bfloat16, device=DEV)
    _gemm_tc(x, False, w, False, 256, 512, 16384, 32, bias=bias, c=z, act=act)
    ref = x.float() @ w.float() + bias
    assert (z - ref).abs().max().item() <= 1e-5 * ref.abs().max().item() + 1e-6
    gelu = 0.5 * ref * (1 + torch.tanh(0.7978845608028654 * (ref + 0.044715 * ref ** 3)))
    assert (act.float() - gelu).abs().max().item() <= 1e-2 * gelu.abs().max().item()
    dz = (0.1 * torch.randn((256, 512), generator=g, device=DEV)).to(torch.bfloat16)
    c0 = torch.randn((16384, 512), generator=g, device=DEV)
    c = c0.clone()
    _gemm_tc(x, True, dz, False, 16384, 512, 256, 1, c=c, accumulate=True)
    ref = c0 + x.float().T @ dz.float()
    assert (c - ref).abs().max().item() <= 1e-5 * ref.abs().max().item() + 1e-6
    # without split K the MMA kernel applies bias and GELU itself (layer 2's shape)
    a2 = (0.1 * torch.randn((256, 512), generator=g, device=DEV)).to(torch.bfloat16)
    w2 = (0.05 * torch.randn((512, 512), generator=g, device=DEV)).to(torch.bfloat16)
    z2 = torch.empty((256, 512), device=DEV)
    act2 = torch.empty((256, 512), dtype=torch.bfloat16, device=DEV)
    _gemm_tc(a2, False, w2, False, 256, 512, 512, 1, bias=bias, c=z2, act=act2)
    ref2 = a2.float() @ w2.float() + bias
    assert (z2 - ref2).abs().max().item() <= 1e-5 * ref2.abs().max().item() + 1e-6
    gelu2 = 0.5 * ref2 * (1 + torch.tanh(0.7978845608028654 * (ref2 + 0.044715 * ref2 ** 3)))
    assert (act2.float() - gelu2).abs().max().item() <= 1e-2 * gelu2.abs().max().item()
    # and the same with only the BF16 activation written
    act3 = torch.empty_like(act2)
    _gemm_tc(a2, False, w2, False, 256, 512, 512, 1, bias=bias, act=act3)
    assert torch.equal(act3, act2)


def test_gemm_tc_rejects_unsupported_shapes():
    lib = _lib.load()
    nbytes = ctypes.c_size_t(0)
    _lib.check(lib.qssb_gemm_tc_workspace_bytes(128, 128, 64, 1, ctypes.byref(nbytes)))
    a = torch.zeros((128, 64), dtype=torch.bfloat16, device=DEV)
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device=DEV)
    c = torch.empty((128, 128), device=DEV)
    rc = lib.qssb_gemm_bf16_tc(ctypes.c_void_p(a.data_ptr()), 64, 0, ctypes.c_void_p(a.data_ptr()), 64,
                               1, 128, 128, 96, 1, None, 0, ctypes.c_void_p(c.data_ptr()), 128, None, 0,
                               ctypes.c_void_p(ws.data_ptr()), ws.numel(), None)
    assert rc == _lib.QSSB_ERR_UNSUPPORTED
    # without split K, C must take 16-byte stores
    rc = lib.qssb_gemm_bf16_tc(ctypes.c_void_p(a.data_ptr()), 64, 0, ctypes.c_void_p(a.data_ptr()), 64,
                               1, 128, 128, 64, 1, None, 0, ctypes.c_void_p(c.data_ptr() + 4), 128,
                               None, 0, ctypes.c_void_p(ws.data_ptr()), ws.numel(), None)
    assert rc == _lib.QSSB_ERR_INVALID
    assert nbytes.value == 256  # no partial tiles without split K
