"""Tensor-core building blocks of the learned warm start against a float64
torch reference on the CPU (floating-point kernels: the reference is the same
operation in FP64 on the BF16-rounded operands).

Tolerance: FP32-accumulated output relative L2 <= 1e-5 and max-abs <=
1e-4 * max|ref|; BF16 output <= 8e-3 (one BF16 rounding of the result).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SLACK = 256


def padded(x, dtype=None):
    """Device tensor in the halo layout; returns (buffer, interior view)."""
    import torch
    D, H, W, Cc = x.shape
    n = (D + 2) * (H + 2) * (W + 2)
    buf = torch.zeros(2 * SLACK + n, Cc, dtype=dtype or x.dtype, device="cuda")
    view = buf[SLACK:SLACK + n].view(D + 2, H + 2, W + 2, Cc)
    view[1:-1, 1:-1, 1:-1] = x
    return buf, view


def conv_ref(x, w, b, relu):
    import torch
    y = torch.nn.functional.conv3d(x.double().cpu().permute(3, 0, 1, 2)[None],
                                   w.double().cpu(), b.double().cpu(), padding=1)[0].permute(1, 2, 3, 0)
    return torch.relu(y) if relu else y


@pytest.mark.parametrize("shape,cin,cout,relu", [
    ((20, 9, 5), 16, 16, False), ((130, 6, 4), 32, 64, True), ((8, 8, 8), 48, 32, True),
    ((33, 17, 3), 16, 128, False), ((64, 64, 2), 64, 16, True)])
@pytest.mark.parametrize("out_f32", [1, 0], ids=["f32", "bf16"])
def test_conv3d_tensor_cores(shape, cin, cout, relu, out_f32):
    import torch
    from blaze_b200 import _lib
    lib = _lib.load()
    from blaze_b200._abi import BlzConvDesc
    W, H, D = shape
    g = torch.Generator().manual_seed(cin * 1000 + cout + W)
    x = torch.randn(D, H, W, cin, generator=g).to(torch.bfloat16).cuda()
    w = (torch.randn(cout, cin, 3, 3, 3, generator=g) / (27 * cin) ** 0.5).to(torch.bfloat16)
    b = torch.randn(cout, generator=g).float()
    xb, _ = padded(x)
    ob = torch.float32 if out_f32 else torch.bfloat16
    yb, yv = padded(torch.zeros(D, H, W, cout, dtype=ob, device="cuda"))
    w_dev = w.permute(2, 3, 4, 0, 1).reshape(27, cout, cin).contiguous().cuda()
    b_dev = b.cuda()
    d = BlzConvDesc(W, H, D, cin, cout, int(relu), out_f32)
    rc = lib.blz_conv3d(C.byref(d), C.c_void_p(xb[SLACK:].data_ptr()), C.c_void_p(w_dev.data_ptr()),
                        C.cast(C.c_void_p(b_dev.data_ptr()), C.POINTER(C.c_float)),
                        C.c_void_p(yb[SLACK:].data_ptr()), None)
    assert rc == 0, lib.blz_last_error(None)
    got = yv[1:-1, 1:-1, 1:-1].double().cpu()
    want = conv_ref(x, w, b, relu)
    err = (got - want).norm() / want.norm()
    mx = (got - want).abs().max() / want.abs().max()
    tol = (1e-5, 1e-4) if out_f32 else (8e-3, 8e-3)
    assert err <= tol[0] and mx <= tol[1], (float(err), float(mx))
    # the halo stays zero
    assert float(yv[0].abs().max()) == 0.0 and float(yv[:, :, 0].abs().max()) == 0.0
