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
    ((33, 17, 3), 16, 128, False), ((64, 64, 2), 64, 16, True),
    # the z-marching kernel (cin, cout in {16, 32}, BF16 out): several z slabs, ragged tiles
    ((37, 11, 21), 32, 32, True), ((24, 8, 17), 32, 16, False), ((19, 13, 33), 16, 32, True),
    ((5, 3, 1), 16, 16, True)])
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


# ---------------------------------------------------------------------------
# The whole warm-start network against the FP64 oracle with BF16 rounding
# emulated at the GPU's storage points (oracle/unet_oracle.py).  Each
# operation matches the oracle to BF16 rounding on identical inputs
# (test_gpu_unet_ops.py); end to end, the rare rounding flips that FP32
# versus FP64 accumulation causes compound through 14 layers and flip ReLU
# masks downstream, so the bounds here are relative L2 2e-2 on the output
# and 5e-2 on the whole gradient vector.
# ---------------------------------------------------------------------------
def _grid(W, H, D, bc=1):
    from blaze_b200.scenes import SceneSettings
    return SceneSettings(gridRes=(W, H, D), dx=1.0 / W, closedBounds=(1, 1, 1, 0, 1, 1), bc_mode=bc).to_params()


def _net_params(seed):
    from oracle import unet_oracle as uo
    rng = np.random.default_rng(seed)
    lay, n = uo.layout()
    p = np.zeros(n, np.float32)
    for name, (kind, cin, cout, taps, wo, bo) in lay.items():
        fan = taps * cin if kind != uo.UP else cin
        p[wo:bo] = rng.standard_normal(bo - wo) * np.sqrt(2.0 / fan)
        p[bo:bo + cout] = 0.05 * rng.standard_normal(cout)
    return p


def _fields(W, H, D, seed):
    rng = np.random.default_rng(seed)
    rhs = rng.standard_normal((D, H, W)).astype(np.float32)
    p = (0.5 * rng.standard_normal((D, H, W))).astype(np.float32)
    pt = p + (0.2 * rng.standard_normal((D, H, W))).astype(np.float32)
    return rhs, p, pt


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("grid_dims,crop,origin,bc", [
    ((16, 16, 16), (16, 16, 16), (0, 0, 0), 1),
    ((24, 16, 16), (16, 8, 16), (8, 4, 0), 1),
    ((16, 16, 24), (16, 16, 16), (0, 0, 8), 0)])
def test_unet_forward_matches_oracle(grid_dims, crop, origin, bc):
    import torch
    from oracle import unet_oracle as uo
    from blaze_b200.unet import WarmStartUNet
    W, H, D = grid_dims
    g = _grid(W, H, D, bc)
    rhs, p, _ = _fields(W, H, D, 1)
    params = _net_params(2)
    net = WarmStartUNet(crop, params, kappa=0.8)
    got = net.forward(g, torch.from_numpy(rhs).cuda(), torch.from_numpy(p).cuda(), origin).cpu().numpy()
    want = uo.forward(params, g, rhs, p, origin, crop, 0.8)
    assert _rel(got, want) <= 2e-2, _rel(got, want)
    net.close()


def test_unet_gradients_match_oracle():
    import torch
    from oracle import unet_oracle as uo
    from blaze_b200.unet import WarmStartUNet
    W, H, D = 32, 32, 32
    g = _grid(W, H, D)
    rhs, p, pt = _fields(W, H, D, 3)
    params = _net_params(4)
    net = WarmStartUNet((W, H, D), params, kappa=0.5)
    dev = lambda a: torch.from_numpy(a).cuda()
    loss, t2 = net.loss_grad(g, dev(rhs), dev(p), dev(pt))
    got = net.get_grads()
    wl, wt2, want, _ = uo.loss_and_grads(params, g, rhs, p, pt, (0, 0, 0), (W, H, D), 0.5)
    assert abs(loss - wl) <= 1e-2 * wl and abs(t2 - wt2) <= 1e-5 * wt2, (loss, wl, t2, wt2)
    assert _rel(got, want) <= 5e-2, _rel(got, want)
    # Adam against the same update in FP64
    net.adam(1e-3)
    new = net.get_params()
    z = np.zeros_like(want)
    ref, _, _ = uo.adam(params.astype(np.float64), got.astype(np.float64), z, z, 1, 1e-3)
    assert np.abs(new - ref).max() <= 1e-6, np.abs(new - ref).max()
    net.close()


def test_unet_training_lowers_the_loss():
    import torch
    from blaze_b200.unet import WarmStartUNet, init_params
    W, H, D = 16, 16, 16
    g = _grid(W, H, D)
    rhs, p, pt = _fields(W, H, D, 5)
    net = WarmStartUNet((W, H, D), init_params(0))
    dev = lambda a: torch.from_numpy(a).cuda()
    r, pp, tt = dev(rhs), dev(p), dev(pt)
    first = net.loss_grad(g, r, pp, tt)[0]
    for _ in range(40):
        net.adam(2e-3)
        last = net.loss_grad(g, r, pp, tt)[0]
    assert last < 0.5 * first, (first, last)
    net.close()


@pytest.mark.parametrize("mode", ["residual", "energy"])
def test_warm_start_through_the_solver(mode):
    """Without smoothing, blz_solve with a network attached starts from
    p + alpha d, d = kappa rms(r) delta, with alpha = <r, A d> / <A d, A d>
    (residual-norm step) or <d, r> / <d, A d> (energy-norm step)."""
    import torch
    from oracle import unet_oracle as uo
    from blaze_b200 import FluidSolver, Timer, _abi
    from blaze_b200.scenes import SceneSettings
    from blaze_b200.unet import WarmStartUNet
    W, H, D = 16, 16, 16
    scn = SceneSettings(gridRes=(W, H, D), dx=1.0 / W, closedBounds=(1, 1, 1, 0, 1, 1), bc_mode=1,
                        maxIterSolve=0, tol=0.0, device_loop=0)
    rhs, p, _ = _fields(W, H, D, 7)
    params = _net_params(8)
    net = WarmStartUNet((W, H, D), params, kappa=0.6)
    net.set_smoothing(0)
    net.set_step(_abi.BLZ_WARM_STEP_RESIDUAL if mode == "residual" else _abi.BLZ_WARM_STEP_ENERGY)
    g = scn.to_params()
    delta = net.forward(g, torch.from_numpy(rhs).cuda(), torch.from_numpy(p).cuda()).cpu().numpy()
    so = uo.scales(g, rhs, p, 0.6)[3]
    solver = FluidSolver(Timer(), scn)
    solver.set("RHS", rhs)
    solver.set("P", p)
    solver.set_warm_start(net)
    st = solver.solve()
    assert st["warm_started"] == 1 and st["ms_warm_start"] > 0.0 and st["iterations"] == 0
    got = solver.get("P")
    d = float(so) * delta.astype(np.float64)
    _, _, r = uo.residual_parts(g, rhs, p)
    Ad = -uo.residual_parts(g, np.zeros_like(rhs), d.astype(np.float32))[2].astype(np.float64)
    r = r.astype(np.float64)
    alpha = float(np.sum(r * Ad) / np.sum(Ad * Ad)) if mode == "residual" else float(np.sum(d * r) / np.sum(d * Ad))
    assert abs(net.last_alpha() - alpha) <= 1e-4 * abs(alpha), (net.last_alpha(), alpha)
    want = p.astype(np.float64) + net.last_alpha() * d
    assert np.abs(got - want).max() <= 1e-5 * np.abs(want - p).max() + 1e-6
    solver.set_warm_start(None)
    solver.set("P", p)
    st = solver.solve()
    assert st["warm_started"] == 0 and np.array_equal(solver.get("P"), p)
    solver.close()
    net.close()


def test_smoothed_warm_start_never_raises_the_residual():
    """With k smoothing sweeps and the residual-norm step the warm start's
    residual is at most that of k plain sweeps from the same pressure
    (alpha = 0 is among the choices)."""
    from blaze_b200 import FluidSolver, Timer
    from blaze_b200.scenes import SceneSettings
    from blaze_b200.unet import WarmStartUNet
    W, H, D = 32, 32, 32
    scn = SceneSettings(gridRes=(W, H, D), dx=1.0 / W, closedBounds=(1, 1, 1, 0, 1, 1), bc_mode=1,
                        maxIterSolve=0, tol=0.0, device_loop=0)
    rhs, p, _ = _fields(W, H, D, 9)
    from blaze_b200 import _abi
    net = WarmStartUNet((W, H, D), _net_params(10), kappa=0.6)
    net.set_smoothing(40)
    net.set_step(_abi.BLZ_WARM_STEP_RESIDUAL)
    out = []
    for warm in (False, True):
        solver = FluidSolver(Timer(), scn)
        solver.set("RHS", rhs)
        solver.set("P", p)
        if warm:
            solver.set_warm_start(net)
            st = solver.solve()
            assert st["iterations"] == 40 and st["warm_started"] == 1
        else:
            solver.sweeps(40)
        out.append(solver.residual()[0])
        solver.close()
    assert out[1] <= out[0] * (1 + 1e-6), out
    net.close()


def test_unet_rejects_bad_arguments():
    import ctypes as C
    from blaze_b200 import _lib
    lib = _lib.load()
    h = C.c_void_p()
    assert lib.blz_unet_create(12, 16, 16, C.byref(h)) == -2
    assert lib.blz_unet_create(16, 16, 16, C.byref(h)) == 0
    g = _grid(16, 16, 16)
    org = (C.c_int * 3)(8, 0, 0)
    buf = C.c_void_p(1)
    assert lib.blz_unet_forward(h, C.byref(g), org, buf, buf, buf, None) == -2     # crop leaves the grid
    assert lib.blz_unet_get_grads(h, buf, 1) == -7                                 # no gradients yet
    lib.blz_unet_destroy(h)
