"""Every operation of the warm-start network's forward and backward pass
against the FP64 oracle (oracle/unet_oracle.py), each fed with the GPU's own
BF16 input tensors (read back through blz_unet_get_tensor).

Fed identical inputs, an operation differs from the oracle only by FP32
(tensor memory / atomics) versus FP64 accumulation and, for BF16 outputs, by
the rare element whose rounding flips because of it:
  BF16 outputs   relative L2 <= 2e-3   (a flip is one BF16 ulp, 2^-8 relative)
  FP32 gradients relative L2 <= 1e-4
End to end, flips compound through 14 layers, so the whole-network
comparison (test_gpu_unet.py) uses looser bounds.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BF16_TOL = 2e-3
F32_TOL = 1e-4


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def _inner(t):
    return t[1:-1, 1:-1, 1:-1]


@pytest.fixture(scope="module")
def run():
    import torch
    from blaze_b200.scenes import SceneSettings
    from blaze_b200.unet import TENSOR_NAMES, WarmStartUNet
    from oracle import unet_oracle as uo
    W, H, D = 32, 16, 16
    g = SceneSettings(gridRes=(W, H, D), dx=1.0 / W, closedBounds=(1, 1, 1, 0, 1, 1), bc_mode=1).to_params()
    rng = np.random.default_rng(21)
    rhs = rng.standard_normal((D, H, W)).astype(np.float32)
    p = (0.5 * rng.standard_normal((D, H, W))).astype(np.float32)
    pt = p + (0.2 * rng.standard_normal((D, H, W))).astype(np.float32)
    lay, n = uo.layout()
    params = np.zeros(n, np.float32)
    for name, (kind, cin, cout, taps, wo, bo) in lay.items():
        fan = taps * cin if kind != uo.UP else cin
        params[wo:bo] = rng.standard_normal(bo - wo) * np.sqrt(2.0 / fan)
        params[bo:bo + cout] = 0.05 * rng.standard_normal(cout)
    net = WarmStartUNet((W, H, D), params, kappa=0.7)
    dev = lambda a: torch.from_numpy(a).cuda()
    loss, t2 = net.loss_grad(g, dev(rhs), dev(p), dev(pt))
    T = {name: net.tensor(name).astype(np.float64) for name in TENSOR_NAMES}
    out = {"grid": g, "rhs": rhs, "p": p, "pt": pt, "params": params, "loss": loss, "T": T,
           "grads": net.get_grads().astype(np.float64), "dims": (W, H, D)}
    net.close()
    return out


def _weights(params):
    from oracle import unet_oracle as uo
    W, B = uo.unpack(params)
    for name, kind, *_ in uo.LAYERS:
        if kind in (uo.CONV3, uo.UP):
            W[name] = uo.bf16_round(W[name])
    return W, B


def test_input_tensor(run):
    from oracle import unet_oracle as uo
    want = uo.input_tensor(run["grid"], run["rhs"], run["p"], (0, 0, 0), run["dims"], 0.7)
    assert _rel(run["T"]["X0"], want) <= BF16_TOL


# (layer, input tensor, output tensor, output channel slice)
FWD_CONV = [("e0a", "X0", "e0a", None), ("e0b", "e0a", "cat0", (16, 32)), ("e1a", "p1", "e1a", None),
            ("e1b", "e1a", "cat1", (32, 64)), ("e2a", "p2", "e2a", None), ("e2b", "e2a", "cat2", (64, 128)),
            ("e3a", "p3", "e3a", None), ("e3b", "e3a", "e3b", None), ("d2a", "cat2", "d2a", None),
            ("d2b", "d2a", "d2b", None), ("d1a", "cat1", "d1a", None), ("d1b", "d1a", "d1b", None),
            ("d0a", "cat0", "d0a", None), ("d0b", "d0a", "d0b", None)]


@pytest.mark.parametrize("layer,src,dst,sl", FWD_CONV, ids=[f[0] for f in FWD_CONV])
def test_forward_conv(run, layer, src, dst, sl):
    from oracle import unet_oracle as uo
    W, B = _weights(run["params"])
    want = uo.bf16_round(np.maximum(uo.conv3(run["T"][src], W[layer], B[layer]), 0.0))
    got = _inner(run["T"][dst])
    if sl:
        got = got[..., sl[0]:sl[1]]
    assert _rel(got, want) <= BF16_TOL


@pytest.mark.parametrize("src,c0,c1,dst", [("cat0", 16, 32, "p1"), ("cat1", 32, 64, "p2"), ("cat2", 64, 128, "p3")])
def test_pool(run, src, c0, c1, dst):
    from oracle import unet_oracle as uo
    want = uo.bf16_round(uo.pool2(_inner(run["T"][src])[..., c0:c1]))
    assert _rel(_inner(run["T"][dst]), want) <= BF16_TOL


@pytest.mark.parametrize("layer,src,dst,C", [("u2", "e3b", "cat2", 64), ("u1", "d2b", "cat1", 32),
                                             ("u0", "d1b", "cat0", 16)])
def test_upconv(run, layer, src, dst, C):
    from oracle import unet_oracle as uo
    W, B = _weights(run["params"])
    want = uo.bf16_round(uo.upconv(_inner(run["T"][src]), W[layer], B[layer]))
    assert _rel(_inner(run["T"][dst])[..., :C], want) <= BF16_TOL


def _head(run):
    """Head output, target and dL/dout from the GPU's d0b."""
    from oracle import unet_oracle as uo
    W, B = _weights(run["params"])
    out = _inner(run["T"]["d0b"]) @ W["head"][0, 0] + B["head"][0]
    so = uo.scales(run["grid"], run["rhs"], run["p"], 0.7)[3]
    tgt = ((run["pt"] - run["p"]) / so).astype(np.float64)
    return out, tgt, 2.0 * (out - tgt) / out.size


def test_loss_and_head(run):
    from oracle import unet_oracle as uo
    out, tgt, gout = _head(run)
    assert abs(run["loss"] - np.mean((out - tgt) ** 2)) <= 1e-5 * run["loss"]
    lay, _ = uo.layout()
    _, _, _, _, wo, bo = lay["head"]
    assert _rel(run["grads"][wo:bo], np.tensordot(gout, _inner(run["T"]["d0b"]), axes=3)) <= F32_TOL
    assert _rel(run["grads"][bo:bo + 1], [gout.sum()]) <= F32_TOL
    W, _ = _weights(run["params"])
    d0b = _inner(run["T"]["d0b"])
    want = uo.bf16_round(gout[..., None] * W["head"][0, 0] * (d0b > 0))
    assert _rel(_inner(run["T"]["g_d0b"]), want) <= BF16_TOL


# (layer, input, pre-activation gradient, data-gradient output, ReLU mask of it)
BWD_CONV = [("d0b", "d0a", "g_d0b", "g_d0a", "d0a"), ("d0a", "cat0", "g_d0a", "g_cat0", None),
            ("d1b", "d1a", "g_d1b", "g_d1a", "d1a"), ("d1a", "cat1", "g_d1a", "g_cat1", None),
            ("d2b", "d2a", "g_d2b", "g_d2a", "d2a"), ("d2a", "cat2", "g_d2a", "g_cat2", None),
            ("e3b", "e3a", "g_e3b", "g_e3a", "e3a"), ("e3a", "p3", "g_e3a", "g_p3", None),
            ("e2b", "e2a", "g_e2b", "g_e2a", "e2a"), ("e2a", "p2", "g_e2a", "g_p2", None),
            ("e1b", "e1a", "g_e1b", "g_e1a", "e1a"), ("e1a", "p1", "g_e1a", "g_p1", None),
            ("e0b", "e0a", "g_e0b", "g_e0a", "e0a"), ("e0a", "X0", "g_e0a", None, None)]


@pytest.mark.parametrize("layer,src,gy,gx,mask", BWD_CONV, ids=[b[0] for b in BWD_CONV])
def test_backward_conv(run, layer, src, gy, gx, mask):
    from oracle import unet_oracle as uo
    W, _ = _weights(run["params"])
    dw, db, dx = uo.conv3_back(run["T"][src], _inner(run["T"][gy]), W[layer])
    lay, _ = uo.layout()
    kind, cin, cout, taps, wo, bo = lay[layer]
    assert _rel(run["grads"][wo:bo], dw.reshape(-1)) <= F32_TOL
    assert _rel(run["grads"][bo:bo + cout], db) <= F32_TOL
    if gx:
        want = dx * (_inner(run["T"][mask]) > 0) if mask else dx
        assert _rel(_inner(run["T"][gx]), uo.bf16_round(want)) <= BF16_TOL


@pytest.mark.parametrize("layer,src,gcat,C,gx", [("u0", "d1b", "g_cat0", 16, "g_d1b"),
                                                 ("u1", "d2b", "g_cat1", 32, "g_d2b"),
                                                 ("u2", "e3b", "g_cat2", 64, "g_e3b")])
def test_backward_upconv(run, layer, src, gcat, C, gx):
    from oracle import unet_oracle as uo
    W, _ = _weights(run["params"])
    x = _inner(run["T"][src])
    dw, db, dx = uo.upconv_back(x, _inner(run["T"][gcat])[..., :C], W[layer])
    lay, _ = uo.layout()
    kind, cin, cout, taps, wo, bo = lay[layer]
    assert _rel(run["grads"][wo:bo], dw.reshape(-1)) <= F32_TOL
    assert _rel(run["grads"][bo:bo + cout], db) <= F32_TOL
    assert _rel(_inner(run["T"][gx]), uo.bf16_round(dx * (x > 0))) <= BF16_TOL


@pytest.mark.parametrize("gcat,cat,C,gpool,out", [("g_cat2", "cat2", 64, "g_p3", "g_e2b"),
                                                  ("g_cat1", "cat1", 32, "g_p2", "g_e1b"),
                                                  ("g_cat0", "cat0", 16, "g_p1", "g_e0b")])
def test_skip_gradient(run, gcat, cat, C, gpool, out):
    from oracle import unet_oracle as uo
    T = run["T"]
    want = (_inner(T[gcat])[..., C:] + uo.pool2_back(_inner(T[gpool]))) * (_inner(T[cat])[..., C:] > 0)
    assert _rel(_inner(T[out]), uo.bf16_round(want)) <= BF16_TOL
