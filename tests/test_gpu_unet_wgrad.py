"""Weight and bias gradients of every convolution and transposed convolution
of the warm-start network at 64 x 64 x 32, against the FP64 oracle
(oracle/unet_oracle.py), each fed with the GPU's own BF16 tensors.

At this size the tensor-core weight gradient splits each layer's voxels over
many CTAs, each accumulating several K blocks of 128 voxels in tensor memory
before its atomics, so the multi-block and multi-CTA paths run (the
32 x 16 x 16 case in test_gpu_unet_ops.py fits in one K block at the coarse
levels).  FP32 accumulation against FP64: relative L2 <= 1e-4.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

F32_TOL = 1e-4


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def _inner(t):
    return t[1:-1, 1:-1, 1:-1]


@pytest.fixture(scope="module")
def big():
    import torch
    from blaze_b200.scenes import SceneSettings
    from blaze_b200.unet import TENSOR_NAMES, WarmStartUNet
    from oracle import unet_oracle as uo
    W, H, D = 64, 64, 32
    g = SceneSettings(gridRes=(W, H, D), dx=1.0 / W, closedBounds=(1, 1, 1, 0, 1, 1), bc_mode=1).to_params()
    rng = np.random.default_rng(33)
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
    net.loss_grad(g, dev(rhs), dev(p), dev(pt))
    grads = net.get_grads().astype(np.float64)
    T = {name: net.tensor(name) for name in TENSOR_NAMES}
    net.close()
    W_, _ = uo.unpack(params)
    for name, kind, *_ in uo.LAYERS:
        if kind in (uo.CONV3, uo.UP):
            W_[name] = uo.bf16_round(W_[name])
    return {"T": T, "grads": grads, "W": W_}


CONV = [("d0b", "d0a", "g_d0b"), ("d0a", "cat0", "g_d0a"), ("d1b", "d1a", "g_d1b"), ("d1a", "cat1", "g_d1a"),
        ("d2b", "d2a", "g_d2b"), ("d2a", "cat2", "g_d2a"), ("e3b", "e3a", "g_e3b"), ("e3a", "p3", "g_e3a"),
        ("e2b", "e2a", "g_e2b"), ("e2a", "p2", "g_e2a"), ("e1b", "e1a", "g_e1b"), ("e1a", "p1", "g_e1a"),
        ("e0b", "e0a", "g_e0b"), ("e0a", "X0", "g_e0a")]


@pytest.mark.parametrize("layer,src,gy", CONV, ids=[c[0] for c in CONV])
def test_conv_weight_gradient_64(big, layer, src, gy):
    from oracle import unet_oracle as uo
    T = big["T"]
    dw, db, _ = uo.conv3_back(T[src].astype(np.float64), _inner(T[gy]).astype(np.float64), big["W"][layer])
    lay, _ = uo.layout()
    kind, cin, cout, taps, wo, bo = lay[layer]
    assert _rel(big["grads"][wo:bo], dw.reshape(-1)) <= F32_TOL
    assert _rel(big["grads"][bo:bo + cout], db) <= F32_TOL


@pytest.mark.parametrize("layer,src,gcat,C", [("u0", "d1b", "g_cat0", 16), ("u1", "d2b", "g_cat1", 32),
                                              ("u2", "e3b", "g_cat2", 64)])
def test_upconv_weight_gradient_64(big, layer, src, gcat, C):
    from oracle import unet_oracle as uo
    T = big["T"]
    dw, db, _ = uo.upconv_back(_inner(T[src]).astype(np.float64), _inner(T[gcat])[..., :C].astype(np.float64),
                               big["W"][layer])
    lay, _ = uo.layout()
    kind, cin, cout, taps, wo, bo = lay[layer]
    assert _rel(big["grads"][wo:bo], dw.reshape(-1)) <= F32_TOL
    assert _rel(big["grads"][bo:bo + cout], db) <= F32_TOL
