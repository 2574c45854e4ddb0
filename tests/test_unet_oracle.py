"""CPU checks of the warm-start network's oracle (no GPU): its backward pass
against central finite differences of its own FP64 forward, its layer table
against the library's, and its residual features against the C oracle."""
import numpy as np
import pytest

from oracle import unet_oracle as uo


def _grid(W, H, D, bc=1):
    from blaze_b200.scenes import SceneSettings
    s = SceneSettings(gridRes=(W, H, D), dx=1.0 / W, closedBounds=(1, 1, 1, 0, 1, 1), bc_mode=bc)
    return s.to_params()


def _params(seed):
    rng = np.random.default_rng(seed)
    lay, n = uo.layout()
    p = np.zeros(n)
    for name, (kind, cin, cout, taps, wo, bo) in lay.items():
        fan = taps * cin if kind != uo.UP else cin
        p[wo:bo] = rng.standard_normal(bo - wo) * np.sqrt(2.0 / fan)
        p[bo:bo + cout] = 0.1 * rng.standard_normal(cout)
    return p


def test_layer_table_matches_library():
    from blaze_b200 import unet
    lay, n = uo.layout()
    lib_layers = unet.layers()
    assert [L["name"] for L in lib_layers] == [name for name, *_ in uo.LAYERS]
    for L in lib_layers:
        assert lay[L["name"]] == (L["kind"], L["cin"], L["cout"], L["taps"], L["w_off"], L["b_off"])
    assert unet.num_params() == n


def test_backward_matches_finite_differences():
    W, H, D = 16, 8, 8
    g = _grid(W, H, D)
    rng = np.random.default_rng(5)
    rhs = rng.standard_normal((D, H, W)).astype(np.float32)
    p = (0.3 * rng.standard_normal((D, H, W))).astype(np.float32)
    pt = p + (0.1 * rng.standard_normal((D, H, W))).astype(np.float32)
    params = _params(11)
    args = (g, rhs, p, pt, (0, 0, 0), (W, H, D), 0.7)
    loss, _, grads, _ = uo.loss_and_grads(params, *args, bf16=False)
    lay, _ = uo.layout()
    pick = np.random.default_rng(7)
    for name, (kind, cin, cout, taps, wo, bo) in lay.items():
        for idx in list(pick.integers(wo, bo, 2)) + [bo]:
            h = 1e-6 * max(1.0, abs(params[idx]))
            pp, pm = params.copy(), params.copy()
            pp[idx] += h
            pm[idx] -= h
            fd = (uo.loss_and_grads(pp, *args, bf16=False)[0] - uo.loss_and_grads(pm, *args, bf16=False)[0]) / (2 * h)
            assert abs(fd - grads[idx]) <= 1e-5 * max(abs(fd), 1e-3 * loss), (name, idx, fd, grads[idx])


@pytest.mark.parametrize("bc", [0, 1])
def test_residual_features_match_c_oracle(bc):
    from oracle import oracle
    W, H, D = 16, 12, 10
    g = _grid(W, H, D, bc)
    rng = np.random.default_rng(3)
    rhs = rng.standard_normal((D, H, W)).astype(np.float32)
    p = rng.standard_normal((D, H, W)).astype(np.float32)
    b, pc, r = uo.residual_parts(g, rhs, p)
    st = oracle.State(g, np.float64)
    st.RHS[...] = rhs
    st.P[...] = p
    rn, bn = st.residual_norms()
    assert np.isclose(np.linalg.norm(r.astype(np.float64)), rn, rtol=1e-5)
    assert np.isclose(np.linalg.norm(b.astype(np.float64)), bn, rtol=1e-6)


def test_neumann_channel():
    W, H, D = 8, 8, 8
    g = _grid(W, H, D, bc=1)                     # walls except the top (j = 0 side)
    z = np.zeros((D, H, W), np.float32)
    x = uo.input_tensor(g, z, z, (0, 0, 0), (W, H, D), 1.0)
    neu = x[..., 1]
    assert neu[1:-1, 0, 1:-1].max() == 0.0       # free-surface ghosts above the top
    assert neu[1:-1, -1, 1:-1].min() == 1.0      # floor
    assert neu[0].min() == 1.0 and neu[:, :, 0].min() == 1.0
    assert neu[1:-1, 1:-1, 1:-1].max() == 0.0    # interior
    g0 = _grid(W, H, D, bc=0)                    # no Dirichlet ghost: every face is Neumann
    x0 = uo.input_tensor(g0, z, z, (0, 0, 0), (W, H, D), 1.0)
    assert x0[1:-1, 0, 1:-1, 1].min() == 1.0
