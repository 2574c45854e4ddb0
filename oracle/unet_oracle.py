"""CPU restatement of the learned warm start's network (numpy, FP64).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the CUDA
network (csrc/unet.cu, csrc/unet_conv.cu); never by the product path.

The reference has no learned components: the architecture restated here is
the one the warm start defines (4-level 3-D U-Net, channels 16/32/64/128, two
3x3x3 convolutions + ReLU per level, 2x2x2 average pooling, 2x2x2 stride-2
transposed convolutions, concat [upsampled, skip], a 1x1x1 head), and the
solver operator it reads (the residual r = b - A p) is the pressure system of
the reference's Gauss-Seidel solve (src/FluidSolver.cu:517-599) with the
boundary handling of blz_params (walls; free-surface p = 0 ghosts).

With ``bf16=True`` every tensor the GPU stores in BF16 (input, activations,
activation gradients) and the 3x3x3 and transposed-convolution weights (the
GPU's forward passes and data gradients read BF16 copies of them) are
rounded to BF16 (round to nearest even) at the same points, so the only
remaining difference to the GPU is the FP32-vs-FP64 accumulation order.  With ``bf16=False`` it is the
plain FP64 network, used for the finite-difference check of the backward
pass.  Arrays are numpy (z, y, x[, c]).
"""
import numpy as np

CONV3, UP, HEAD = 0, 1, 2
# (name, kind, cin, cout, level): level of the output (fine level for UP)
LAYERS = [
    ("e0a", CONV3, 16, 16, 0), ("e0b", CONV3, 16, 16, 0), ("e1a", CONV3, 16, 32, 1), ("e1b", CONV3, 32, 32, 1),
    ("e2a", CONV3, 32, 64, 2), ("e2b", CONV3, 64, 64, 2), ("e3a", CONV3, 64, 128, 3), ("e3b", CONV3, 128, 128, 3),
    ("d2a", CONV3, 128, 64, 2), ("d2b", CONV3, 64, 64, 2), ("d1a", CONV3, 64, 32, 1), ("d1b", CONV3, 32, 32, 1),
    ("d0a", CONV3, 32, 16, 0), ("d0b", CONV3, 16, 16, 0),
    ("u2", UP, 128, 64, 2), ("u1", UP, 64, 32, 1), ("u0", UP, 32, 16, 0),
    ("head", HEAD, 16, 1, 0)]
TAPS = {CONV3: 27, UP: 8, HEAD: 1}


def layout():
    """{name: (kind, cin, cout, taps, w_off, b_off)} of the flat parameter array."""
    out, off = {}, 0
    for name, kind, cin, cout, _ in LAYERS:
        wn = TAPS[kind] * cout * cin
        out[name] = (kind, cin, cout, TAPS[kind], off, off + wn)
        off += wn + cout
    return out, off


def unpack(params):
    lay, _ = layout()
    W, B = {}, {}
    for name, (kind, cin, cout, taps, wo, bo) in lay.items():
        W[name] = np.asarray(params[wo:wo + taps * cout * cin], np.float64).reshape(taps, cout, cin)
        B[name] = np.asarray(params[bo:bo + cout], np.float64)
    return W, B


def bf16_round(x):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


# ---------------------------------------------------------------------------
# Input features
# ---------------------------------------------------------------------------
def open_faces(params):
    cb = list(params.closed_bounds)
    # OpenFaces order (xlo, xhi, ylo, yhi, zlo, zhi); grid j = 0 is the world
    # top, so world yMax (index 3) is the j = 0 side.
    return (not cb[0], not cb[1], not cb[3], not cb[2], not cb[4], not cb[5])


def residual_parts(params, rhs, p):
    """b, p and r = b - A p per cell in FP32 in the solver's order (A p = sum
    over in-domain neighbours of p - p_nb, plus p per Dirichlet ghost)."""
    f32 = np.float32
    scale = f32(params.density) * f32(params.dx) * f32(params.dx) / f32(params.dt)
    rhs = np.asarray(rhs, f32)
    p = np.asarray(p, f32)
    b = scale * rhs
    dirichlet = params.bc_mode == 1
    o = open_faces(params)
    D, H, W = p.shape
    ap = np.zeros_like(p)
    ghost = f32(1) if dirichlet else f32(0)
    # (axis, side, open flag): x-, x+, y-, y+, z-, z+ in that order
    for axis, side, op in ((2, -1, o[0]), (2, 1, o[1]), (1, -1, o[2]), (1, 1, o[3]), (0, -1, o[4]), (0, 1, o[5])):
        nb = np.roll(p, -side, axis=axis)
        d = p - nb
        edge = [slice(None)] * 3
        edge[axis] = 0 if side < 0 else p.shape[axis] - 1
        d[tuple(edge)] = p[tuple(edge)] * (ghost if op else f32(0))
        ap = ap + d
    return b, p, b - ap


def scales(params, rhs, p, kappa):
    b, pc, r = residual_parts(params, rhs, p)
    n = float(b.size)
    rms = [np.sqrt(np.sum(a.astype(np.float64) ** 2) / n) for a in (b, pc, r)]
    inv = [np.float32(1.0 / v) if v > 0 else np.float32(0) for v in rms]
    return inv[0], inv[1], inv[2], np.float32(kappa * rms[2])


def input_tensor(params, rhs, p, origin, dims, kappa, bf16=True):
    """The 16-channel padded input of the crop [origin, origin + dims) (W, H, D)."""
    b, pc, r = residual_parts(params, rhs, p)
    sb, sp, sr, _ = scales(params, rhs, p, kappa)
    Wc, Hc, Dc = dims
    ox, oy, oz = origin
    D, H, W = pc.shape
    x = np.zeros((Dc + 2, Hc + 2, Wc + 2, 16), np.float32)
    feats = np.stack([b * sb, np.zeros_like(b), pc * sp, r * sr], axis=-1).astype(np.float32)
    o = open_faces(params)
    dirichlet = params.bc_mode == 1
    zz, yy, xx = np.meshgrid(np.arange(oz - 1, oz + Dc + 1), np.arange(oy - 1, oy + Hc + 1),
                             np.arange(ox - 1, ox + Wc + 1), indexing="ij")
    inside = (xx >= 0) & (xx < W) & (yy >= 0) & (yy < H) & (zz >= 0) & (zz < D)
    x[inside, :4] = feats[zz[inside], yy[inside], xx[inside]]
    neu = np.zeros_like(inside)
    for cond, op in ((xx < 0, o[0]), (xx >= W, o[1]), (yy < 0, o[2]), (yy >= H, o[3]), (zz < 0, o[4]),
                     (zz >= D, o[5])):
        neu |= cond & (not (dirichlet and op))
    x[~inside, 1] = np.where(neu[~inside], 1.0, 0.0)
    x = x.astype(np.float64)
    return bf16_round(x) if bf16 else x


# ---------------------------------------------------------------------------
# Layers (padded tensors: (D+2, H+2, W+2, C) with a zero halo)
# ---------------------------------------------------------------------------
def pad(x):
    return np.pad(x, ((1, 1), (1, 1), (1, 1), (0, 0)))


def shifted(xp, t, shape):
    dz, dy, dx = t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1
    D, H, W = shape
    return xp[1 + dz:1 + dz + D, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W, :]


def conv3(xp, w, b):
    D, H, W = xp.shape[0] - 2, xp.shape[1] - 2, xp.shape[2] - 2
    y = np.broadcast_to(b, (D, H, W, w.shape[1])).copy()
    for t in range(27):
        y += shifted(xp, t, (D, H, W)) @ w[t].T
    return y


def conv3_back(xp, gy, w):
    """(dW, db, dx_interior) of y = conv3(xp, w, b)."""
    D, H, W = gy.shape[:3]
    g2 = gy.reshape(-1, gy.shape[3])
    dw = np.stack([g2.T @ shifted(xp, t, (D, H, W)).reshape(-1, xp.shape[3]) for t in range(27)])
    dxp = np.zeros(xp.shape)
    for t in range(27):
        dz, dy, dx = t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1
        dxp[1 + dz:1 + dz + D, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W, :] += gy @ w[t]
    return dw, gy.sum(axis=(0, 1, 2)), dxp[1:-1, 1:-1, 1:-1, :]


def pool2(x):
    D, H, W, Cc = x.shape
    return x.reshape(D // 2, 2, H // 2, 2, W // 2, 2, Cc).mean(axis=(1, 3, 5))


def pool2_back(g):
    return np.repeat(np.repeat(np.repeat(g, 2, 0), 2, 1), 2, 2) / 8.0


def upconv(x, w, b):
    D, H, W, _ = x.shape
    y = np.zeros((2 * D, 2 * H, 2 * W, w.shape[1]))
    for par in range(8):
        px, py, pz = par & 1, (par >> 1) & 1, par >> 2
        y[pz::2, py::2, px::2, :] = x @ w[par].T + b
    return y


def upconv_back(x, gy, w):
    dw = np.zeros_like(w)
    dx = np.zeros(x.shape)
    for par in range(8):
        px, py, pz = par & 1, (par >> 1) & 1, par >> 2
        g = gy[pz::2, py::2, px::2, :]
        dw[par] = g.reshape(-1, g.shape[3]).T @ x.reshape(-1, x.shape[3])
        dx += g @ w[par]
    return dw, gy.sum(axis=(0, 1, 2)), dx


# ---------------------------------------------------------------------------
# Network
# ---------------------------------------------------------------------------
class Net:
    def __init__(self, params, bf16=True):
        self.W, self.B = unpack(params)
        self.bf16 = bf16
        if bf16:
            for name, kind, *_ in LAYERS:
                if kind in (CONV3, UP):
                    self.W[name] = bf16_round(self.W[name])

    def r(self, a):
        return bf16_round(a) if self.bf16 else a

    def conv(self, name, x):
        return self.r(np.maximum(conv3(pad(x), self.W[name], self.B[name]), 0.0))

    def forward(self, x0p):
        """x0p: padded input (its halo is part of the input).  Returns the head
        output (D, H, W) and the cache for backward."""
        c = {"x0p": x0p}
        c["e0a"] = self.r(np.maximum(conv3(x0p, self.W["e0a"], self.B["e0a"]), 0.0))
        c["e0b"] = self.conv("e0b", c["e0a"])
        c["p1"] = self.r(pool2(c["e0b"]))
        c["e1a"] = self.conv("e1a", c["p1"])
        c["e1b"] = self.conv("e1b", c["e1a"])
        c["p2"] = self.r(pool2(c["e1b"]))
        c["e2a"] = self.conv("e2a", c["p2"])
        c["e2b"] = self.conv("e2b", c["e2a"])
        c["p3"] = self.r(pool2(c["e2b"]))
        c["e3a"] = self.conv("e3a", c["p3"])
        c["e3b"] = self.conv("e3b", c["e3a"])
        c["u2"] = self.r(upconv(c["e3b"], self.W["u2"], self.B["u2"]))
        c["cat2"] = np.concatenate([c["u2"], c["e2b"]], axis=-1)
        c["d2a"] = self.conv("d2a", c["cat2"])
        c["d2b"] = self.conv("d2b", c["d2a"])
        c["u1"] = self.r(upconv(c["d2b"], self.W["u1"], self.B["u1"]))
        c["cat1"] = np.concatenate([c["u1"], c["e1b"]], axis=-1)
        c["d1a"] = self.conv("d1a", c["cat1"])
        c["d1b"] = self.conv("d1b", c["d1a"])
        c["u0"] = self.r(upconv(c["d1b"], self.W["u0"], self.B["u0"]))
        c["cat0"] = np.concatenate([c["u0"], c["e0b"]], axis=-1)
        c["d0a"] = self.conv("d0a", c["cat0"])
        c["d0b"] = self.conv("d0b", c["d0a"])
        out = c["d0b"] @ self.W["head"][0, 0] + self.B["head"][0]
        return out, c

    def backward(self, c, gout):
        """Parameter gradients {name: (dW, db)} for dL/dout = gout."""
        G = {}
        mask = lambda a: (a > 0).astype(np.float64)
        G["head"] = ((np.tensordot(gout, c["d0b"], axes=3))[None, None, :], np.array([gout.sum()]))
        g = self.r(gout[..., None] * self.W["head"][0, 0] * mask(c["d0b"]))

        def conv_back(name, x, gy, act):
            dw, db, dx = conv3_back(pad(x), gy, self.W[name])
            G[name] = (dw, db)
            return self.r(dx * mask(act)) if act is not None else self.r(dx)

        def up_back(name, x, gy, C):
            dw, db, dx = upconv_back(x, gy[..., :C], self.W[name])
            G[name] = (dw, db)
            return self.r(dx * mask(x))

        g = conv_back("d0b", c["d0a"], g, c["d0a"])
        gcat0 = conv_back("d0a", c["cat0"], g, None)
        g = up_back("u0", c["d1b"], gcat0, 16)
        g = conv_back("d1b", c["d1a"], g, c["d1a"])
        gcat1 = conv_back("d1a", c["cat1"], g, None)
        g = up_back("u1", c["d2b"], gcat1, 32)
        g = conv_back("d2b", c["d2a"], g, c["d2a"])
        gcat2 = conv_back("d2a", c["cat2"], g, None)
        g = up_back("u2", c["e3b"], gcat2, 64)
        g = conv_back("e3b", c["e3a"], g, c["e3a"])
        gp3 = conv_back("e3a", c["p3"], g, None)
        g = self.r((gcat2[..., 64:] + pool2_back(gp3)) * mask(c["e2b"]))
        g = conv_back("e2b", c["e2a"], g, c["e2a"])
        gp2 = conv_back("e2a", c["p2"], g, None)
        g = self.r((gcat1[..., 32:] + pool2_back(gp2)) * mask(c["e1b"]))
        g = conv_back("e1b", c["e1a"], g, c["e1a"])
        gp1 = conv_back("e1a", c["p1"], g, None)
        g = self.r((gcat0[..., 16:] + pool2_back(gp1)) * mask(c["e0b"]))
        g = conv_back("e0b", c["e0a"], g, c["e0a"])
        dw, db, _ = conv3_back(c["x0p"], g, self.W["e0a"])
        G["e0a"] = (dw, db)
        return G


def flat_grads(G):
    lay, n = layout()
    out = np.zeros(n)
    for name, (kind, cin, cout, taps, wo, bo) in lay.items():
        dw, db = G[name]
        out[wo:wo + taps * cout * cin] = np.asarray(dw).reshape(-1)
        out[bo:bo + cout] = db
    return out


def loss_and_grads(params, grid, rhs, p, p_target, origin, dims, kappa, bf16=True):
    """(loss, mean target^2, flat gradients, network output) of one sample,
    as blz_unet_loss_grad defines them."""
    x0p = input_tensor(grid, rhs, p, origin, dims, kappa, bf16)
    net = Net(params, bf16)
    out, cache = net.forward(x0p)
    so = scales(grid, rhs, p, kappa)[3]
    Wc, Hc, Dc = dims
    ox, oy, oz = origin
    sl = (slice(oz, oz + Dc), slice(oy, oy + Hc), slice(ox, ox + Wc))
    dp = np.asarray(p_target, np.float32)[sl] - np.asarray(p, np.float32)[sl]
    tgt = (dp / so).astype(np.float64) if so > 0 else np.zeros(dp.shape)
    diff = out - tgt
    n = diff.size
    G = net.backward(cache, 2.0 * diff / n)
    return float(np.mean(diff ** 2)), float(np.mean(tgt ** 2)), flat_grads(G), out


def forward(params, grid, rhs, p, origin, dims, kappa, bf16=True):
    out, _ = Net(params, bf16).forward(input_tensor(grid, rhs, p, origin, dims, kappa, bf16))
    return out


def adam(params, grads, m, v, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One bias-corrected Adam step (t counts from 1); returns (params, m, v)."""
    m = b1 * m + (1 - b1) * grads
    v = b2 * v + (1 - b2) * grads * grads
    p = params - lr * (m / (1 - b1 ** t)) / (np.sqrt(v / (1 - b2 ** t)) + eps)
    return p, m, v
