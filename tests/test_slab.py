"""Host logic of the z-slab decomposed solve (blaze_b200/slab.py) on CPU:
the driver (slab.solve), the slab bounds, LocalExchange and DistExchange over
gloo (world size 2), with a numpy stand-in for a rank's device work.

The stand-in solves a small Neumann pressure system in float64 with the
same structure as the device path: a pass is four red-black half-sweeps
over the slab and the BLZ_SLAB_HALO planes around it (the pass's dependency
cone: what it computes outside the slab is discarded), the residual is a sum
of per-tile partials in tile order, computed from p on the slab and one
plane around it only.  Decomposed over any number of ranks it must give the
whole-grid stand-in's pressure and sweep count bit for bit, which holds only
if every rank receives the right planes of the right buffer at the right
time.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from blaze_b200 import slab

ALIGN, HALO = slab.ALIGN, slab.HALO


def _half_sweep(x, b, colour, zoff, D):
    """Gauss-Seidel update of the cells of `colour` ((i + j + k) & 1, k the
    global plane) of sub-volume x (planes zoff ..), Neumann walls at the
    global grid's faces; neighbours beyond the sub-volume count as zero."""
    d, H, W = x.shape
    k = np.arange(d)[:, None, None] + zoff
    j = np.arange(H)[None, :, None]
    i = np.arange(W)[None, None, :]
    pad = np.pad(x, 1)
    s = np.zeros_like(x)
    n = np.zeros_like(x)
    for (dz, dy, dx), exists in (((0, 0, -1), i > 0), ((0, 0, 1), i < W - 1), ((0, -1, 0), j > 0),
                                 ((0, 1, 0), j < H - 1), ((-1, 0, 0), k > 0), ((1, 0, 0), k < D - 1)):
        nb = pad[1 + dz:1 + dz + d, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W]
        s = s + np.where(exists, nb, 0.0)
        n = n + exists
    upd = ((i + j + k) & 1) == colour
    x[...] = np.where(upd, (b + s) / n, x)


def _residual_tiles(p, b):
    """Per-tile (r^2, b^2) of r = b - A p (Neumann), tiles of ALIGN planes."""
    D, H, W = p.shape
    k = np.arange(D)[:, None, None]
    j = np.arange(H)[None, :, None]
    i = np.arange(W)[None, None, :]
    pad = np.pad(p, 1)
    ap = np.zeros_like(p)
    for (dz, dy, dx), exists in (((0, 0, -1), i > 0), ((0, 0, 1), i < W - 1), ((0, -1, 0), j > 0),
                                 ((0, 1, 0), j < H - 1), ((-1, 0, 0), k > 0), ((1, 0, 0), k < D - 1)):
        nb = pad[1 + dz:1 + dz + D, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W]
        ap = ap + np.where(exists, p - nb, 0.0)
    r = b - ap
    out = []
    for t in range(-(-D // ALIGN)):
        sl = slice(t * ALIGN, min((t + 1) * ALIGN, D))
        out += [float(np.sum(r[sl] ** 2)), float(np.sum(b[sl] ** 2))]
    return out


class NpRank:
    """A rank of the stand-in: whole-grid arrays per buffer and colour (the
    colour's cells are the valid ones), work restricted to planes [z0, z1)."""

    def __init__(self, b, p0, z0, z1):
        self.b, self.D = b, b.shape[0]
        self.z0, self.z1 = z0, z1
        D, H, W = b.shape
        par = (np.arange(D)[:, None, None] + np.arange(H)[None, :, None] + np.arange(W)[None, None, :]) & 1
        self.black = par == 1
        self.plane = H * W
        self._arr = {(buf, c): torch.from_numpy(p0.copy()) for buf in ("p", "q") for c in ("r", "b")}
        self.partials = torch.zeros(2 * (-(-D // ALIGN)), dtype=torch.float64)

    def read(self, buf, colour, a, b):
        return self._arr[(buf, colour)][a:b].reshape(-1).clone()

    def write(self, buf, colour, a, b, t):
        assert t.numel() == (b - a) * self.plane
        self._arr[(buf, colour)][a:b] = t.reshape(b - a, *self.b.shape[1:])

    def empty(self, a, b):
        return torch.empty((b - a) * self.plane, dtype=torch.float64)

    def whole(self, buf):
        return np.where(self.black, self._arr[(buf, "b")].numpy(), self._arr[(buf, "r")].numpy())

    def pass_(self, buf):
        out = "q" if buf == "p" else "p"
        lo, hi = max(self.z0 - HALO, 0), min(self.z1 + HALO, self.D)
        x = np.where(self.black[lo:hi], self._arr[(buf, "b")].numpy()[lo:hi], 0.0)
        for colour in (0, 1, 0, 1):
            _half_sweep(x, self.b[lo:hi], colour, lo, self.D)
        for c in ("r", "b"):
            self._arr[(out, c)].numpy()[self.z0:self.z1] = x[self.z0 - lo:self.z1 - lo]

    def residual(self):
        self.partials.zero_()
        lo, hi = max(self.z0 - 1, 0), min(self.z1 + 1, self.D)
        kk = np.arange(self.D)[:, None, None]
        pairs = _residual_tiles(np.where((kk < lo) | (kk >= hi), 0.0, self.whole("p")), self.b)
        for t in range(self.z0 // ALIGN, -(-self.z1 // ALIGN)):
            self.partials[2 * t] = pairs[2 * t]
            self.partials[2 * t + 1] = pairs[2 * t + 1]

    def reduce(self, partials):
        r2 = b2 = 0.0
        pv = partials.numpy()
        for t in range(len(pv) // 2):
            r2 += float(pv[2 * t])
            b2 += float(pv[2 * t + 1])
        return float(np.sqrt(r2)), float(np.sqrt(b2))


def _whole_grid_solve(b, p0, tol, max_iter, check_every):
    """The stand-in on one rank holding the whole grid."""
    r = NpRank(b, p0, 0, b.shape[0])
    st = slab.solve(slab.LocalExchange([r]), tol, max_iter, check_every)
    return r.whole("p"), st


def _problem(D=40, H=6, W=8, seed=5):
    rng = np.random.default_rng(seed)
    b = rng.standard_normal((D, H, W))
    b -= b.mean()                                   # compatible right side (Neumann)
    p0 = 0.1 * rng.standard_normal((D, H, W))
    return b, p0


def test_slab_bounds():
    assert slab.slab_bounds(256, 8) == [(32 * r, 32 * (r + 1)) for r in range(8)]
    assert slab.slab_bounds(40, 3) == [(0, 16), (16, 32), (32, 40)]
    assert slab.slab_bounds(33, 3) == [(0, 16), (16, 32), (32, 33)]
    assert slab.slab_bounds(40, 1) == [(0, 40)]
    for D in (16, 17, 40, 100, 256):
        for ws in range(1, -(-D // ALIGN) + 1):
            bd = slab.slab_bounds(D, ws)
            assert bd[0][0] == 0 and bd[-1][1] == D
            assert all(a[1] == c[0] for a, c in zip(bd, bd[1:]))
            assert all(z0 % ALIGN == 0 and z1 > z0 for z0, z1 in bd)
            assert all(z1 - z0 >= ALIGN for z0, z1 in bd[:-1])
    with pytest.raises(ValueError):
        slab.slab_bounds(40, 4)
    with pytest.raises(ValueError):
        slab.slab_bounds(40, 0)


def test_halo_ranges_match_between_neighbours():
    """What a slab sends its neighbour is exactly what that neighbour expects."""
    for D in (33, 40, 100):
        for ws in range(2, -(-D // ALIGN) + 1):
            bd = slab.slab_bounds(D, ws)
            for depth in (1, HALO):
                for r in range(ws - 1):
                    _, _, send_hi, recv_hi = slab._halo_ranges(*bd[r], D, depth, r > 0, True)
                    send_lo, recv_lo, _, _ = slab._halo_ranges(*bd[r + 1], D, depth, True, r + 2 < ws)
                    assert send_hi == recv_lo and recv_hi == send_lo


def test_solve_rejects_bad_interval():
    b, p0 = _problem()
    with pytest.raises(ValueError):
        slab.solve(slab.LocalExchange([NpRank(b, p0, 0, 40)]), 1e-3, 40, 6)
    with pytest.raises(ValueError):
        slab.solve(slab.LocalExchange([NpRank(b, p0, 0, 40)]), 1e-3, 42, 8)


@pytest.mark.parametrize("ws", [2, 3])
@pytest.mark.parametrize("D", [40, 33])
def test_local_exchange_equals_whole_grid(ws, D):
    b, p0 = _problem(D=D)
    want, st0 = _whole_grid_solve(b, p0, 0.05, 96, 8)
    ranks = [NpRank(b, p0, z0, z1) for z0, z1 in slab.slab_bounds(D, ws)]
    st = slab.solve(slab.LocalExchange(ranks), 0.05, 96, 8)
    assert st == st0
    assert 0 < st["iterations"] < 96                # stops at a check before the cap
    for r in ranks:
        assert np.array_equal(r.whole("p"), want)


def test_missing_exchange_is_detected():
    """A fault planted in the stand-in's exchange (halo planes not moved)
    must break the equality the tests rely on."""
    b, p0 = _problem()
    want, _ = _whole_grid_solve(b, p0, 0.0, 16, 8)

    class NoHalo(slab.LocalExchange):
        def halo(self, buf, colours, depth):
            pass

    ranks = [NpRank(b, p0, z0, z1) for z0, z1 in slab.slab_bounds(40, 2)]
    slab.solve(NoHalo(ranks), 0.0, 16, 8)
    assert not np.array_equal(ranks[0].whole("p"), want)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, ws, port, D, q):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        b, p0 = _problem(D=D)
        bounds = slab.slab_bounds(D, ws)
        r = NpRank(b, p0, *bounds[rank])
        st = slab.solve(slab.DistExchange(r, bounds), 0.05, 96, 8)
        q.put((rank, st, r.whole("p")))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("D", [40, 33])
def test_two_gloo_ranks_equal_whole_grid(D):
    ws = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, ws, port, D, q)) for r in range(ws)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(ws)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    b, p0 = _problem(D=D)
    want, st0 = _whole_grid_solve(b, p0, 0.05, 96, 8)
    for rank, st, p in got:
        assert st == st0
        assert np.array_equal(p, want)
