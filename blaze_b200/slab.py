"""Z-slab decomposition of one grid's pressure solve over ranks.

No counterpart in the reference, which solves the whole grid on one GPU
(src/FluidSolver.cu:517-599).  Every rank holds a FluidSolver of the whole
grid and runs the frame's other stages on the whole grid; only the solve,
most of a frame, is split.  Rank r updates the planes [z0, z1) of its slab,
whole residual tiles of BLZ_SLAB_ALIGN planes:

* a temporal-blocking pass (two red-black sweeps, blz_slab_pass) over a slab
  reads the black pressure BLZ_SLAB_HALO planes beyond it, so before each
  pass every rank receives those planes of its pass input from its
  neighbours;
* a residual check reads p one plane beyond the slab (both colours); each
  rank writes the FP64 partial sums of its tiles into a whole-grid array
  (blz_slab_residual), the arrays are summed over ranks (each entry comes
  from one rank, so the sum is exact) and reduced in the whole-grid order
  (blz_reduce_partials), and every rank takes the same decision;
* after the solve every rank gathers the whole pressure.

The same sweeps on the same planes and the same reduction order make the
decomposed solve bitwise equal to FluidSolver.solve on one GPU, sweep count
included (RB3D order, check interval a multiple of 4 dividing max_iter, no
defect correction).

Two exchanges move the planes: DistExchange (torch.distributed, one rank per
process and GPU: point-to-point plane transfers, an all-reduce of the
partials, one broadcast per slab) and LocalExchange (every rank's solver in
one process on one device).  Planes leave and enter a solver only through
copies (blz_slab_get_planes / blz_slab_set_planes) into ordinary torch
tensors.  A rank's state is a SlabRank over its solver; anything with the
same methods (tests use a numpy stand-in) runs under the same driver.
"""
import contextlib
import ctypes as C

from . import _abi
from ._lib import BlazeError, check

ALIGN = _abi.BLZ_SLAB_ALIGN
HALO = _abi.BLZ_SLAB_HALO
_BUF = {"p": 0, "q": 1}
_COLOUR = {"r": 0, "b": 1}


def slab_bounds(D, world):
    """[(z0, z1)] of each rank: the D planes' tiles of ALIGN planes split as
    evenly as possible (the last tile may be shorter).  Every slab is at
    least one tile; interior slabs are whole tiles, so each neighbour of a
    slab holds the HALO planes a pass reads beyond it (or the grid ends)."""
    tiles = -(-int(D) // ALIGN)
    if world < 1 or world > tiles:
        raise ValueError(f"{world} ranks for {D} planes: at most {tiles} (one tile of {ALIGN} planes each)")
    out = []
    for r in range(world):
        t0, t1 = r * tiles // world, (r + 1) * tiles // world
        out.append((t0 * ALIGN, min(t1 * ALIGN, int(D))))
    return out


class SlabRank:
    """One rank's solver and its slab.  The solver is moved to `stream` (a
    torch.cuda.Stream, a new one by default) and slab.solve runs the
    exchanges' copies and transfers on the same stream, so they are ordered
    with the solver's launches.  (torch's legacy default stream has handle 0,
    which the solver would replace by a stream of its own, unordered with
    torch's work.)"""

    def __init__(self, solver, z0, z1, stream=None):
        import torch
        self.solver, self.z0, self.z1 = solver, int(z0), int(z1)
        self.stream = stream if stream is not None else torch.cuda.Stream()
        if not self.stream.cuda_stream:
            raise ValueError("the slab solve needs a stream other than the legacy default stream")
        lib, h = solver._lib, solver._h
        self._lib, self._h = lib, h
        ok, npart, pf = C.c_int(), C.c_int(), C.c_longlong()
        check(lib.blz_slab_info(h, C.byref(ok), C.byref(npart), C.byref(pf)), h)
        if not ok.value:
            raise BlazeError(_abi.BLZ_ERR_STATE, "slab solve needs W % 8 == 0 with the temporal-blocking pass, "
                                                 "RB3D order and no defect correction")
        self.D = int(solver.params.dims()[2])
        if not (0 <= self.z0 < self.z1 <= self.D):
            raise ValueError(f"slab [{self.z0}, {self.z1}) of {self.D} planes")
        check(lib.blz_set_stream(h, C.c_void_p(self.stream.cuda_stream)), h)
        self.plane = int(pf.value)
        self.n_partials = int(npart.value)
        with torch.cuda.stream(self.stream):
            self.partials = torch.zeros(2 * self.n_partials, dtype=torch.float64, device="cuda")

    def read(self, buf, colour, a, b):
        """Planes [a, b) of colour 'r' or 'b' of buffer 'p' or 'q', copied
        into a new device tensor."""
        import torch
        t = torch.empty((b - a) * self.plane, dtype=torch.float32, device="cuda")
        check(self._lib.blz_slab_get_planes(self._h, _BUF[buf], _COLOUR[colour], a, b, C.c_void_p(t.data_ptr())),
              self._h)
        return t

    def write(self, buf, colour, a, b, t):
        """Copies device tensor t into planes [a, b) of (buf, colour)."""
        if t.numel() != (b - a) * self.plane:
            raise ValueError("plane count mismatch")
        check(self._lib.blz_slab_set_planes(self._h, _BUF[buf], _COLOUR[colour], a, b, C.c_void_p(t.data_ptr())),
              self._h)

    def empty(self, a, b):
        """A device tensor the size of planes [a, b) of one colour."""
        import torch
        return torch.empty((b - a) * self.plane, dtype=torch.float32, device="cuda")

    def pass_(self, buf):
        """One pass over the slab from buffer buf ('p' or 'q') into the other."""
        check(self._lib.blz_slab_pass(self._h, self.z0, self.z1, _BUF[buf]), self._h)

    def residual(self):
        """This slab's partial sums into self.partials (zero elsewhere)."""
        self.partials.zero_()
        first, count = C.c_int(), C.c_int()
        check(self._lib.blz_slab_residual(self._h, self.z0, self.z1, C.c_void_p(self.partials.data_ptr()),
                                          C.byref(first), C.byref(count)), self._h)

    def reduce(self, partials):
        """(||r||, ||b||) of a whole-grid partials array, whole-grid order."""
        r, b = C.c_double(), C.c_double()
        check(self._lib.blz_reduce_partials(self._h, C.c_void_p(partials.data_ptr()), C.byref(r), C.byref(b)),
              self._h)
        return r.value, b.value


def _halo_ranges(z0, z1, D, depth, lower, upper):
    """(send_lo, recv_lo, send_hi, recv_hi) plane ranges of a slab: the planes
    its lower / upper neighbour needs and the ones it receives from them
    (None where there is no neighbour)."""
    send_lo = (z0, min(z0 + depth, z1)) if lower else None
    recv_lo = (max(z0 - depth, 0), z0) if lower else None
    send_hi = (max(z1 - depth, z0), z1) if upper else None
    recv_hi = (z1, min(z1 + depth, D)) if upper else None
    return send_lo, recv_lo, send_hi, recv_hi


class LocalExchange:
    """All ranks in this process (one device); the moves are copies.  The
    ranks must share one stream (SlabRank(..., stream=s))."""

    def __init__(self, ranks):
        self.ranks = list(ranks)
        self.stream = getattr(self.ranks[0], "stream", None)
        if any(getattr(r, "stream", None) is not self.stream for r in self.ranks):
            raise ValueError("the ranks of a LocalExchange must share one stream")

    def halo(self, buf, colours, depth):
        rs = self.ranks
        for i, r in enumerate(rs):
            _, recv_lo, _, recv_hi = _halo_ranges(r.z0, r.z1, r.D, depth, i > 0, i + 1 < len(rs))
            for c in colours:
                if recv_lo:
                    r.write(buf, c, *recv_lo, rs[i - 1].read(buf, c, *recv_lo))
                if recv_hi:
                    r.write(buf, c, *recv_hi, rs[i + 1].read(buf, c, *recv_hi))

    def sum_partials(self):
        total = self.ranks[0].partials.clone()
        for r in self.ranks[1:]:
            total += r.partials
        return total

    def gather(self, buf="p"):
        for r in self.ranks:
            for o in self.ranks:
                if o is not r:
                    for c in ("r", "b"):
                        r.write(buf, c, o.z0, o.z1, o.read(buf, c, o.z0, o.z1))


class DistExchange:
    """One rank per process (torch.distributed, NCCL on GPUs): point-to-point
    plane transfers with the neighbours, an all-reduce of the partials,
    one broadcast per slab to gather the pressure.  Every rank takes the
    same collective steps in the same order."""

    def __init__(self, rank_state, bounds, group=None):
        import torch.distributed as dist
        self.dist, self.group = dist, group
        self.r = rank_state
        self.bounds = list(bounds)
        self.rank, self.world = dist.get_rank(group), dist.get_world_size(group)
        self.ranks = [rank_state]
        self.stream = getattr(rank_state, "stream", None)
        if self.bounds[self.rank] != (rank_state.z0, rank_state.z1):
            raise ValueError("the rank's slab differs from bounds[rank]")

    def _peer(self, i):
        return i if self.group is None else self.dist.get_global_rank(self.group, i)

    def halo(self, buf, colours, depth):
        dist, r = self.dist, self.r
        send_lo, recv_lo, send_hi, recv_hi = _halo_ranges(r.z0, r.z1, r.D, depth, self.rank > 0,
                                                          self.rank + 1 < self.world)
        ops, into = [], []
        for c in colours:
            if send_lo:
                t = r.empty(*recv_lo)
                ops.append(dist.P2POp(dist.isend, r.read(buf, c, *send_lo), self._peer(self.rank - 1), self.group))
                ops.append(dist.P2POp(dist.irecv, t, self._peer(self.rank - 1), self.group))
                into.append((c, recv_lo, t))
            if send_hi:
                t = r.empty(*recv_hi)
                ops.append(dist.P2POp(dist.isend, r.read(buf, c, *send_hi), self._peer(self.rank + 1), self.group))
                ops.append(dist.P2POp(dist.irecv, t, self._peer(self.rank + 1), self.group))
                into.append((c, recv_hi, t))
        if ops:
            for q in dist.batch_isend_irecv(ops):
                q.wait()
        for c, rng, t in into:
            r.write(buf, c, *rng, t)

    def sum_partials(self):
        total = self.r.partials.clone()
        self.dist.all_reduce(total, group=self.group)
        return total

    def gather(self, buf="p"):
        for i, (z0, z1) in enumerate(self.bounds):
            for c in ("r", "b"):
                t = self.r.read(buf, c, z0, z1) if i == self.rank else self.r.empty(z0, z1)
                self.dist.broadcast(t, self._peer(i), group=self.group)
                if i != self.rank:
                    self.r.write(buf, c, z0, z1, t)


def solve(exchange, tol, max_iter, check_every=20):
    """The residual-controlled RBGS solve over the exchange's ranks, with
    blz_solve's stopping rule: a check before the first sweep, then every
    check_every sweeps until ||r|| / ||b|| <= tol or max_iter sweeps.
    Leaves the whole pressure in every rank's p.  Returns the statistics."""
    if check_every % 4 or max_iter % check_every:
        raise ValueError("check_every must be a multiple of 4 dividing max_iter")
    stream = getattr(exchange, "stream", None)
    if stream is None:
        ctx = contextlib.nullcontext()
    else:
        import torch
        ctx = torch.cuda.stream(stream)
    with ctx:
        return _solve(exchange, tol, max_iter, check_every)


def _solve(exchange, tol, max_iter, check_every):
    ranks = exchange.ranks

    def residual():
        exchange.halo("p", ("r", "b"), 1)
        for r in ranks:
            r.residual()
        return ranks[0].reduce(exchange.sum_partials())

    done, checks = 0, 1
    res, bn = residual()
    buf = "p"
    while done < max_iter and not (bn == 0.0 or res / bn <= tol):
        for _ in range(check_every // 2):
            exchange.halo(buf, ("b",), HALO)
            for r in ranks:
                r.pass_(buf)
            buf = "q" if buf == "p" else "p"
        done += check_every
        res, bn = residual()
        checks += 1
    exchange.gather("p")
    return {"iterations": done, "residual": res, "rhs_norm": bn, "rel_residual": res / bn if bn > 0 else 0.0,
            "converged": bn == 0.0 or res / bn <= tol, "residual_checks": checks}
