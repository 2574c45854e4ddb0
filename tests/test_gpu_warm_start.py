"""What the trained warm start gains, on a held-out 256^3 plume-family seed
(not among the training seeds recorded in the weight file).  Every
warm-started solve reaches FP64 relative residual 1e-4, and the warm-started
solves together need at most half the sweeps of the plain ones (a plain solve
that stops at the sweep cap counts as the cap, a lower bound of what it
needs), in two settings:

- from plain states: each frame is solved from the plain trajectory's state,
  once plain (RBGS from the previous frame's pressure) and once
  warm-started;
- along a trajectory: the same frames replayed from one snapshot, once with
  plain solves and once with the network on every frame, each trajectory
  feeding on its own solutions as a simulation does.

Both use the warm start's defaults (residual-norm step after 40 smoothing
sweeps)."""
import json
import os

import pytest

pytestmark = pytest.mark.gpu

SEED = 902


def _held_out_net():
    from blaze_b200.unet import WarmStartUNet, weights_path
    path = weights_path("plume256.npz")
    assert os.path.exists(path), "trained weights missing"
    net = WarmStartUNet((256, 256, 256)).load(path)
    trained_on = set()
    for rnd in net.meta.get("rounds", []):
        trained_on.update(int(x) for x in rnd.get("seeds", []))
    for key in ("plain_seeds", "policy_seeds", "train_seeds"):
        spec = net.meta.get(key) or ""
        for part in str(spec).split(","):
            if "-" in part:
                a, b = part.split("-")
                trained_on.update(range(int(a), int(b) + 1))
    assert trained_on and SEED not in trained_on
    return net


def test_trained_network_halves_the_sweeps_from_plain_states():
    import torch
    from blaze_b200 import FluidSolver, Timer, family_scene
    net = _held_out_net()
    scn, parts = family_scene(n=256, seed=SEED, tol=1e-4, max_iter=60000, check_every=20)
    tmr = Timer()
    solver = FluidSolver(tmr, scn, particles=parts)
    shape = scn.to_params().field_shape("P")
    rows = []
    for f in range(8):
        solver.addSource()
        solver.forces(tmr.time)
        solver.divergence()
        if f >= 5:
            p_prev = torch.empty(shape, dtype=torch.float32, device="cuda")
            solver.get_device("P", p_prev.data_ptr())
            plain = solver.solve()
            p_plain = torch.empty_like(p_prev)
            solver.get_device("P", p_plain.data_ptr())
            solver.set_device("P", p_prev.data_ptr())
            solver.set_warm_start(net)
            learned = solver.solve()
            solver.set_warm_start(None)
            solver.set_device("P", p_plain.data_ptr())
            rows.append((plain["iterations"], learned["iterations"], plain["rel_residual"], learned["rel_residual"],
                         learned["warm_started"]))
        else:
            solver.solve()
        solver.gradient()
        solver.advect()
        tmr.iter += 1
        tmr.time += scn.dt
    solver.close()
    net.close()
    print(json.dumps({"plain_vs_learned_sweeps": rows}))
    for n_plain, n_learned, rel_p, rel_l, warm in rows:
        assert warm == 1 and rel_l <= 1e-4, rows
    assert sum(r[1] for r in rows) <= 0.5 * sum(r[0] for r in rows), rows


def test_trained_network_halves_the_sweeps_along_a_trajectory():
    import torch
    from blaze_b200 import FluidSolver, Timer, family_scene
    net = _held_out_net()
    scn, parts = family_scene(n=256, seed=SEED, tol=1e-4, max_iter=60000, check_every=20)
    tmr = Timer()
    solver = FluidSolver(tmr, scn, particles=parts)

    def frame():
        solver.addSource()
        st = solver.step(tmr.time)
        tmr.iter += 1
        tmr.time += scn.dt
        return st

    for _ in range(5):
        frame()
    snap = {f: solver.get(f) for f in ("T", "U", "V", "W", "P")}
    clock = (tmr.iter, tmr.time)
    runs = {}
    for name, warm in (("plain", None), ("learned", net)):
        for f, a in snap.items():
            solver.set(f, a)
        tmr.iter, tmr.time = clock
        solver.set_warm_start(warm)
        runs[name] = [frame() for _ in range(4)]
    solver.set_warm_start(None)
    solver.close()
    net.close()
    plain = [st["iterations"] for st in runs["plain"]]
    learned = [st["iterations"] for st in runs["learned"]]
    print(json.dumps({"plain": plain, "learned": learned}))
    assert all(st["warm_started"] == 1 and st["rel_residual"] <= 1e-4 for st in runs["learned"]), learned
    assert sum(learned) <= 0.5 * sum(plain), (plain, learned)
