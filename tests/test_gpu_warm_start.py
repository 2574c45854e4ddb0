"""What the trained warm start gains: on a held-out 256^3 plume-family seed
(not among the training seeds recorded in the weight file), the same frames
are solved from the same state plain (RBGS from the previous frame's
pressure) and warm-started by the network.  Every warm-started solve reaches
FP64 relative residual 1e-4, and together they need at most half the sweeps
of the plain solves (a plain solve that stops at the sweep cap counts as the
cap, a lower bound of what it needs)."""
import json
import os

import pytest

pytestmark = pytest.mark.gpu

SEED = 902


def test_trained_network_halves_the_sweeps():
    import torch
    from blaze_b200 import FluidSolver, Timer, family_scene
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
