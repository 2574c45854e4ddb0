"""Harvest, training and evaluation of the learned warm start.

    python -m blaze_b200.train_warm_start --grid 256 --plain-seeds 100-107 \
        --policy-seeds 108-115 --rounds 2 --out blaze_b200/weights/plume256.npz

1. Harvest: plume-family scenes (blaze_b200.scenes.family_scene) run as
   deployed: RBGS to relative residual `--tol` every frame, either plain
   (warm-started from the previous frame's pressure) or with the current
   network's warm start ("on policy").  For each harvested frame the pair is
   (rhs, p_prev) -> p*, where p* continues the frame's own solve in FP64
   (blz_tight_solve: red-black SOR, O(N) sweeps where Gauss-Seidel needs
   O(N^2), below the FP32 floor of ~1e-4 relative residual) to
   `--target-tol`; the simulation then goes on from the
   `--tol` solution, so the next p_prev carries exactly the error a
   deployed solve leaves.  On-policy rounds (as in DAgger) add pairs from
   trajectories the network itself shaped, so it learns to correct its own
   accumulated error.  Pairs stay on the GPU (FP32).
2. Training: Adam on single samples, each a random pair, a random crop whose
   origin is a multiple of 8 (the pooling grid of the full-grid inference)
   and a random mirror in x and/or z (the pressure system is symmetric under
   both); half the samples add a smooth random perturbation to p_prev (the
   target stays p*).  Loss and gradients come from the library's own forward
   and backward kernels (blz_unet_loss_grad); kappa is the pairs' mean
   rms(p* - p_prev) / rms(b - A p_prev).
3. Evaluation: held-out seeds, each run twice from the same start, a plain
   trajectory and a learned one (each frame warm-started by the network,
   then RBGS to the same residual, continuing from its own solutions);
   reports sweeps and solve time per frame.

Evaluation alone, of given weights (no training, nothing saved):

    python -m blaze_b200.train_warm_start --eval-only --init blaze_b200/weights/plume256.npz \
        --eval-seeds 902-905 --eval-frames 50 --report eval.json
"""
import argparse
import json
import math
import time

import numpy as np


def _seed_list(spec):
    out = []
    for part in str(spec).split(","):
        if "-" in part:
            a, b = part.split("-")
            out.extend(range(int(a), int(b) + 1))
        elif part:
            out.append(int(part))
    return out


# Which scene family harvest and evaluation run: "plume" (the plume family,
# scenes.family_scene) or "fire" (the large fire with moving emitters,
# scenes.large_fire_scene, whose particles are re-uploaded every frame).
SCENE = "plume"


def _solver(n, seed, tol, max_iter, check_every):
    """(solver, scene, timer, per-frame particle hook)."""
    from .scenes import Timer, family_scene, large_fire_scene
    from .solver import FluidSolver
    tmr = Timer()
    if SCENE == "fire":
        scn, frame_parts = large_fire_scene(n=n, seed=seed)
        scn.tol, scn.maxIterSolve = tol, max_iter
        solver = FluidSolver(tmr, scn, particles=frame_parts(0))

        def hook():
            solver.setParticles(frame_parts(tmr.iter))
        return solver, scn, tmr, hook
    scn, parts = family_scene(n=n, seed=seed, tol=tol, max_iter=max_iter, check_every=check_every)
    return FluidSolver(tmr, scn, particles=parts), scn, tmr, (lambda: None)


def _field(solver, name, shape):
    import torch
    t = torch.empty(shape, dtype=torch.float32, device="cuda")
    solver.get_device(name, t.data_ptr())
    return t


def sor_omega(dims):
    """Relaxation factor of the target solve: 2 / (1 + sin(pi / (2 N))),
    Young's optimum for the slowest mode of an N-cell axis with a wall at one
    end and a free surface (or wall) at the other."""
    n = max(dims)
    return 2.0 / (1.0 + math.sin(math.pi / (2.0 * n)))


def harvest(n, seeds, frames, warmup, tol, target_tol, max_iter, check_every, log=print, policy=None,
            extra_cap=6000, stride=1, omega=None):
    """List of dicts {rhs, p_prev, p_star} (device FP32, (D, H, W)) and the
    rms(p* - p_prev) / rms(r) ratios.  With `policy` (a full-grid
    WarmStartUNet) the frames after the warm-up are solved warm-started by
    it, as deployed.  `omega` is the target solve's relaxation factor (None:
    Young's optimum, sor_omega; 1: FP64 Gauss-Seidel, whose targets after
    `extra_cap` sweeps keep the smooth error Gauss-Seidel removes slowest)."""
    pairs, ratios = [], []
    for seed in seeds:
        solver, scn, tmr, hook = _solver(n, seed, tol, max_iter, check_every)
        shape = scn.to_params().field_shape("P")
        t0 = time.time()
        for f in range(warmup + frames):
            hook()
            solver.addSource()
            solver.forces(tmr.time)
            solver.divergence()
            keep = f >= warmup and (f - warmup) % stride == 0
            if keep:
                rhs = _field(solver, "RHS", shape)
                p_prev = _field(solver, "P", shape)
                r0, b0 = solver.residual()
            if f >= warmup and policy is not None:
                solver.set_warm_start(policy)
            st = solver.solve()
            solver.set_warm_start(None)
            if keep:
                p_tol = _field(solver, "P", shape)
                extra, rel = solver.tight_solve(target_tol, extra_cap, omega or sor_omega((n, n, n)))
                p_star = _field(solver, "P", shape)
                solver.set_device("P", p_tol.data_ptr())
                d = (p_star - p_prev).double()
                rms_d = float(d.pow(2).mean().sqrt())
                rms_r = r0 / math.sqrt(p_prev.numel())
                if rms_r > 0:
                    ratios.append(rms_d / rms_r)
                pairs.append({"rhs": rhs, "p_prev": p_prev, "p_star": p_star, "seed": seed, "frame": f,
                              "sweeps": st["iterations"], "extra": extra, "rel": rel})
            solver.gradient()
            solver.advect()
            tmr.iter += 1
            tmr.time += scn.dt
        kept = [p for p in pairs if p["seed"] == seed]
        log(f"harvest seed {seed} ({'on policy' if policy is not None else 'plain'}): {len(kept)} pairs in "
            f"{time.time() - t0:.1f}s, sweeps {[p['sweeps'] for p in kept]}, "
            f"target rel {[float('%.2g' % p['rel']) for p in kept]}")
        solver.close()
    return pairs, ratios


def _smooth_noise(shape, gen):
    """Unit-rms random field varying on scales of 8-32 cells."""
    import torch
    D, H, W = shape
    f = 8 * (1 << int(torch.randint(0, 3, (1,), generator=gen)))
    c = torch.randn((1, 1, max(1, D // f), max(1, H // f), max(1, W // f)), generator=gen).cuda()
    n = torch.nn.functional.interpolate(c, size=(D, H, W), mode="trilinear", align_corners=False)[0, 0]
    return n / n.pow(2).mean().sqrt().clamp_min(1e-20)


def train(net, params_blz, pairs, iters, crop, lr=1e-3, lr_end=2e-5, seed=0, log=print, log_every=100,
          perturb=0.5):
    import torch
    rng = np.random.default_rng(seed)
    gen = torch.Generator().manual_seed(seed)
    W, H, D = params_blz.width, params_blz.height, params_blz.depth
    cw, ch, cd = crop
    hist = []
    t0 = time.time()
    for it in range(iters):
        pr = pairs[int(rng.integers(len(pairs)))]
        fx, fz = bool(rng.integers(2)), bool(rng.integers(2))
        dims = [a for a, f in ((2, fx), (0, fz)) if f]
        rhs, pp, ps = pr["rhs"], pr["p_prev"], pr["p_star"]
        if dims:
            rhs, pp, ps = (torch.flip(a, dims).contiguous() for a in (rhs, pp, ps))
        if rng.random() < perturb:
            amp = float(rng.uniform(0.1, 0.6)) * float((ps - pp).pow(2).mean().sqrt())
            pp = pp + amp * _smooth_noise(pp.shape, gen)
        org = (8 * int(rng.integers((W - cw) // 8 + 1)), 8 * int(rng.integers((H - ch) // 8 + 1)),
               8 * int(rng.integers((D - cd) // 8 + 1)))
        loss, t2 = net.loss_grad(params_blz, rhs, pp, ps, org)
        frac = it / max(1, iters - 1)
        cur = lr_end + 0.5 * (lr - lr_end) * (1.0 + math.cos(math.pi * frac))
        net.adam(cur)
        hist.append((loss, t2))
        if log_every and (it % log_every == 0 or it == iters - 1):
            recent = np.array(hist[-log_every:])
            log(f"iter {it}: loss {recent[:, 0].mean():.4f} (target^2 {recent[:, 1].mean():.4f}, "
                f"rel {recent[:, 0].mean() / max(recent[:, 1].mean(), 1e-30):.4f}) lr {cur:.2e} "
                f"{time.time() - t0:.1f}s")
    torch.cuda.synchronize()
    return hist, time.time() - t0


def evaluate(net, n, seeds, frames, warmup, tol, max_iter, check_every, log=print):
    """Per seed, a plain and a learned trajectory from the same start (the
    first `warmup` frames plain in both); per frame: sweeps and solve ms."""
    rows = []
    for seed in seeds:
        for learned in (False, True):
            solver, scn, tmr, hook = _solver(n, seed, tol, max_iter, check_every)
            for f in range(warmup + frames):
                hook()
                solver.addSource()
                solver.forces(tmr.time)
                solver.divergence()
                solver.set_warm_start(net if (learned and f >= warmup) else None)
                st = solver.solve()
                if f >= warmup:
                    rows.append({"seed": seed, "frame": f, "learned": learned, "sweeps": st["iterations"],
                                 "ms": st["ms_sweeps"] + st["ms_checks"] + st["ms_warm_start"],
                                 "warm_ms": st["ms_warm_start"], "rel": st["rel_residual"],
                                 "converged": bool(st["converged"])})
                solver.gradient()
                solver.advect()
                tmr.iter += 1
                tmr.time += scn.dt
            sw = [r["sweeps"] for r in rows if r["seed"] == seed and r["learned"] == learned]
            log(f"eval seed {seed} {'learned' if learned else 'plain'}: sweeps {sw}")
            solver.close()
    return rows


def _ratios(rows):
    plain = [r for r in rows if not r["learned"]]
    learned = [r for r in rows if r["learned"]]
    return (sum(r["sweeps"] for r in plain) / max(1, sum(r["sweeps"] for r in learned)),
            sum(r["ms"] for r in plain) / max(1e-9, sum(r["ms"] for r in learned)),
            all(r["converged"] for r in rows))


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--grid", type=int, default=256)
    ap.add_argument("--scene", choices=("plume", "fire"), default="plume",
                    help="scene family harvested and evaluated: the plume family or the large fire")
    ap.add_argument("--plain-seeds", default="100-107", help="seeds harvested with plain solves ('' for none)")
    ap.add_argument("--policy-seeds", default="108-115", help="seeds harvested on policy in each round")
    ap.add_argument("--rounds", type=int, default=1, help="on-policy harvest + training rounds")
    ap.add_argument("--eval-seeds", default="900-901")
    ap.add_argument("--frames", type=int, default=8, help="frames after the warm-up per harvested seed")
    ap.add_argument("--stride", type=int, default=1, help="harvest every stride-th of those frames")
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--eval-frames", type=int, default=8)
    ap.add_argument("--tol", type=float, default=1e-4)
    ap.add_argument("--target-tol", type=float, default=1e-8)
    ap.add_argument("--extra-cap", type=int, default=6000, help="FP64 SOR sweeps spent tightening each target")
    ap.add_argument("--target-omega", type=float, default=0.0,
                    help="relaxation factor of the target solve (0: Young's optimum; 1: Gauss-Seidel)")
    ap.add_argument("--max-iter", type=int, default=40000)
    ap.add_argument("--check-every", type=int, default=20)
    ap.add_argument("--iters", type=int, default=1500, help="Adam steps per training round")
    ap.add_argument("--crop", type=int, default=128)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--perturb", type=float, default=0.5)
    ap.add_argument("--harvest", default=None,
                    help="harvest schedule 'kind:seeds:frames:stride,...' (kind plain or policy; seed lists "
                         "use '/' between items), all harvested before one training round; overrides "
                         "--plain-seeds/--policy-seeds/--rounds")
    ap.add_argument("--keep-kappa", action="store_true", help="keep the --init weights' kappa")
    ap.add_argument("--init", default=None, help="start from these weights (npz)")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=None, help="where the trained weights go (required unless --eval-only)")
    ap.add_argument("--eval-only", action="store_true",
                    help="evaluate the --init weights on --eval-seeds for --eval-frames frames; no training")
    ap.add_argument("--report", default=None, help="JSON summary path")
    args = ap.parse_args(argv)
    if args.eval_only and not args.init:
        ap.error("--eval-only needs --init")
    if not args.eval_only and not args.out:
        ap.error("--out is required")

    import torch
    from .unet import WarmStartUNet, init_params
    from .scenes import family_scene

    def log(msg):
        print(msg, flush=True)

    torch.cuda.set_device(0)
    global SCENE
    SCENE = args.scene
    n = args.grid
    crop = (min(args.crop, n),) * 3
    grid = family_scene(n=n, seed=0)[0].to_params()
    params = init_params(args.seed)
    kappa = 1.0
    if args.init:
        with np.load(args.init, allow_pickle=False) as z:
            params, kappa = z["params"], float(z["kappa"])
    pairs, ratios, hist_all = [], [], []
    t_harvest = t_train = 0.0
    full = WarmStartUNet((n, n, n), params, kappa=kappa)
    rounds = []
    plain_seeds = _seed_list(args.plain_seeds)
    policy_seeds = _seed_list(args.policy_seeds)
    if args.eval_only:
        rows = evaluate(full, n, _seed_list(args.eval_seeds), args.eval_frames, args.warmup, args.tol,
                        args.max_iter, args.check_every, log)
        sweep_ratio, time_ratio, conv = _ratios(rows)
        per_seed = {}
        for seed in _seed_list(args.eval_seeds):
            sub = [r for r in rows if r["seed"] == seed]
            per_seed[str(seed)] = dict(zip(("sweep_ratio", "time_ratio", "all_converged"), _ratios(sub)))
        summary = {"grid": n, "scene": args.scene, "weights": args.init, "kappa": kappa, "eval_seeds": args.eval_seeds,
                   "eval_frames": args.eval_frames, "warmup": args.warmup, "tol": args.tol, "max_iter": args.max_iter,
                   "steps_per_arm": len(rows) // 2, "sweep_ratio": sweep_ratio, "time_ratio": time_ratio,
                   "eval_all_converged": conv, "per_seed": per_seed, "eval": rows}
        full.close()
        log(json.dumps({k: v for k, v in summary.items() if k != "eval"}))
        if args.report:
            with open(args.report, "w") as f:
                json.dump(summary, f, indent=1)
        return
    if args.harvest:
        # one round that trains on every harvested group
        groups = []
        for item in args.harvest.split(","):
            kind, seeds, frames, stride = item.split(":")
            groups.append((kind, _seed_list(seeds.replace("/", ",")), int(frames), int(stride)))
        schedule = [groups]
    else:
        schedule = ([[("plain", plain_seeds, args.frames, args.stride)]] if plain_seeds else []) + \
                   [[("policy", policy_seeds, args.frames, args.stride)]] * args.rounds
    init_kappa = kappa
    for r, round_groups in enumerate(schedule):
        new = []
        for kind, seeds, frames, stride in round_groups:
            if kind == "policy" and not args.init and r == 0:
                raise SystemExit("on-policy rounds need a network: give --plain-seeds or --init")
            t0 = time.time()
            got, rat = harvest(n, seeds, frames, args.warmup, args.tol, args.target_tol, args.max_iter,
                               args.check_every, log, policy=full if kind == "policy" else None,
                               extra_cap=args.extra_cap, stride=stride, omega=args.target_omega or None)
            t_harvest += time.time() - t0
            new += got
            ratios += rat
        kind = "+".join(sorted({g[0] for g in round_groups}))
        seeds = [x for g in round_groups for x in g[1]]
        pairs += new
        kappa = init_kappa if (args.keep_kappa and args.init) else (float(np.mean(ratios)) if ratios else 1.0)
        log(f"round {r} ({kind}): {len(new)} new pairs, {len(pairs)} in all, kappa {kappa:.4f}")
        net = WarmStartUNet(crop, full.get_params(), kappa=kappa)
        lr = args.lr if (r == 0 and not args.init) else 0.3 * args.lr
        hist, t = train(net, grid, pairs, args.iters, crop, lr=lr, seed=args.seed + r, log=log,
                        perturb=args.perturb)
        t_train += t
        hist_all += hist
        full.set_params(net.get_params())
        full.set_kappa(kappa)
        net.close()
        rounds.append({"kind": kind, "seeds": seeds, "pairs": len(pairs),
                       "final_loss": float(np.mean([h[0] for h in hist[-100:]])),
                       "final_target2": float(np.mean([h[1] for h in hist[-100:]]))})
    del pairs
    torch.cuda.empty_cache()
    rows = evaluate(full, n, _seed_list(args.eval_seeds), args.eval_frames, args.warmup, args.tol, args.max_iter,
                    args.check_every, log)
    sweep_ratio, time_ratio, conv = _ratios(rows)
    summary = {
        "grid": n, "scene": args.scene, "plain_seeds": args.plain_seeds, "policy_seeds": args.policy_seeds,
        "rounds": rounds,
        "harvest": args.harvest, "keep_kappa": args.keep_kappa,
        "eval_seeds": args.eval_seeds, "frames": args.frames, "stride": args.stride, "warmup": args.warmup,
        "tol": args.tol,
        "target_tol": args.target_tol, "extra_cap": args.extra_cap, "target_omega": args.target_omega or "sor", "iters": args.iters, "crop": crop[0],
        "perturb": args.perturb, "init": args.init, "kappa": kappa, "harvest_s": t_harvest, "train_s": t_train,
        "eval": rows, "sweep_ratio": sweep_ratio, "time_ratio": time_ratio, "eval_all_converged": conv}
    full.meta = {k: v for k, v in summary.items() if k != "eval"}
    full.save(args.out)
    full.close()
    log(json.dumps({k: v for k, v in summary.items() if k not in ("eval", "rounds")}))
    if args.report:
        with open(args.report, "w") as f:
            json.dump(summary, f, indent=1)


if __name__ == "__main__":
    main()
