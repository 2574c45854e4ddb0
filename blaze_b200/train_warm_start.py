"""Harvest, training and evaluation of the learned warm start.

    python -m blaze_b200.train_warm_start --grid 256 --train-seeds 100-111 \
        --frames 10 --iters 2000 --out blaze_b200/weights/plume256.npz

1. Harvest: plume-family scenes (blaze_b200.scenes.family_scene) run with the
   plain solver exactly as deployed (warm-started RBGS to relative residual
   `--tol`).  For each harvested frame the pair is (rhs, p_prev) -> p*, where
   p* continues the frame's own solve with more sweeps to `--target-tol`; the
   simulation then goes on from the `--tol` solution, so the next p_prev has
   the error a deployed solve leaves.  Pairs stay on the GPU (FP32).
2. Training: Adam on single samples, each a random pair, a random crop whose
   origin is a multiple of 8 (the pooling grid of the full-grid inference)
   and a random mirror in x and/or z (the pressure system is symmetric under
   both).  Loss and gradients come from the library's own forward and
   backward kernels (blz_unet_loss_grad); kappa is the pairs' mean
   rms(p* - p_prev) / rms(b - A p_prev).
3. Evaluation: held-out seeds, each frame solved twice from the same state,
   plain and warm-started, both to `--tol`; reports sweeps and solve time.
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


def _solver(n, seed, tol, max_iter, check_every):
    from .scenes import Timer, family_scene
    from .solver import FluidSolver
    scn, parts = family_scene(n=n, seed=seed, tol=tol, max_iter=max_iter, check_every=check_every)
    tmr = Timer()
    return FluidSolver(tmr, scn, particles=parts), scn, tmr


def _field(solver, name, shape):
    import torch
    t = torch.empty(shape, dtype=torch.float32, device="cuda")
    solver.get_device(name, t.data_ptr())
    return t


def _tighten(solver, target, cap, chunk=500):
    """Sweeps the current pressure on to relative residual `target`."""
    done = 0
    r, b = solver.residual()
    while b > 0 and r / b > target and done < cap:
        solver.sweeps(chunk)
        done += chunk
        r, b = solver.residual()
    return done, (r / b if b > 0 else 0.0)


def harvest(n, seeds, frames, warmup, tol, target_tol, max_iter, check_every, log=print):
    """List of dicts {rhs, p_prev, p_star} (device FP32, (D, H, W)) and the
    kappa statistic."""
    pairs, ratios = [], []
    for seed in seeds:
        solver, scn, tmr = _solver(n, seed, tol, max_iter, check_every)
        shape = scn.to_params().field_shape("P")
        t0 = time.time()
        for f in range(warmup + frames):
            solver.addSource()
            solver.forces(tmr.time)
            solver.divergence()
            if f >= warmup:
                rhs = _field(solver, "RHS", shape)
                p_prev = _field(solver, "P", shape)
                r0, b0 = solver.residual()
            st = solver.solve()
            if f >= warmup:
                p_tol = _field(solver, "P", shape)
                extra, rel = _tighten(solver, target_tol, 100000)
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
        log(f"harvest seed {seed}: {frames} pairs in {time.time() - t0:.1f}s, "
            f"sweeps {[p['sweeps'] for p in pairs[-frames:]]}, extra {[p['extra'] for p in pairs[-frames:]]}")
        solver.close()
    kappa = float(np.mean(ratios)) if ratios else 1.0
    return pairs, kappa


def train(net, params_blz, pairs, iters, crop, lr=1e-3, lr_end=2e-5, seed=0, log=print, log_every=100):
    import torch
    rng = np.random.default_rng(seed)
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
    """Per frame: sweeps and solve ms, plain and warm-started, from the same state."""
    import torch
    rows = []
    for seed in seeds:
        solver, scn, tmr = _solver(n, seed, tol, max_iter, check_every)
        shape = scn.to_params().field_shape("P")
        for f in range(warmup + frames):
            solver.addSource()
            solver.forces(tmr.time)
            solver.divergence()
            if f >= warmup:
                p_prev = _field(solver, "P", shape)
                torch.cuda.synchronize()
                sp = solver.solve()
                p_plain = _field(solver, "P", shape)
                solver.set_device("P", p_prev.data_ptr())
                solver.set_warm_start(net)
                sl = solver.solve()
                solver.set_warm_start(None)
                solver.set_device("P", p_plain.data_ptr())
                rows.append({"seed": seed, "frame": f, "plain_sweeps": sp["iterations"],
                             "learned_sweeps": sl["iterations"], "plain_ms": sp["ms_sweeps"] + sp["ms_checks"],
                             "learned_ms": sl["ms_sweeps"] + sl["ms_checks"] + sl["ms_warm_start"],
                             "warm_ms": sl["ms_warm_start"], "plain_rel": sp["rel_residual"],
                             "learned_rel": sl["rel_residual"],
                             "converged": bool(sp["converged"] and sl["converged"])})
                log(f"eval seed {seed} frame {f}: plain {sp['iterations']} sweeps, learned {sl['iterations']} "
                    f"(+{sl['ms_warm_start']:.2f} ms network)")
            else:
                solver.solve()
            solver.gradient()
            solver.advect()
            tmr.iter += 1
            tmr.time += scn.dt
        solver.close()
    return rows


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--grid", type=int, default=256)
    ap.add_argument("--train-seeds", default="100-111")
    ap.add_argument("--eval-seeds", default="900-901")
    ap.add_argument("--frames", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--eval-frames", type=int, default=4)
    ap.add_argument("--tol", type=float, default=1e-4)
    ap.add_argument("--target-tol", type=float, default=1e-5)
    ap.add_argument("--max-iter", type=int, default=40000)
    ap.add_argument("--check-every", type=int, default=20)
    ap.add_argument("--iters", type=int, default=2000)
    ap.add_argument("--crop", type=int, default=128)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--init", default=None, help="start from these weights (npz)")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", required=True)
    ap.add_argument("--report", default=None, help="JSON summary path")
    args = ap.parse_args(argv)

    import torch
    from .unet import WarmStartUNet, init_params
    from .scenes import family_scene

    def log(msg):
        print(msg, flush=True)

    torch.cuda.set_device(0)
    n = args.grid
    t0 = time.time()
    pairs, kappa = harvest(n, _seed_list(args.train_seeds), args.frames, args.warmup, args.tol, args.target_tol,
                           args.max_iter, args.check_every, log)
    t_harvest = time.time() - t0
    log(f"harvested {len(pairs)} pairs in {t_harvest:.1f}s, kappa {kappa:.4f}")
    crop = (min(args.crop, n),) * 3
    net = WarmStartUNet(crop, init_params(args.seed), kappa=kappa)
    if args.init:
        net.load(args.init)
        net.set_kappa(kappa)
    grid = family_scene(n=n, seed=_seed_list(args.train_seeds)[0])[0].to_params()
    hist, t_train = train(net, grid, pairs, args.iters, crop, lr=args.lr, seed=args.seed, log=log)
    params = net.get_params()
    net.close()
    del pairs
    torch.cuda.empty_cache()
    full = WarmStartUNet((n, n, n), params, kappa=kappa)
    rows = evaluate(full, n, _seed_list(args.eval_seeds), args.eval_frames, args.warmup, args.tol, args.max_iter,
                    args.check_every, log)
    plain = sum(r["plain_sweeps"] for r in rows)
    learned = sum(r["learned_sweeps"] for r in rows)
    summary = {
        "grid": n, "train_seeds": args.train_seeds, "eval_seeds": args.eval_seeds, "frames": args.frames,
        "warmup": args.warmup, "pairs": len(hist) and len(_seed_list(args.train_seeds)) * args.frames,
        "tol": args.tol, "target_tol": args.target_tol, "iters": args.iters, "crop": crop[0], "kappa": kappa,
        "harvest_s": t_harvest, "train_s": t_train,
        "final_loss": float(np.mean([h[0] for h in hist[-100:]])),
        "final_target2": float(np.mean([h[1] for h in hist[-100:]])),
        "eval": rows, "sweep_ratio": plain / max(learned, 1),
        "time_ratio": sum(r["plain_ms"] for r in rows) / max(sum(r["learned_ms"] for r in rows), 1e-9)}
    full.meta = {k: v for k, v in summary.items() if k != "eval"}
    full.save(args.out)
    full.close()
    log(json.dumps({k: v for k, v in summary.items() if k != "eval"}))
    if args.report:
        with open(args.report, "w") as f:
            json.dump(summary, f, indent=1)


if __name__ == "__main__":
    main()
