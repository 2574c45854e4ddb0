"""Benchmark of the per-frame fluid step at 256^3 (plume-family scene).

A step is one frame: particle sourcing + FluidSolver::step (forces,
divergence, red-black Gauss-Seidel to relative FP64 residual 1e-4, gradient,
RK3 advection).  After W warm-up frames the state is snapshotted and the same
K frames are timed twice from it: plain (RBGS warm-started from the previous
frame's pressure) and learned (the U-Net warm start of
blaze_b200/weights/plume<N>.npz, then RBGS to the same residual).  `value`
is the learned pass when those weights exist; both passes are in the line.
Prints one JSON line (rank 0).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--plain-only] [--weights PATH]

--impl reference times the reference's own CUDA build (oracle/_ref) on the
same scene and particles through its FluidSolver API, each frame with
maxIterSolve equal to the sweeps the plain RBGS step needs on that frame
(measured by a plain-only run of this script in a child process; the
reference has no residual control).  N > 1 runs independent replicas, one
per GPU (the single grid does not shard); value is the sum over ranks, timed
as the max over ranks.  --workload fire384 runs the 384^3 large fire with
moving emitters the same way; --workload batch splits one set of 64
simulations across the ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "256³ steps/s: learned warm-start vs plain RBGS at equal residual; HBM GB/s"
METRIC_FIRE = "384³ large-fire steps/s: learned warm-start vs plain RBGS at equal residual; HBM GB/s"


def metric_of(args):
    return METRIC_FIRE if args.workload == "fire384" else METRIC
GRID = 256
SEED = 3
TOL = 1e-4
MAX_ITER = 40000
CHECK_EVERY = 20          # residual-check interval of the batched simulations
CHECK_AUTO = -1           # the 256^3 step: interval chosen per frame (blz_params.check_every < 0)
# The reference arm runs, frame by frame, the sweep count (maxIterSolve) the
# plain RBGS step needs on the same frame, measured by a plain-only run of
# this script in a child process just before (BLZ_REF_SWEEPS=<n> fixes n
# sweeps per frame instead, for short runs).
REF_SWEEPS_ENV = "BLZ_REF_SWEEPS"


def load_peaks():
    return _peak("hbm_gbs", 6650.0)


def _peak(key, fallback):
    """A measured peak of this pool's B200s (MEASURED_PEAKS.json), else the
    earlier measurement given as fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d[key]), "measured"
    except Exception:
        return fallback, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = [r.split(",") for r in (self.out or "").strip().splitlines() if r.count(",") >= 8]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if "Active" in v and "Not" not in v})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def step_bytes(W, H, D, sweeps, checks):
    """Algorithmic HBM bytes of one frame (FP32; velocity read once per pass)."""
    cT = W * H * D
    cF = (W + 1) * H * D + W * (H + 1) * D + W * H * (D + 1)
    forces = 8 * cT + 8 * cF
    divergence = 4 * cF + 4 * cT
    rbgs = 12 * cT * sweeps
    residual = 8 * cT * checks
    gradient = 4 * cT + 8 * cF
    advect = 8 * cT + 8 * cF
    return forces + divergence + rbgs + residual + gradient + advect


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def cpu_baseline(scn, parts, mean_sweeps):
    """FP64 oracle (OpenMP) on a bounded sample of the same frame: the
    non-solver stages once plus 10 sweeps, extrapolated to the mean sweep
    count of the GPU run."""
    from oracle import oracle
    p = scn.to_params()
    st = oracle.State(p, np.float64)
    st.add_source(parts)
    t0 = time.perf_counter()
    st.add_source(parts)
    st.forces(0.0)
    st.divergence()
    t1 = time.perf_counter()
    n_s = 10
    st.gs_sweeps(n_s)
    t2 = time.perf_counter()
    st.residual_norms()
    st.gradient()
    st.advect()
    t3 = time.perf_counter()
    cores = oracle.num_threads()
    # the same sweeps on one core (a few of them: about ten times slower)
    n_1 = 3
    per_sweep_1 = None
    if oracle.set_num_threads(1):
        try:
            t4 = time.perf_counter()
            st.gs_sweeps(n_1)
            per_sweep_1 = (time.perf_counter() - t4) / n_1
        finally:
            oracle.set_num_threads(cores)
    per_sweep = (t2 - t1) / n_s
    per_step = (t1 - t0) + (t3 - t2) + per_sweep * mean_sweeps
    one = (f"; {n_1} sweeps on one core ({per_sweep_1 * 1e3:.1f} ms/sweep)" if per_sweep_1 else "")
    return {"value": 1.0 / per_step, "unit": "steps/s", "cores": cores, "kind": "port",
            "ms_per_sweep": per_sweep * 1e3,
            "ms_per_sweep_1core": per_sweep_1 * 1e3 if per_sweep_1 else None,
            "value_1core_sweeps_only": 1.0 / (per_sweep_1 * mean_sweeps) if per_sweep_1 else None,
            "sample": f"one {scn.gridRes[0]}^3 frame of the FP64 oracle: non-solver stages timed once, "
                      f"{n_s} GS sweeps timed and scaled to {mean_sweeps:.0f} sweeps "
                      f"({per_sweep * 1e3:.1f} ms/sweep, {per_step:.1f} s/step){one}"}


def unet_flops(dims):
    """Multiply-add FLOPs (x2) of one forward pass of the warm-start network
    at grid dims (W, H, D): 3x3x3 convolutions at their level, 2x2x2
    transposed convolutions at their output level, the 1x1 head."""
    from blaze_b200.unet import layers, KIND_CONV3, KIND_UP
    W, H, D = dims
    vox = [(W >> l) * (H >> l) * (D >> l) for l in range(4)]
    total = 0
    for L in layers():
        name = L["name"]
        if L["kind"] == KIND_CONV3:
            total += 2 * 27 * L["cin"] * L["cout"] * vox[int(name[1])]
        elif L["kind"] == KIND_UP:
            total += 2 * L["cin"] * L["cout"] * vox[int(name[1])]
        else:
            total += 2 * L["cin"] * L["cout"] * vox[0]
    return total


def unet_roofline(net, scn, solver, stream, reps=3):
    """The forward pass on the solver's current rhs and pressure: mean of
    `reps` runs after one untimed, CUDA events on `stream`."""
    import torch
    W, H, D = scn.gridRes
    rhs = torch.from_numpy(np.ascontiguousarray(solver.get("RHS"))).cuda()
    p = torch.from_numpy(np.ascontiguousarray(solver.get("P"))).cuda()
    out = torch.empty((D, H, W), dtype=torch.float32, device="cuda")
    params = scn.to_params()
    net.forward(params, rhs, p, out=out, stream=stream.cuda_stream)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(reps):
        net.forward(params, rhs, p, out=out, stream=stream.cuda_stream)
    b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / reps
    flops = unet_flops((W, H, D))
    peak, kind = _peak("bf16_tflops", 1590.0)             # burst: the forward timed on its own
    achieved = flops / (ms * 1e-3) / 1e12
    return {"bound": "tensor", "kernel": "warm-start network forward (k_conv3d_zm / k_conv3d_tc / k_upconv_tc "
                                          "on tcgen05, BF16 in, FP32 accumulate; pooling, input, norms and head "
                                          "on SIMT)",
            "ms": ms, "tflop": flops / 1e12, "achieved": achieved, "peak": peak, "peak_kind": kind,
            "unit": "TFLOP/s", "frac": achieved / peak,
            "timing": f"CUDA events around {reps} forward passes on the bench stream, outside the timed region"}


def _load_net(args, W, H, D):
    """The trained warm-start network for this grid, or (None, reason).  The
    network is fully convolutional: without weights trained at this size the
    256^3 weights are applied (and the line says so)."""
    from blaze_b200.unet import WarmStartUNet, weights_path
    if args.plain_only:
        return None, "disabled (--plain-only)"
    path = args.weights or weights_path(f"plume{W}.npz")
    note = ""
    if not os.path.exists(path) and not args.weights:
        path, note = weights_path("plume256.npz"), f" (trained at 256^3, applied at {W}x{H}x{D})"
    if not os.path.exists(path):
        return None, f"no trained weights for {W}^3 ({os.path.relpath(path, ROOT)})"
    net = WarmStartUNet((W, H, D)).load(path)
    return net, os.path.relpath(path, ROOT) + note


def make_workload(args, seed, tol=TOL, max_iter=None, check_every=None, bc_mode=None):
    """(SceneSettings, frame_particles, description) of the --workload:
    plume, the 256^3 plume-family benchmark scene (one static particle set);
    fire384, the large fire scene (a static ground disc and two spheres
    moving 1 cell per frame, re-sourced every frame as an animated source)."""
    from blaze_b200 import family_scene
    from blaze_b200.scenes import large_fire_scene
    max_iter = args.max_iter if max_iter is None else max_iter
    if check_every is None:
        check_every = CHECK_AUTO if max_iter % 320 == 0 else CHECK_EVERY
    if args.workload == "fire384":
        scn, fp = large_fire_scene(n=args.grid if args.grid != GRID else 384, seed=5 + seed - SEED)
        scn.tol, scn.maxIterSolve, scn.check_every = tol, max_iter, check_every
        if bc_mode is not None:
            scn.bc_mode = bc_mode
            scn.defect_correction = 0 if bc_mode == 0 else scn.defect_correction
        n = scn.gridRes[0]
        desc = (f"large fire {n}^3 (ground disc of 30000 particles, two spheres moving 1 cell/frame as an "
                f"animated source, curl noise 0.8 / 8 cells, wind 0.3 cells/step)")
        return scn, fp, desc
    scn, parts = family_scene(n=args.grid, seed=seed, tol=tol, max_iter=max_iter, check_every=check_every,
                              **({} if bc_mode is None else {"bc_mode": bc_mode}))
    if bc_mode is not None and bc_mode == 0:
        scn.defect_correction = 0
    desc = (f"plume-family {args.grid}^3 scene (seed {seed}, {scn.extra['sources']} sources, "
            f"wind {scn.extra['wind_cells_per_step']:.2f} cells/step)")
    return scn, (lambda f: parts), desc


def run_ours(args, ws, rank, local):
    import torch
    from blaze_b200 import FluidSolver, Timer

    torch.cuda.set_device(local)
    scn, frame_parts, desc = make_workload(args, SEED + rank)
    check = scn.check_every
    animated = args.workload == "fire384"
    parts = frame_parts(0)
    if args.host_loop:
        scn.device_loop = 0
    W, H, D = scn.gridRes
    # A dedicated stream shared by the solver and the timing events (the
    # legacy default stream has handle 0, which the library reads as "use
    # your own stream").
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    tmr = Timer()
    solver = FluidSolver(tmr, scn, particles=parts, stream=stream.cuda_stream)
    net, net_src = _load_net(args, W, H, D)

    def frame():
        if animated:                                    # the reference re-reads an animated source every frame
            solver.setParticles(frame_parts(tmr.iter))
        solver.addSource()
        st = solver.step(tmr.time)
        tmr.iter += 1
        tmr.time += scn.dt
        return st

    for _ in range(args.warmup):
        frame()
    torch.cuda.synchronize()
    # State after warm-up: every timed pass below replays the same frames from it.
    snap = {f: solver.get(f) for f in ("T", "U", "V", "W", "P")}
    clock0 = (tmr.iter, tmr.time)

    def restore():
        for f, a in snap.items():
            solver.set(f, a)
        tmr.iter, tmr.time = clock0
        torch.cuda.synchronize()

    def timed_pass(learned):
        """K frames from the snapshot; device time (max over ranks), stats, launches."""
        restore()
        solver.set_warm_start(net if learned else None)
        if ws > 1:
            torch.distributed.barrier()
        l0 = solver.kernel_launches()
        stats = []
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            stats.append(frame())
        e1.record(stream)
        torch.cuda.synchronize()
        if ws > 1:
            torch.distributed.barrier()
        ms = e0.elapsed_time(e1)
        if ws > 1:
            t = torch.tensor([ms], device="cuda")
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            ms = float(t.item())
        return ms, stats, solver.kernel_launches() - l0

    with ClockSampler(local) as clk:
        ms_plain, st_plain, launches_plain = timed_pass(False)
        if net is not None:
            ms_learn, st_learn, launches_learn = timed_pass(True)
    head_learned = net is not None
    ms, stats, launches = (ms_learn, st_learn, launches_learn) if head_learned else (ms_plain, st_plain, launches_plain)

    # The dominant kernel (half sweep) timed with CUDA events on this stream,
    # on the state the timed passes left.
    solver.set_warm_start(None)
    n_meas = 20
    m0, m1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    solver.sweeps(2)
    m0.record(stream)
    solver.sweeps(n_meas)
    m1.record(stream)
    torch.cuda.synchronize()
    sweep_ms_events = m0.elapsed_time(m1) / n_meas

    # The network's forward pass alone (its convolutions run on the tcgen05
    # tensor cores), timed with CUDA events on this stream, against the
    # measured BF16 peak: the tensor-core roofline of the warm start.
    unet_line = None
    if head_learned:
        unet_line = unet_roofline(net, scn, solver, stream)

    e2e_s = None
    # e2e through the public API with host buffers: per frame the particle
    # records go host->device (the reference re-reads an animated source every
    # frame) and the advanced temperature field comes back device->host.
    if not args.no_e2e:
        restore()
        solver.set_warm_start(net if head_learned else None)
        pinned_parts = torch.empty((len(parts), 8), dtype=torch.float32, pin_memory=True)
        pinned_parts.numpy()[...] = parts
        t_host = torch.empty(scn.to_params().field_shape("T"), dtype=torch.float32, pin_memory=True)
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        for _ in range(args.steps):
            if animated:
                pinned_parts.numpy()[...] = frame_parts(tmr.iter)
            solver.setParticles(pinned_parts.numpy())
            solver.addSource()
            solver.step(tmr.time)
            solver.get("T", out=t_host.numpy())
            tmr.iter += 1
            tmr.time += scn.dt
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - w0
        if ws > 1:
            t = torch.tensor([e2e_s], device="cuda")
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            e2e_s = float(t.item())
    solver.set_warm_start(None)

    if rank != 0:
        solver.close()
        return None
    peak, peak_kind = load_peaks()
    n_cells = W * H * D

    def summary(ms_, st_):
        sw = np.array([s["iterations"] for s in st_], float)
        ck = np.array([s["residual_checks"] for s in st_], float)
        rel = np.array([s["rel_residual"] for s in st_], float)
        out = {"steps_per_s": ws * args.steps / (ms_ * 1e-3), "ms_per_step": ms_ / args.steps,
               "mean_sweeps": float(sw.mean()), "sweeps_per_frame": [int(x) for x in sw],
               "max_rel_residual": float(rel.max()), "all_converged": all(s["converged"] for s in st_),
               "hbm_gbs_step": float(np.mean([step_bytes(W, H, D, a, c) for a, c in zip(sw, ck)]))
               / (ms_ / args.steps * 1e-3) / 1e9,
               "ms_per_sweep": float(sum(s["ms_sweeps"] for s in st_) / max(1.0, sw.sum())),
               "stage_ms": {k: float(np.mean([s[k] for s in st_])) for k in
                            ("ms_forces", "ms_divergence", "ms_solve", "ms_gradient", "ms_advect", "ms_sweeps",
                             "ms_checks", "ms_warm_start")}}
        return out

    plain = summary(ms_plain, st_plain)
    learned = summary(ms_learn, st_learn) if head_learned else None
    sweeps = np.array([s["iterations"] for s in st_plain], float)
    ms_sweeps = float(sum(s["ms_sweeps"] for s in st_plain))
    variant = st_plain[-1]["sweep_variant"]
    blocked = variant >= 6
    # Algorithmic bytes: the unblocked model of a red-black sweep, 12 B per
    # cell (rhs and the other colour read, p written once).  A temporal-
    # blocking launch performs two sweeps, so its algorithmic bytes are
    # 24 B/cell and its fraction can exceed 1.0; the bytes it must move at
    # least (rhs 4 B, the black half of p 2 B, p written 4 B per cell) are
    # reported beside them, with the ncu DRAM traffic.
    if blocked:
        kernel, per_sweep, alg_launch = "k_rbgs_tb2 (two sweeps per pass)", 0.5, 24.0 * n_cells
        min_launch = 10.0 * n_cells
    else:
        # one launch = half a sweep: rhs_c + p_other read, p_c written (4 B each, half the cells)
        kernel, per_sweep, alg_launch = "k_rbgs_seg (half sweep)", 2.0, 6.0 * n_cells
        min_launch = alg_launch
    launch_ms_events = sweep_ms_events / per_sweep
    region_launches = per_sweep * sweeps.sum()
    avg_launch_ms_region = ms_sweeps / region_launches if region_launches else float("nan")
    achieved = alg_launch / (launch_ms_events * 1e-3) / 1e9
    traffic = None
    prof = os.path.join(ROOT, "profiles", f"{'tb2' if blocked else 'rbgs_half'}_{W}.json")
    if os.path.exists(prof):
        try:
            traffic = json.load(open(prof)).get("dram_bytes_per_launch")
        except Exception:
            traffic = None
    value = ws * args.steps / (ms * 1e-3)
    head = learned if head_learned else plain
    line = {
        "metric": metric_of(args), "value": value, "unit": "steps/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{desc}, "
                               f"{'learned warm start + ' if head_learned else 'plain '}RBGS with free-surface "
                               f"top to FP64 relative residual {TOL:g} per frame"
                               f"{' (defect correction: sweeps on the correction to the previous pressure)' if scn.defect_correction else ''}",
                   "grid": [W, H, D], "particles": int(len(parts)), "tol": TOL,
                   "check_every": "auto: per frame from 20..320, minimising checks plus sweeps past convergence"
                   if check < 0 else check,
                   "check_intervals": [int(x["check_interval"]) for x in (st_learn if head_learned else st_plain)],
                   "max_iter": args.max_iter, "mean_sweeps": head["mean_sweeps"],
                   "sweeps_per_frame": head["sweeps_per_frame"], "max_rel_residual": head["max_rel_residual"],
                   "all_converged": head["all_converged"],
                   "l2": "inputs larger than L2 (0.9 GB of fields per replica)",
                   "parallelism": f"replicas x{ws}", "device_loop": bool(st_plain[-1]["device_loop"]),
                   "learned_warm_start": net_src if head_learned else f"off: {net_src}",
                   "timed_passes": "plain and learned each replay the same K frames from one post-warm-up "
                                   "snapshot; value is the learned pass when a network is loaded"},
        "plain": plain,
        "learned": learned,
        "learned_speedup": (learned["steps_per_s"] / plain["steps_per_s"]) if head_learned else None,
        "hbm_gbs_step": head["hbm_gbs_step"],
        "roofline": {"bound": "hbm", "kernel": kernel, "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "alg_bytes_per_launch": alg_launch, "min_bytes_per_launch": min_launch,
                     "avg_launch_ms": launch_ms_events,
                     "avg_launch_ms_in_timed_region": avg_launch_ms_region,
                     "sweep_ms": sweep_ms_events,
                     "unblocked_sweep_equivalent_gbs": 12.0 * n_cells / (sweep_ms_events * 1e-3) / 1e9,
                     "timing": f"CUDA events around {n_meas} sweeps on the bench stream after the timed passes; "
                               "in-region figure from the device global timer around each sweep batch",
                     "sweep_variant": variant},
        "roofline_warm_start": unet_line,
        "e2e": None if e2e_s is None else
               {"value": ws * args.steps / e2e_s, "unit": "steps/s",
                "h2d_bytes_per_step": int(parts.nbytes), "d2h_bytes_per_step": int(n_cells * 4)},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
        "stage_ms": head["stage_ms"],
    }
    if head_learned:
        keep = ("plain_seeds", "policy_seeds", "train_seeds", "frames", "iters", "crop", "kappa", "target_tol",
                "eval_seeds", "sweep_ratio", "time_ratio")
        line["config"]["network"] = {k: net.meta[k] for k in keep if k in net.meta}
        if "rounds" in net.meta:
            line["config"]["network"]["rounds"] = [(r["kind"], r["pairs"]) for r in net.meta["rounds"]]
    if not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(scn, parts, float(sweeps.mean()))
    solver.close()
    if net is not None:
        net.close()
    return line


def run_batch(args, ws, rank, local):
    """Config 4: one seeded set of 64 independent plume simulations of uneven
    sizes, plain and learned mixed (every second simulation warm-started by
    the network, one network instance per grid size, the 256^3 weights
    applied at each size), stepped as one batch; value = aggregate cells x
    steps / s.  With N ranks the set is split by cell count
    (parallel.shard_sims: no data-path collective), so the total work is fixed
    (strong scaling).  The same simulations are also stepped one by one (each
    its own device-loop solve, all on one stream) for the same frames: that
    pass is timed the same way and every field of every simulation is
    compared bit for bit."""
    import torch
    from blaze_b200 import FluidSolver, Timer
    from blaze_b200.batch import Batch
    from blaze_b200.parallel import shard_sims
    from blaze_b200.scenes import batch_scenes
    from blaze_b200.unet import WarmStartUNet, weights_path

    torch.cuda.set_device(local)
    all_scenes = batch_scenes(args.batch_sims, seed=4, tol=TOL, max_iter=MAX_ITER, check_every=CHECK_EVERY)
    all_cells = [s.gridRes[0] * s.gridRes[1] * s.gridRes[2] for s, _ in all_scenes]
    mine = shard_sims(all_cells, ws)[rank]
    scenes = [all_scenes[i] for i in mine]
    cells = sum(all_cells[i] for i in mine)
    total_cells = sum(all_cells)
    dt = scenes[0][0].dt
    wpath = weights_path("plume256.npz")
    nets = {}

    def net_for(i, scn):
        """Every second simulation (by its index in the whole set) is learned."""
        if args.plain_only or mine[i] % 2 == 0 or not os.path.exists(wpath):
            return None
        dims = tuple(scn.gridRes)
        if dims not in nets:
            nets[dims] = WarmStartUNet(dims).load(wpath)
        return nets[dims]

    # batched
    sims = [FluidSolver(Timer(), s, particles=p) for s, p in scenes]
    for i, (sm, (s, _)) in enumerate(zip(sims, scenes)):
        sm.set_warm_start(net_for(i, s))
    batch = Batch(sims)

    def frame(f):
        batch.add_source()
        return batch.step([f * dt] * len(sims))

    for f in range(args.warmup):
        frame(f)
    st = torch.cuda.ExternalStream(batch.stream)
    if ws > 1:
        torch.distributed.barrier()
    l0 = batch.kernel_launches()
    stats = []
    with ClockSampler(local) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        for f in range(args.warmup, args.warmup + args.steps):
            stats.append(frame(f))
        e1.record(st)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = batch.kernel_launches() - l0
    fields = [{k: sm.get(k) for k in ("T", "U", "V", "W", "P")} for sm in sims]
    batch.close()
    for sm in sims:
        sm.close()

    # one by one, same frames
    alone_stream = torch.cuda.Stream()
    alone = [FluidSolver(Timer(), s, particles=p, stream=alone_stream.cuda_stream) for s, p in scenes]
    for i, (sm, (s, _)) in enumerate(zip(alone, scenes)):
        sm.set_warm_start(net_for(i, s))

    def frame_alone(f):
        for sm in alone:
            sm.addSource()
            sm.step(f * dt)

    for f in range(args.warmup):
        frame_alone(f)
    a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a0.record(alone_stream)
    for f in range(args.warmup, args.warmup + args.steps):
        frame_alone(f)
    a1.record(alone_stream)
    torch.cuda.synchronize()
    ms_alone = a0.elapsed_time(a1)
    agree = all(np.array_equal(sm.get(k), v) for sm, fd in zip(alone, fields) for k, v in fd.items())
    for sm in alone:
        sm.close()
    for n_ in nets.values():
        n_.close()
    if ws > 1:
        t = torch.tensor([ms, ms_alone], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms, ms_alone = float(t[0].item()), float(t[1].item())
    if rank != 0:
        return None
    sweeps = np.array([[x["iterations"] for x in fr] for fr in stats], float)
    learned_mask = np.array([bool(x["warm_started"]) for x in stats[0]])
    value = total_cells * args.steps / (ms * 1e-3)
    dims = {}
    for s, _ in scenes:
        dims[str(tuple(s.gridRes))] = dims.get(str(tuple(s.gridRes)), 0) + 1
    return {"metric": "batched simulations: aggregate cells x steps/s", "value": value, "unit": "cell-steps/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{len(all_scenes)} plume simulations of uneven sizes (seed 4), plain and learned "
                                   f"mixed, in one batch per GPU, RBGS to FP64 relative residual {TOL:g} each",
                       "sims": len(all_scenes), "sims_rank0": len(scenes), "dims_rank0": dims,
                       "cells": total_cells, "cells_rank0": cells,
                       "learned_sims_rank0": int(learned_mask.sum()),
                       "learned_weights": os.path.relpath(wpath, ROOT) + " (trained at 256^3)" if nets else None,
                       "mean_sweeps": float(sweeps.mean()), "max_sweeps": float(sweeps.max()),
                       "mean_sweeps_plain_sims": float(sweeps[:, ~learned_mask].mean()) if (~learned_mask).any() else None,
                       "mean_sweeps_learned_sims": float(sweeps[:, learned_mask].mean()) if learned_mask.any() else None,
                       "all_converged": all(x["converged"] for fr in stats for x in fr),
                       "batch_sweep_kernel": _batch_kernel_name(stats[0][0]["sweep_variant"]),
                       "per_sim_agreement_with_unbatched": "bitwise, all fields of all sims" if agree else "DIFFERS",
                       "parallelism": f"simulations split over {ws} GPU(s) by cell count (parallel.shard_sims)"},
            "unbatched": {"value": total_cells * args.steps / (ms_alone * 1e-3), "ms_per_step": ms_alone / args.steps,
                          "how": "the same simulations and frames, one solver after another on one stream, each "
                                 "with its own device-loop solve graph"},
            "batch_speedup": ms_alone / ms,
            "gpu_launches": int(launches), "clocks": clk.summary()}


def _batch_kernel_name(v):
    """The batch autotuner's choice as reported in the stats' sweep_variant."""
    if v > 200:
        return f"temporal blocking, two sweeps per pass, tiles of {v - 200} planes, paired-FP32 stencil (autotuned)"
    if v > 100:
        return f"temporal blocking, two sweeps per pass, tiles of {v - 100} planes (autotuned)"
    return f"segment kernel, one sweep per pass, {v} plane(s) per thread (autotuned)"


def plain_sweeps_per_frame(args, local):
    """Sweeps per frame of the plain RBGS step on the timed frames, from a
    plain-only run of this script (same grid, steps and warm-up) in a child
    process, so the reference process itself loads no code of this
    repository's library.  Returns (per-frame list, how)."""
    fixed = os.environ.get(REF_SWEEPS_ENV)
    if fixed:
        return [int(fixed)] * args.steps, f"{REF_SWEEPS_ENV}={fixed} sweeps per frame"
    cmd = [sys.executable, os.path.abspath(__file__), "--plain-only", "--no-cpu", "--no-e2e", "--grid",
           str(args.grid), "--steps", str(args.steps), "--warmup", str(args.warmup), "--max-iter", str(args.max_iter),
           "--workload", args.workload]
    env = dict(os.environ, CUDA_VISIBLE_DEVICES=os.environ.get("CUDA_VISIBLE_DEVICES", str(local)))
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        env.pop(k, None)
    res = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=1800)
    lines = [ln for ln in res.stdout.splitlines() if ln.startswith("{")]
    if res.returncode != 0 or not lines:
        raise RuntimeError("plain run for the reference's sweep counts failed:\n" + res.stderr[-2000:])
    plain = json.loads(lines[-1])["plain"]
    return [int(x) for x in plain["sweeps_per_frame"]], "measured by a plain-only run of this script just before"


def run_reference(args, ws, rank, local):
    if rank != 0:
        return None
    import torch
    from oracle import ref
    from blaze_b200 import BLZ_BC_REF_COMPAT
    if not ref.available():
        return {"impl": "reference", "unavailable": "reference CUDA build (oracle/_ref) not built"}
    sweeps, how = plain_sweeps_per_frame(args, local)
    mean_sweeps = float(np.mean(sweeps))
    torch.cuda.set_device(local)
    scn, frame_parts, desc = make_workload(args, SEED, tol=0.0, max_iter=int(round(mean_sweeps)),
                                           check_every=20, bc_mode=BLZ_BC_REF_COMPAT)
    p = scn.to_params()
    r = ref.RefSolver(p)
    it, t = 0, 0.0

    def frame(n_sweeps):
        nonlocal it, t
        r.set_max_iter(n_sweeps)
        r.set_time(it, t)
        r.set_particles(frame_parts(it))
        r.add_source()
        r.step()
        it += 1
        t += scn.dt

    for _ in range(args.warmup):
        frame(int(round(mean_sweeps)))
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        w0 = time.perf_counter()
        for f in range(args.steps):
            frame(sweeps[f])
        torch.cuda.synchronize()
        wall = time.perf_counter() - w0
    r.close()
    value = args.steps / wall
    return {
        "metric": metric_of(args), "impl": "reference", "value": value, "unit": "steps/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": wall / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{desc} through the reference's "
                               f"own CUDA build (src/FluidSolver.cu, -O3 --use_fast_math, sm_100a), "
                               f"maxIterSolve per frame = the plain RBGS step's sweeps on that frame "
                               f"(mean {mean_sweeps:.0f}; equal sweep count, the reference has no residual "
                               f"control)", "grid": list(scn.gridRes),
                   "sweeps_per_frame": sweeps, "mean_sweeps": mean_sweeps, "sweep_counts": how},
        "ms_per_sweep": wall * 1e3 / float(sum(sweeps)),
        "cpu_baseline": {"value": value, "unit": "steps/s", "cores": 1, "kind": "reference",
                         "sample": "the reference's CUDA build on the same B200 (it has no CPU path); "
                                   "its frame includes the .part file read of an animated source"},
        "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "clocks": clk.summary(),
    }


RENDER_RES = (1280, 720)


def plume_field(n, seed=SEED):
    """A seeded synthetic temperature field shaped like the plume family at
    frame 12: three columns rising from the lower half with mushroom caps,
    smooth, zero elsewhere, with 10 % multiplicative noise; (z, y, x), float32."""
    rng = np.random.default_rng(seed)
    ax = (np.arange(n, dtype=np.float32) + 0.5) / n
    z, y, x = ax[:, None, None], ax[None, :, None], ax[None, None, :]
    T = np.zeros((n, n, n), np.float32)
    for _ in range(3):
        cx, cz = rng.uniform(0.25, 0.75, 2)
        top, r = rng.uniform(0.35, 0.7), rng.uniform(0.06, 0.1)
        yy = 1.0 - y                                   # grid y runs down from the top
        d2 = (x - cx) ** 2 + (z - cz) ** 2
        stem = np.exp(-d2 / (2 * (0.3 * r) ** 2)) * ((yy < top) & (yy > 0.02))
        cap = np.exp(-(d2 / (2 * r * r) + (yy - top) ** 2 / (2 * (0.6 * r) ** 2)))
        T += (1.5 * stem + 2.0 * cap).astype(np.float32)
    T *= (1.0 + 0.1 * rng.standard_normal(T.shape)).astype(np.float32)
    T[T < 1e-3] = 0.0
    return T


def _render_setup(args):
    from blaze_b200.render import default_render_params
    from blaze_b200.scenes import SceneSettings
    n = args.grid
    scn = SceneSettings(gridRes=(n, n, n), dx=1.0 / n)
    rp = default_render_params(scn, width=RENDER_RES[0], height=RENDER_RES[1], lights=1, multi_scatter=True)
    return scn, rp, plume_field(n)


def _render_config(args, rp):
    return {"workload": f"volume render of a {args.grid}^3 temperature field (seeded synthetic plumes) at "
                        f"{rp.width}x{rp.height}, 1 directional light with shadow rays, multiple scattering "
                        f"(3 blur passes), primary step dx, shadow step 2 dx",
            "grid": [args.grid] * 3, "image": [rp.width, rp.height], "lights": rp.light_count,
            "l2": "T (67 MB) exceeds L2 when uploaded; the render reads it through a 3-D texture"}


def run_render(args, ws, rank, local):
    """The renderer (RenderEngine::render, src/RenderEngine.cu:306-365): value
    = renders/s of the device pass (T resident); e2e = T uploaded from pinned
    host memory and the image read back every step, through RenderEngine."""
    import torch
    from blaze_b200.render import RenderEngine
    from blaze_b200.scenes import Timer
    torch.cuda.set_device(local)
    scn, rp, T = _render_setup(args)
    Td = torch.from_numpy(T).cuda()
    eng = RenderEngine(Timer(), scn, rp)
    for _ in range(args.warmup):
        eng.render(Td)
    if ws > 1:
        torch.distributed.barrier()
    l0 = eng.kernel_launches
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        ms_each = [eng.render(Td) for _ in range(args.steps)]
        torch.cuda.synchronize()
    ms = float(sum(ms_each))
    launches = eng.kernel_launches - l0
    img = eng.image()
    e2e = None
    if not args.no_e2e:
        host = torch.from_numpy(T).pin_memory()
        e0 = time.perf_counter()
        for _ in range(args.steps):
            Td.copy_(host, non_blocking=True)
            torch.cuda.current_stream().synchronize()
            eng.render(Td)
            eng.image()
        e2e = args.steps / (time.perf_counter() - e0)
    eng.close()
    if ws > 1:
        t = torch.tensor([ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t[0].item())
    if rank != 0:
        return None
    cpu = None
    if not args.no_cpu:
        from oracle import oracle
        from blaze_b200 import _abi
        g = scn.to_params()
        sub = _abi.BlzRenderParams()
        C_ = __import__("ctypes")
        C_.pointer(sub)[0] = rp
        sub.width, sub.height = rp.width // 8, rp.height // 8          # 1/64 of the pixels, same camera
        c0 = time.perf_counter()
        oracle.render(sub, g, T)
        cs = time.perf_counter() - c0
        cpu = {"value": 1.0 / (cs * 64.0), "unit": "renders/s", "cores": oracle.num_threads(), "kind": "port",
               "sample": f"the oracle's render pass (render_oracle.cpp) at {sub.width}x{sub.height}, the same "
                         f"camera, scaled by the pixel count to {rp.width}x{rp.height} ({cs:.1f} s)"}
    value = ws * args.steps / (ms * 1e-3)
    return {"metric": f"{args.grid}³ volume renders/s at {rp.width}x{rp.height}", "value": value,
            "unit": "renders/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic", "config": _render_config(args, rp),
            "render_ms": ms_each, "image_mean": float(img.mean()), "image_max": float(img.max()),
            "roofline": None,
            "roofline_note": "k_render is bound by texture-filter issue and the latency of dependent ray "
                             "steps, not by HBM bytes or tensor FLOPs (see the k_render ncu summary under profiles/)",
            "cpu_baseline": cpu,
            "e2e": None if e2e is None else {"value": ws * e2e, "unit": "renders/s",
                                             "h2d_bytes_per_step": int(T.nbytes),
                                             "d2h_bytes_per_step": int(img.nbytes)},
            "gpu_launches": int(launches), "clocks": clk.summary()}


def run_render_reference(args, ws, rank, local):
    """The reference's RenderEngine (built from its sources into oracle/_ref)
    on the same field, camera and settings, timed with CUDA events."""
    if rank != 0:
        return None
    import torch
    from oracle import ref
    if not ref.available():
        return {"impl": "reference", "unavailable": "reference CUDA build (oracle/_ref) not built"}
    torch.cuda.set_device(local)
    scn, rp, T = _render_setup(args)
    with ref.RefSolver(scn.to_params()) as sim:
        sim.set("T", T)
        with ref.RefRenderer(sim, rp) as rr:
            for _ in range(args.warmup):
                rr.render()
            with ClockSampler(local) as clk:
                ms_each = [rr.render() for _ in range(args.steps)]
    ms = float(sum(ms_each))
    value = args.steps / (ms * 1e-3)
    return {"metric": f"{args.grid}³ volume renders/s at {rp.width}x{rp.height}", "impl": "reference",
            "value": value, "unit": "renders/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic", "config": _render_config(args, rp), "render_ms": ms_each,
            "cpu_baseline": {"value": value, "unit": "renders/s", "cores": 1, "kind": "reference",
                             "sample": "the reference's RenderEngine (src/RenderEngine.cu, -O3 --use_fast_math, "
                                       "sm_100a) on the same B200 (it has no CPU path)"},
            "e2e": {"value": value, "unit": "renders/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "clocks": clk.summary()}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--grid", type=int, default=GRID)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU oracle baseline")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end (host buffer) pass")
    ap.add_argument("--max-iter", type=int, default=MAX_ITER, help="GS sweep cap per frame (profiling runs)")
    ap.add_argument("--workload", default="plume", choices=["plume", "fire384", "batch", "render"],
                    help="plume: the 256^3 step (default); fire384: the 384^3 large fire with moving emitters; "
                         "batch: 64 uneven simulations in one batch; render: the volume renderer on a 256^3 field")
    ap.add_argument("--batch-sims", type=int, default=64)
    ap.add_argument("--plain-only", action="store_true", help="skip the learned warm-start pass")
    ap.add_argument("--weights", default=None, help="warm-start network weights (npz)")
    ap.add_argument("--host-loop", action="store_true",
                    help="drive the convergence loop from the host (every kernel a separate launch, for launch lists)")
    args = ap.parse_args()
    ws, rank, local = dist_setup()
    if args.impl == "reference":
        # rank 0 alone runs the reference; the other ranks exit without work
        line = (run_render_reference if args.workload == "render" else run_reference)(args, ws, rank, local)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    if ws > 1:
        import torch
        import datetime
        torch.cuda.set_device(local)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        if args.workload == "batch":
            line = run_batch(args, ws, rank, local)
        elif args.workload == "fire384":
            line = run_ours(args, ws, rank, local)
        elif args.workload == "render":
            line = run_render(args, ws, rank, local)
        else:
            line = run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch
            torch.distributed.destroy_process_group()
    if line is not None and rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
