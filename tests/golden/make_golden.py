"""Generates tests/golden/*.npz from the reference's own CUDA build.

Runs on a CUDA machine with oracle/_ref/libblaze_ref.so built (make -C oracle
ref, from the reference sources).  Each case of cases.py is run twice; the
first run's outputs are written, and the largest difference between the two
runs (the reference's run-to-run spread: float atomics, racy boundary copy)
goes to meta.json.

    python tests/golden/make_golden.py [out_dir]
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import cases  # noqa: E402
from oracle import ref  # noqa: E402


def run_case(name):
    ovr, stage, seed, time, outs = cases.CASES[name]
    p = cases.scene(**ovr).to_params()
    with ref.RefSolver(p) as r:
        r.set_time(0, time)
        for k, v in cases.inputs(p, seed).items():
            r.set(k, v)
        if stage == "source":
            r.set_particles(cases.particles(p, seed))
            r.add_source()
        elif stage == "step":
            parts = cases.particles(p, seed)
            for n in range(cases.STEP_FRAMES):
                r.set_time(n, n * p.dt)
                r.set_particles(parts)
                r.add_source()
                r.step()
        else:
            r.stage(stage)
        return {f: r.get(f) for f in outs}


def perlin_case():
    rng = np.random.default_rng(7)
    pos = np.concatenate([rng.uniform(-20, 300, (1500, 3)), rng.uniform(0, 25000, (500, 3))]).astype(np.float32)
    out = {"pos": pos}
    for scale, seed in ((0.25, 123), (1.6, 456), (0.125, 789)):
        out[f"n_{scale}_{seed}"] = ref.perlin(pos, scale, seed)
    return out


def main(out_dir):
    os.makedirs(out_dir, exist_ok=True)
    meta = {}
    for name in cases.CASES:
        a, b = run_case(name), run_case(name)
        np.savez_compressed(os.path.join(out_dir, f"{name}.npz"), **a)
        meta[name] = {f: float(np.max(np.abs(a[f].astype(np.float64) - b[f]))) for f in a}
        print(name, "ref-vs-ref max |diff|:", meta[name], flush=True)
    np.savez_compressed(os.path.join(out_dir, "perlin.npz"), **perlin_case())
    with open(os.path.join(out_dir, "meta.json"), "w") as f:
        json.dump({"ref_vs_ref_max_abs": meta, "dims": cases.DIMS}, f, indent=1)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
