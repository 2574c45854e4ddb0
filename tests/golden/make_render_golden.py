"""Generates tests/golden/render.npz from the reference's own RenderEngine.

Runs on a CUDA machine with oracle/_ref/libblaze_ref.so built (make -C oracle
ref, from the reference sources).  Each case of render_cases.py is rendered
twice by the reference; the first image is written and the largest
difference between the two renders goes to render_meta.json.

    python tests/golden/make_render_golden.py [out_dir]
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import render_cases  # noqa: E402
from oracle import ref  # noqa: E402


def render_case(name):
    _, g, rp, T = render_cases.setup(name)
    with ref.RefSolver(g.copy()) as sim:
        sim.set("T", T)
        with ref.RefRenderer(sim, rp) as rr:
            rr.render()
            return rr.image()


def main(out_dir):
    os.makedirs(out_dir, exist_ok=True)
    images, meta = {}, {}
    for name in render_cases.CASES:
        a, b = render_case(name), render_case(name)
        images[name] = a
        meta[name] = float(np.max(np.abs(a.astype(np.float64) - b)))
        print(name, "max", float(a.max()), "ref-vs-ref max |diff|:", meta[name], flush=True)
    np.savez_compressed(os.path.join(out_dir, "render.npz"), **images)
    with open(os.path.join(out_dir, "render_meta.json"), "w") as f:
        json.dump({"ref_vs_ref_max_abs": meta, "n": render_cases.N,
                   "image": [render_cases.WIDTH, render_cases.HEIGHT]}, f, indent=1)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
