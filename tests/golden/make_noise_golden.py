"""Generates tests/golden/noise.npz from the reference's own noise library.

Runs on a CUDA machine with oracle/_ref/libblaze_ref.so built (make -C oracle
ref, from the reference sources).  Each case of noise_cases.py is evaluated
twice at noise_cases.positions(); the first result is written, and the
largest difference between the two runs goes to noise_meta.json.

    python tests/golden/make_noise_golden.py [out_dir]
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import noise_cases  # noqa: E402
from oracle import ref  # noqa: E402


def main(out_dir):
    os.makedirs(out_dir, exist_ok=True)
    pos = noise_cases.positions()
    out, meta = {"pos": pos}, {}
    for name in noise_cases.CASES:
        a = ref.noise(noise_cases.args(name), pos)
        b = ref.noise(noise_cases.args(name), pos)
        out[name] = a
        meta[name] = float(np.max(np.abs(a.astype(np.float64) - b)))
        print(f"{name}: range [{a.min():.4f}, {a.max():.4f}] ref-vs-ref {meta[name]}", flush=True)
    np.savez_compressed(os.path.join(out_dir, "noise.npz"), **out)
    with open(os.path.join(out_dir, "noise_meta.json"), "w") as f:
        json.dump({"ref_vs_ref_max_abs": meta, "positions": len(pos)}, f, indent=1)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
