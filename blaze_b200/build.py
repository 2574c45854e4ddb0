"""Builds libblaze_b200.so in-tree with nvcc for sm_100a.

``python -m blaze_b200.build`` or ``blaze_b200.build.build()``.  The library
lands in ``blaze_b200/lib/`` next to the sources so that it travels with the
working tree; nothing is installed into site-packages.
"""
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libblaze_b200.so")
SOURCES = ["k_source.cu", "k_forces.cu", "k_project.cu", "k_advect.cu", "graph_solve.cu", "solver.cu",
           "unet_conv.cu", "unet.cu", "batch.cu", "render.cu",
           "noalloc.cu", "noise.cu", "tight.cu"]
HEADERS = ["common.cuh", "kernels.cuh", "noise.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-shared"] + ARCH


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, ptxas_info=False):
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, h) for h in HEADERS] + \
        [os.path.join(os.path.dirname(PKG), "include", "blaze_b200.h")]
    if not force and not _stale(LIB, deps):
        return LIB
    cmd = [_nvcc()] + NVCC_FLAGS + (["-Xptxas", "-v"] if ptxas_info else []) + ["-o", LIB] + srcs
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stdout + res.stderr)
    if verbose or ptxas_info:
        sys.stderr.write(res.stderr)
    return LIB


SHIM_SRC = os.path.join(PKG, "shim", "FluidSolver_blaze.cu")
SHIM_LIB = os.path.join(LIBDIR, "libblaze_fluidsolver.so")


def build_shim(ref_src, force=False, verbose=False):
    """Builds the drop-in FluidSolver (shim/FluidSolver_blaze.cu) against the
    reference's own headers in `ref_src` (its src/ directory), linked to
    libblaze_b200.so.  Returns None when those headers are absent."""
    if not os.path.exists(os.path.join(ref_src, "FluidSolver.h")):
        return None
    build(verbose=verbose)
    if not force and not _stale(SHIM_LIB, [SHIM_SRC, LIB]):
        return SHIM_LIB
    cmd = [_nvcc(), "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared"] + ARCH + [
        "-I", ref_src, "-I", os.path.join(os.path.dirname(PKG), "include"),
        "-diag-suppress", "177,550,3012,20012,20013,20014,20015",
        "-Xcompiler", "-Wno-format-overflow", "-o", SHIM_LIB, SHIM_SRC,
        "-L", LIBDIR, "-lblaze_b200", "-Xlinker", "-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc (shim) failed:\n" + res.stdout + res.stderr)
    return SHIM_LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
