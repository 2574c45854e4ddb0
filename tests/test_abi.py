"""The C-ABI library loads and exports every symbol include/blaze_b200.h
declares; the ctypes structs match the C layout; argument checks work without
a GPU.  CPU only (no compute calls)."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from blaze_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", h) for h in sorted(os.listdir(os.path.join(ROOT, "include"))) if h.endswith(".h")]


def declared():
    names = set()
    for h in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        names |= set(re.findall(r"\b(blz_\w+)\s*\(", text))
    return names


@pytest.fixture(scope="module")
def lib():
    from blaze_b200 import build
    path = build.build()
    return C.CDLL(path)


def test_every_declared_symbol_is_exported(lib):
    names = declared()
    assert "blz_step" in names and "blz_create" in names
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_ctypes_table_covers_header():
    assert declared() == set(_abi.EXPORTS)


def test_struct_layout_matches_c(tmp_path):
    src = tmp_path / "layout.c"
    fields = [f for f, _ in _abi.BlzParams._fields_]
    sfields = [f for f, _ in _abi.BlzStepStats._fields_]
    nfields = [f for f, _ in _abi.BlzNoiseArgs._fields_]
    body = "".join(f'printf("p {f} %zu\\n", offsetof(blz_params, {f}));' for f in fields)
    body += "".join(f'printf("s {f} %zu\\n", offsetof(blz_step_stats, {f}));' for f in sfields)
    body += "".join(f'printf("n {f} %zu\\n", offsetof(blz_noise_args, {f}));' for f in nfields)
    src.write_text(f'#include <stdio.h>\n#include <stddef.h>\n#include "blaze_b200.h"\nint main(void){{'
                   f'printf("P %zu\\nS %zu\\nN %zu\\n", sizeof(blz_params), sizeof(blz_step_stats), '
                   f'sizeof(blz_noise_args));{body} return 0;}}\n')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {}
    for line in out:
        parts = line.split()
        if len(parts) == 2:
            got[parts[0]] = int(parts[1])
        elif len(parts) == 3:
            got[(parts[0], parts[1])] = int(parts[2])
    assert got["P"] == C.sizeof(_abi.BlzParams)
    assert got["S"] == C.sizeof(_abi.BlzStepStats)
    for f in fields:
        assert got[("p", f)] == getattr(_abi.BlzParams, f).offset, f
    for f in sfields:
        assert got[("s", f)] == getattr(_abi.BlzStepStats, f).offset, f
    assert got["N"] == C.sizeof(_abi.BlzNoiseArgs)
    for f in nfields:
        assert got[("n", f)] == getattr(_abi.BlzNoiseArgs, f).offset, f


def test_argument_checks_need_no_gpu(lib):
    _abi.bind(lib)
    p = _abi.BlzParams()
    assert lib.blz_default_params(C.byref(p)) == 0
    assert p.density == pytest.approx(0.1) and p.max_iter == 200
    h = C.c_void_p()
    # 1290^3: (W + 1)(H + 1)(D + 1) reaches 2^31, past 32-bit field offsets
    for bad in (dict(width=3), dict(width=15), dict(dx=0.0), dict(bc_mode=7), dict(max_iter=-1),
                dict(width=1290, height=1290, depth=1290)):
        q = p.copy()
        for k, v in bad.items():
            setattr(q, k, v)
        assert lib.blz_create(C.byref(q), C.byref(h)) == _abi.BLZ_ERR_ARG
        assert lib.blz_last_error(None)
    assert lib.blz_create(None, C.byref(h)) == _abi.BLZ_ERR_ARG
    assert lib.blz_set_particles(None, None, 0) == _abi.BLZ_ERR_ARG


def _err(lib):
    return lib.blz_last_error(None).decode()


def test_warm_start_and_batch_argument_checks_need_no_gpu(lib):
    """The network's and the batch's entry points reject bad arguments before
    any device call, and say why in the thread's last error."""
    _abi.bind(lib)
    h = C.c_void_p(1)
    for dims in ((0, 8, 8), (12, 16, 16), (16, 16, 4), (-8, 8, 8)):
        assert lib.blz_unet_create(*dims, C.byref(h)) == _abi.BLZ_ERR_ARG
        assert h.value is None and "multiples of 8" in _err(lib)
    assert lib.blz_unet_create(8, 8, 8, None) == _abi.BLZ_ERR_ARG
    assert lib.blz_unet_set_smoothing(None, 10) == _abi.BLZ_ERR_ARG
    assert lib.blz_unet_set_step(None, _abi.BLZ_WARM_STEP_ENERGY) == _abi.BLZ_ERR_ARG
    assert "step mode" in _err(lib)
    assert lib.blz_unet_set_kappa(None, 0.5) == _abi.BLZ_ERR_ARG
    assert lib.blz_unet_set_params(None, None, 0) == _abi.BLZ_ERR_ARG
    assert lib.blz_unet_get_params(None, None, 0) == _abi.BLZ_ERR_ARG
    assert lib.blz_unet_get_grads(None, None, 0) == _abi.BLZ_ERR_ARG
    info = (C.c_longlong * 6)()
    for layer in (-1, 10 ** 6):
        assert lib.blz_unet_layer_info(layer, info) == _abi.BLZ_ERR_ARG
        assert f"no layer {layer}" in _err(lib)
    assert lib.blz_unet_layer_info(0, info) == 0 and (info[0], info[3]) == (0, 27) and info[1] > 0
    assert lib.blz_batch_create(None, 0, C.byref(h)) == _abi.BLZ_ERR_ARG
    assert "at least one solver" in _err(lib)
    sims = (C.c_void_p * 2)(None, None)
    assert lib.blz_batch_create(sims, 2, C.byref(h)) == _abi.BLZ_ERR_ARG
    assert "solver 0 is null" in _err(lib)
    assert lib.blz_batch_add_source(None) == _abi.BLZ_ERR_ARG
    assert lib.blz_batch_solve(None, None) == _abi.BLZ_ERR_ARG
    assert lib.blz_batch_step(None, None, None) == _abi.BLZ_ERR_ARG
    assert "null batch" in _err(lib)
    assert lib.blz_batch_set_sweep(None, 16, 0) == _abi.BLZ_ERR_ARG
    assert "null batch" in _err(lib)
    assert lib.blz_unet_create(648, 648, 648, C.byref(h)) == _abi.BLZ_ERR_ARG
    assert "2^28" in _err(lib)


def test_slab_entry_points_refuse_null_arguments(lib):
    """The z-slab solve's entry points reject a null solver or null outputs
    before any device call."""
    _abi.bind(lib)
    ok, n, pf = C.c_int(), C.c_int(), C.c_longlong()
    assert lib.blz_slab_info(None, C.byref(ok), C.byref(n), C.byref(pf)) == _abi.BLZ_ERR_ARG
    assert lib.blz_slab_get_planes(None, 0, 0, 0, 1, None) == _abi.BLZ_ERR_ARG
    assert lib.blz_slab_set_planes(None, 0, 0, 0, 1, None) == _abi.BLZ_ERR_ARG
    assert lib.blz_slab_pass(None, 0, 16, 0) == _abi.BLZ_ERR_ARG
    first, count = C.c_int(), C.c_int()
    assert lib.blz_slab_residual(None, 0, 16, None, C.byref(first), C.byref(count)) == _abi.BLZ_ERR_ARG
    r, b = C.c_double(), C.c_double()
    assert lib.blz_reduce_partials(None, None, C.byref(r), C.byref(b)) == _abi.BLZ_ERR_ARG
    assert _abi.BLZ_SLAB_ALIGN == 16 and _abi.BLZ_SLAB_HALO == 4


def test_noalloc_residual_argument_checks_need_no_gpu(lib):
    """The allocation-free residual refuses what blz_create refuses (an
    unknown bc_mode, bad dims, non-positive dx/dt/density) and grids deeper
    than its static scratch, before any device call."""
    _abi.bind(lib)
    p = _abi.BlzParams()
    assert lib.blz_default_params(C.byref(p)) == 0
    p.width, p.height, p.depth = 16, 16, 16
    dummy = C.c_void_p(256)                               # never dereferenced: rejected first
    for bad, words in ((dict(bc_mode=7), "bc_mode"), (dict(bc_mode=-1), "bc_mode"), (dict(width=3), ">= 4"),
                       (dict(dt=0.0), "positive"), (dict(depth=4097), "4096")):
        q = p.copy()
        for k, v in bad.items():
            setattr(q, k, v)
        assert lib.blz_residual_noalloc(C.byref(q), dummy, dummy, dummy, None) == _abi.BLZ_ERR_ARG
        assert words in _err(lib), (bad, _err(lib))
    assert lib.blz_residual_noalloc(C.byref(p), None, dummy, dummy, None) == _abi.BLZ_ERR_ARG


def test_oracle_library_loads(oracle_mod):
    assert oracle_mod.num_threads() >= 1
