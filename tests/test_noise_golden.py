"""The noise oracle (oracle/noise_oracle.cpp) against the reference's own
noise library (thirdparty/cuda-noise/cuda_noise.cuh, built from its sources
with the reference's flags) at seeded positions: tests/golden/noise.npz,
made by tests/golden/make_noise_golden.py.

Bars:
  - bit for bit (NaN equal to NaN) for every case where the reference build
    compiles the function in its standalone form;
  - call sites where the reference build shares lattice products between
    inlined value-noise blends and fuses the other product of some hash
    sums: bit for bit with that call site's pattern given to the oracle's
    test hook (PATTERNS);
  - faded-value turbulence into cubic value, whose faded offsets use
    unscaled fractions and overflow at most positions: bit for bit at
    >= 99.5 % of positions, the rest within 2e-5 relative or non-finite in
    both.
"""
import json
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
sys.path.insert(0, GOLDEN)

import noise_cases  # noqa: E402

FIXTURE = os.path.join(GOLDEN, "noise.npz")
# Per-call-site lattice patterns of the reference build (see the test hook
# orc_noise_set_lattice_patterns): one entry per value-noise blend in
# evaluation order, the last repeating.
PATTERNS = {
    "repeater_cubicvalue": [0x00cc00cc00cc00cc],
    "turbulence_worley_linearvalue": [0xbb],
    "turbulence_checker_fadedvalue": [0xbb],
    "turbulence_linearvalue_checker": [0x0, 0xbf, 0x0],
}
LOOSE_CASES = {"turbulence_fadedvalue_cubicvalue"}
EXACT_CASES = [n for n in noise_cases.CASES if n not in set(PATTERNS) | LOOSE_CASES]

pytestmark = pytest.mark.skipif(not os.path.exists(FIXTURE), reason="noise fixture not generated")


@pytest.fixture(scope="module")
def gold():
    with np.load(FIXTURE) as z:
        return {k: z[k] for k in z.files}


def bit_mismatch(a, b):
    return (a.view(np.uint32) != b.view(np.uint32)) & ~(np.isnan(a) & np.isnan(b))


def test_fixture_positions_and_reference_repeatability(gold):
    np.testing.assert_array_equal(gold["pos"], noise_cases.positions())
    assert set(gold) - {"pos"} == set(noise_cases.CASES)
    meta = json.load(open(os.path.join(GOLDEN, "noise_meta.json")))
    assert all(v == 0.0 or v != v for v in meta["ref_vs_ref_max_abs"].values())


@pytest.mark.parametrize("name", EXACT_CASES)
def test_oracle_bit_exact(gold, name):
    from oracle import oracle
    got = oracle.noise(noise_cases.args(name), gold["pos"])
    bad = bit_mismatch(got, gold[name])
    assert not bad.any(), f"{bad.sum()} positions differ, e.g. {np.flatnonzero(bad)[:5]}"


@pytest.mark.parametrize("name", sorted(PATTERNS))
def test_oracle_with_call_site_pattern_bit_exact(gold, name):
    from oracle import oracle
    got = oracle.noise(noise_cases.args(name), gold["pos"], PATTERNS[name])
    bad = bit_mismatch(got, gold[name])
    assert not bad.any(), f"{bad.sum()} positions differ"
    # the pattern is what separates the standalone form from that call site
    assert bit_mismatch(oracle.noise(noise_cases.args(name), gold["pos"]), gold[name]).any()


@pytest.mark.parametrize("name", sorted(LOOSE_CASES))
def test_oracle_overflowing_turbulence(gold, name):
    from oracle import oracle
    got = oracle.noise(noise_cases.args(name), gold["pos"])
    want = gold[name]
    bad = bit_mismatch(got, want)
    assert bad.mean() <= 0.005
    both_finite = np.isfinite(got) & np.isfinite(want)
    with np.errstate(invalid="ignore"):
        close = np.abs(got - want) <= 2e-5 * np.maximum(1.0, np.abs(want))
    assert np.all(~bad | (both_finite & close) | (~np.isfinite(got) & ~np.isfinite(want)))


def test_solver_perlin_is_the_library_perlin(gold):
    """The solver's gradient noise (blaze_oracle.cpp, the wind and turbulence
    stages) and the library restatement agree bit for bit."""
    from blaze_b200._abi import noise_args
    from oracle import oracle
    pos = gold["pos"][:500]
    for scale, seed in ((0.4, 99), (1.6, -5)):
        lib = oracle.noise(noise_args("perlin", scale=scale, seed=seed), pos)
        solver = np.array([oracle.perlin(*p, scale, seed) for p in pos], np.float32)
        np.testing.assert_array_equal(lib, solver)


def test_blz_noise_rejects_bad_arguments():
    """Argument checks run before any device call."""
    import ctypes as C
    from blaze_b200 import _abi
    from blaze_b200._lib import load
    lib = load()
    pos = np.zeros((4, 3), np.float32)
    out = np.zeros(4, np.float32)
    for bad in (dict(func=19), dict(func=-1), dict(basis=9), dict(basis_out=-2), dict(octaves=65),
                dict(min_num=5, max_num=4), dict(shape=3)):
        a = _abi.noise_args("repeater")
        for k, v in bad.items():
            setattr(a, k, v)
        assert lib.blz_noise(C.byref(a), pos.ctypes.data, 4, out.ctypes.data, 0, None) == _abi.BLZ_ERR_ARG
        assert b"blz_noise" in lib.blz_last_error(None)
    a = _abi.noise_args("perlin")
    assert lib.blz_noise(C.byref(a), None, 4, out.ctypes.data, 0, None) == _abi.BLZ_ERR_ARG
    assert lib.blz_noise(C.byref(a), pos.ctypes.data, -1, out.ctypes.data, 0, None) == _abi.BLZ_ERR_ARG
    assert lib.blz_noise(C.byref(a), pos.ctypes.data, 0, out.ctypes.data, 0, None) == _abi.BLZ_OK
