"""blz_noise (noise.cu) on the GPU against the reference's own noise library
(tests/golden/noise.npz, from the reference's CUDA build) and against the
oracle (oracle/noise_oracle.cpp), at the fixture's seeded positions.

Bars, bit for bit (NaN equal to NaN) throughout:
  - reference: every case the reference build compiles in the library's
    standalone form; the call sites with their own lattice patterns and the
    overflowing faded turbulence are compared with the oracle only;
  - oracle: every case.
"""
import ctypes as C
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import noise_cases  # noqa: E402

pytestmark = pytest.mark.gpu

FIXTURE = os.path.join(HERE, "golden", "noise.npz")
OWN_PATTERN = {"repeater_cubicvalue", "turbulence_worley_linearvalue", "turbulence_checker_fadedvalue",
               "turbulence_linearvalue_checker", "turbulence_fadedvalue_cubicvalue"}


def bit_mismatch(a, b):
    return (a.view(np.uint32) != b.view(np.uint32)) & ~(np.isnan(a) & np.isnan(b))


def blz_noise(args, pos):
    from blaze_b200 import _lib
    lib = _lib.load()
    p = np.ascontiguousarray(pos, np.float32)
    out = np.empty(len(p), np.float32)
    _lib.check(lib.blz_noise(C.byref(args), p.ctypes.data, len(p), out.ctypes.data, 0, None))
    return out


@pytest.fixture(scope="module")
def gold():
    with np.load(FIXTURE) as z:
        return {k: z[k] for k in z.files}


@pytest.mark.parametrize("name", [n for n in noise_cases.CASES if n not in OWN_PATTERN])
def test_blz_noise_equals_reference_build(gold, name):
    got = blz_noise(noise_cases.args(name), gold["pos"])
    bad = bit_mismatch(got, gold[name])
    print(f"{name}: {bad.sum()} of {len(got)} differ from the reference build")
    assert not bad.any()


@pytest.mark.parametrize("name", list(noise_cases.CASES))
def test_blz_noise_equals_oracle(gold, name):
    from oracle import oracle
    got = blz_noise(noise_cases.args(name), gold["pos"])
    want = oracle.noise(noise_cases.args(name), gold["pos"])
    bad = bit_mismatch(got, want)
    assert not bad.any(), f"{bad.sum()} positions differ, e.g. {np.flatnonzero(bad)[:5]}"


def test_device_buffers_on_a_stream_equal_host_buffers(gold):
    import torch
    from blaze_b200 import _abi, _lib
    lib = _lib.load()
    rng = np.random.default_rng(8)
    pos = rng.uniform(-50, 400, (300_000, 3)).astype(np.float32)
    for name in ("simplex", "worley", "repeater_perlin", "turbulence_perlin_simplex"):
        a = noise_cases.args(name)
        host = blz_noise(a, pos)
        s = torch.cuda.Stream()
        dpos = torch.from_numpy(pos).cuda()
        dout = torch.empty(len(pos), device="cuda")
        with torch.cuda.stream(s):
            _lib.check(lib.blz_noise(C.byref(a), dpos.data_ptr(), len(pos), dout.data_ptr(), 1,
                                     C.c_void_p(s.cuda_stream)))
        s.synchronize()
        np.testing.assert_array_equal(dout.cpu().numpy(), host)
    assert _abi.BLZ_NOISE["spots"] == 8
