"""The renderer's host pieces without a GPU: the oracle's texture sampler and
render pass on cases with known answers, and the image writers
(blz_image_write, the writer behind RenderEngine::writeToDisk,
src/RenderEngine.cu:367-476) read back byte-exactly."""
import ctypes as C
import struct
import zlib

import numpy as np
import pytest

from blaze_b200 import _abi
from blaze_b200.render import default_render_params, render_params_from_blz
from blaze_b200.scenes import SceneSettings
from oracle import oracle


def read_png(path):
    data = open(path, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, w, h = 8, b"", None, None
    while pos < len(data):
        n, = struct.unpack(">I", data[pos:pos + 4])
        typ, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        crc, = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])
        assert crc == zlib.crc32(typ + body) & 0xffffffff
        if typ == b"IHDR":
            w, h, depth, ctype = struct.unpack(">IIBB", body[:10])
            assert depth == 8 and ctype == 6
        elif typ == b"IDAT":
            idat += body
        pos += 12 + n
    raw = zlib.decompress(idat)
    rows = np.frombuffer(raw, np.uint8).reshape(h, 1 + 4 * w)
    assert (rows[:, 0] == 0).all()
    return rows[:, 1:].reshape(h, w, 4)


def read_exr(path):
    data = open(path, "rb").read()
    magic, version = struct.unpack("<II", data[:8])
    assert magic == 20000630 and version == 2
    pos, attrs = 8, {}
    while data[pos] != 0:
        end = data.index(b"\0", pos)
        name = data[pos:end].decode()
        tend = data.index(b"\0", end + 1)
        typ = data[end + 1:tend].decode()
        size, = struct.unpack("<i", data[tend + 1:tend + 5])
        attrs[name] = (typ, data[tend + 5:tend + 5 + size])
        pos = tend + 5 + size
    pos += 1
    xmin, ymin, xmax, ymax = struct.unpack("<4i", attrs["dataWindow"][1])
    w, h = xmax - xmin + 1, ymax - ymin + 1
    assert attrs["compression"][1] == b"\0"
    chl, cpos, names = attrs["channels"][1], 0, []
    while chl[cpos] != 0:
        end = chl.index(b"\0", cpos)
        names.append(chl[cpos:end].decode())
        ptype, = struct.unpack("<i", chl[end + 1:end + 5])
        assert ptype == 2                                              # FLOAT
        cpos = end + 17
    assert names == ["B", "G", "R"]
    offsets = struct.unpack(f"<{h}Q", data[pos:pos + 8 * h])
    img = np.zeros((h, w, 3), np.float32)
    for y, off in enumerate(offsets):
        yy, size = struct.unpack("<ii", data[off:off + 8])
        assert yy == y and size == 12 * w
        line = np.frombuffer(data[off + 8:off + 8 + size], np.float32).reshape(3, w)
        img[y, :, 2], img[y, :, 1], img[y, :, 0] = line[0], line[1], line[2]
    return img


def write(path, rgb):
    from blaze_b200._lib import load
    lib = load()
    a = np.ascontiguousarray(rgb, np.float32)
    rc = lib.blz_image_write(str(path).encode(), a.ctypes.data_as(C.c_void_p), a.shape[1], a.shape[0])
    assert rc == 0, lib.blz_last_error(None)
    return a


@pytest.fixture
def image():
    rng = np.random.default_rng(5)
    img = rng.uniform(-0.2, 1.3, (7, 11, 3)).astype(np.float32)
    img[0, 0] = (0.0, 0.5, 1.0)
    return img


def test_png_round_trip(tmp_path, image):
    write(tmp_path / "a.png", image)
    got = read_png(tmp_path / "a.png")
    want = np.clip((image.astype(np.float64) * 255.0).astype(np.int64), 0, 255)
    np.testing.assert_array_equal(got[..., :3], want)
    assert (got[..., 3] == 255).all()


def test_exr_round_trip(tmp_path, image):
    write(tmp_path / "a.exr", image)
    np.testing.assert_array_equal(read_exr(tmp_path / "a.exr"), image)


def test_ppm_matches_reference_scaling(tmp_path, image):
    write(tmp_path / "a.ppm", image)
    lines = open(tmp_path / "a.ppm").read().split("\n")
    assert lines[:3] == ["P3", "11 7", "255"]
    vals = np.array([[int(v) for v in ln.split()] for ln in lines[3:] if ln], np.int64).reshape(7, 11, 3)
    np.testing.assert_array_equal(vals, (255.99 * image.astype(np.float64)).astype(np.int64))


def test_unknown_extension_is_an_error(tmp_path, image):
    from blaze_b200._lib import load
    a = np.ascontiguousarray(image)
    assert load().blz_image_write(str(tmp_path / "a.jpg").encode(), a.ctypes.data_as(C.c_void_p), 11, 7) == \
        _abi.BLZ_ERR_ARG


def test_sampler_exact_at_texel_centres_and_clamped():
    rng = np.random.default_rng(1)
    T = rng.standard_normal((5, 6, 7)).astype(np.float32)          # (z, y, x)
    k, j, i = np.meshgrid(np.arange(5), np.arange(6), np.arange(7), indexing="ij")
    pos = np.stack([i + 0.5, j + 0.5, k + 0.5], -1).reshape(-1, 3)
    for q in (0, 1, 2, 3):
        np.testing.assert_array_equal(oracle.tex_sample(T, pos, q), T.reshape(-1))
    far = np.array([[-3.0, -3.0, -3.0], [30.0, 30.0, 30.0]], np.float32)
    np.testing.assert_array_equal(oracle.tex_sample(T, far), [T[0, 0, 0], T[-1, -1, -1]])


def test_sampler_is_trilinear_between_centres():
    T = np.zeros((2, 2, 2), np.float32)
    T[1, 1, 1] = 1.0
    pos = np.array([[1.0, 1.0, 1.0]], np.float32)                   # halfway in every axis
    assert oracle.tex_sample(T, pos, 2)[0] == pytest.approx(0.125)
    pos = np.array([[0.5 + 0.3, 0.5, 0.5]], np.float32)             # 0.3 of the way in x only
    T2 = np.zeros((1, 1, 2), np.float32)
    T2[0, 0, 1] = 1.0
    assert oracle.tex_sample(T2, pos, 2)[0] == pytest.approx(0.3, abs=1e-6)
    assert oracle.tex_sample(T2, pos, 0)[0] == pytest.approx(round(0.3 * 256) / 256, abs=1e-7)
    assert oracle.tex_sample(T2, pos, 1)[0] == pytest.approx(int(0.3 * 256) / 256, abs=1e-7)


def _scene(n=16):
    s = SceneSettings(gridRes=(n, n, n), dx=1.0 / n)
    return s, s.to_params()


def test_empty_volume_renders_black():
    s, g = _scene()
    rp = default_render_params(s, width=24, height=16)
    img = oracle.render(rp, g, np.zeros((16, 16, 16), np.float32))
    assert not img.any()


def test_emission_slab_matches_the_closed_form():
    """No lights, one ramp colour, constant T: a ray accumulates
    emission * (1 - dT^N) over its N samples (RenderEngine.cu:225-229)."""
    s, g = _scene()
    rp = default_render_params(s, width=8, height=8, lights=0, multi_scatter=False)
    rp.ramp_size = 1
    for c in range(3):
        rp.ramp_colors[0][c] = (0.2, 0.5, 0.9)[c]
    rp.cutoff = 0.0
    T = np.full((16, 16, 16), 0.7, np.float32)
    img = oracle.render(rp, g, T)
    # the central pixel's ray runs along -z through the whole box
    ext = -(np.array(rp.scattering) + rp.absorption)
    dens = 0.7 * rp.density_scale
    t0 = 1.4 * 1.0                                     # camera at z = 1 + 1.4, box front at z = 1
    t1 = t0 + 1.0
    pt, n = np.float32(t0 + g.dx * 0.5), 0
    while pt <= t1:
        n += 1
        pt = np.float32(pt + np.float32(rp.p_step))
    dT = np.exp(ext * dens * rp.p_step)
    want = np.array([0.2, 0.5, 0.9]) * rp.emission_scale * (1.0 - dT ** n)
    centre = 0.25 * (img[3, 3] + img[3, 4] + img[4, 3] + img[4, 4])
    np.testing.assert_allclose(centre, want, rtol=2e-2)


def test_render_params_from_blz_keys():
    d = {"renderRes": [32, 16], "cam": {"focal": 1.5, "aperture": 0.7, "rotMat": [[1, 0, 0], [0, 1, 0], [0, 0, 1]],
                                        "t": [0.5, 0.5, 3.0]},
         "primarySampleRate": 0.01, "shadowSamplingRate": 0.02, "cutoff": 0.001, "densityScale": 3.0,
         "shadowDensityScale": 0.5, "volumeColor": [1, 1, 1], "scatteringColor": [0.5, 0.6, 0.7], "absorption": 0.1,
         "gain": 0.2, "emissionScale": 1.0, "shaderColorRamp": {"count": 2, "keys": [0, 1],
                                                                 "colors": [[0, 0, 0], [1, 0.5, 0]]},
         "shaderTempRange": [0.1, 2.0], "multiScatterScale": 0.3, "multiScatterDensityMask": [0.1, 0.9],
         "multiScatterColor": [1, 0.5, 0.2], "multiScatterBlurIter": 2, "lightCount": 1,
         "lights": [{"light_exposure": 1.0, "light_intensity": 2.0, "light_samples": 4, "light_dir": [0, -1, 0],
                     "light_color": [1, 1, 1]}]}
    rp = render_params_from_blz(d)
    assert (rp.width, rp.height, rp.ramp_size, rp.light_count, rp.multi_scatter_blur_iter) == (32, 16, 2, 1, 2)
    assert rp.cam_trans[2] == 3.0 and rp.scattering[2] == pytest.approx(0.7) and rp.light_dir[0][1] == -1.0
    assert rp.ramp_colors[1][1] == pytest.approx(0.5) and rp.temp_range[1] == 2.0


@pytest.mark.parametrize("field,value,msg", [
    ("width", 0, "bad render resolution"),
    ("height", -3, "bad render resolution"),
    ("p_step", 0.0, "steps and dx must be positive"),
    ("s_step", float("nan"), "steps and dx must be positive"),
    ("ramp_size", 0, "ramp_size must be 1..10"),
    ("ramp_size", 11, "ramp_size must be 1..10"),
    ("light_count", -1, "light_count must be 0..10"),
    ("light_count", 11, "light_count must be 0..10"),
    ("multi_scatter_blur_iter", -1, "negative multi_scatter_blur_iter"),
])
def test_renderer_rejects_bad_parameters(field, value, msg):
    """blz_render_create checks its arguments before touching the device, and
    leaves the handle null on failure."""
    from blaze_b200._lib import load
    lib = load()
    s, g = _scene()
    rp = default_render_params(s, width=8, height=8)
    setattr(rp, field, value)
    h = C.c_void_p(1)
    assert lib.blz_render_create(C.byref(rp), C.byref(g), C.byref(h)) == _abi.BLZ_ERR_ARG
    assert h.value is None
    assert msg in lib.blz_render_last_error(None).decode()


def test_renderer_rejects_small_grids_and_null_arguments():
    from blaze_b200._lib import load
    lib = load()
    s, g = _scene()
    rp = default_render_params(s, width=8, height=8)
    g.depth = 3
    h = C.c_void_p()
    assert lib.blz_render_create(C.byref(rp), C.byref(g), C.byref(h)) == _abi.BLZ_ERR_ARG
    assert "grid dims must be >= 4" in lib.blz_render_last_error(None).decode()
    assert lib.blz_render_create(None, C.byref(g), C.byref(h)) == _abi.BLZ_ERR_ARG
    assert "null argument" in lib.blz_render_last_error(None).decode()
