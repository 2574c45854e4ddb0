"""Python host API of the CUDA volume renderer, named after the reference's
``class RenderEngine`` (src/RenderEngine.h:46-95):

    rp = render_params_from_blz(scene.raw)        # or default_render_params(...)
    engine = RenderEngine(tmr, scene.settings, rp)
    engine.render(solver)                         # RenderEngine::render(getTempGrid())
    engine.writeToDisk(scene)                     # <sceneDir>/<renderFile stem>_<iter>.<ext>

All work runs in libblaze_b200.so (render.cu); this module fills the
parameter struct and moves the image to the host.
"""
import ctypes as C
import math
import os

import numpy as np

from . import _abi
from ._lib import BlazeError, load


def _check(lib, rc, handle):
    if rc != _abi.BLZ_OK:
        raise BlazeError(rc, lib.blz_render_last_error(handle).decode(errors="replace"))


def _set3(arr, v):
    for i in range(3):
        arr[i] = float(v[i])


def render_params_from_blz(d):
    """blz_render_params from a .blz scene's JSON, with the reference's keys
    (src/Parser.h:73-75, 109-170)."""
    rp = _abi.BlzRenderParams()
    rp.width, rp.height = int(d["renderRes"][0]), int(d["renderRes"][1])
    cam = d["cam"]
    rp.cam_focal, rp.cam_aperture = float(cam["focal"]), float(cam["aperture"])
    _set3(rp.cam_u, cam["rotMat"][0])
    _set3(rp.cam_v, cam["rotMat"][1])
    _set3(rp.cam_w, cam["rotMat"][2])
    _set3(rp.cam_trans, cam["t"])
    rp.p_step, rp.s_step, rp.cutoff = (float(d["primarySampleRate"]), float(d["shadowSamplingRate"]),
                                       float(d["cutoff"]))
    rp.density_scale, rp.shadow_density_scale = float(d["densityScale"]), float(d["shadowDensityScale"])
    _set3(rp.volume_color, d["volumeColor"])
    _set3(rp.scattering, d["scatteringColor"])
    rp.absorption, rp.gain = float(d["absorption"]), float(d["gain"])
    rp.emission_scale = float(d["emissionScale"])
    ramp = d["shaderColorRamp"]
    rp.ramp_size = int(ramp["count"])
    rp.temp_range[0], rp.temp_range[1] = float(d["shaderTempRange"][0]), float(d["shaderTempRange"][1])
    for i in range(rp.ramp_size):
        rp.ramp_keys[i] = float(ramp["keys"][i])
        _set3(rp.ramp_colors[i], ramp["colors"][i])
    rp.multi_scatter_scale = float(d["multiScatterScale"])
    rp.multi_scatter_density_mask[0] = float(d["multiScatterDensityMask"][0])
    rp.multi_scatter_density_mask[1] = float(d["multiScatterDensityMask"][1])
    _set3(rp.multi_scatter_color, d["multiScatterColor"])
    rp.multi_scatter_blur_iter = int(d["multiScatterBlurIter"])
    rp.light_count = int(d["lightCount"])
    for i in range(rp.light_count):
        L = d["lights"][i]
        rp.light_exposure[i], rp.light_intensity[i] = float(L["light_exposure"]), float(L["light_intensity"])
        _set3(rp.light_dir[i], L["light_dir"])
        _set3(rp.light_color[i], L["light_color"])
    return rp


def default_render_params(settings, width=640, height=360, lights=1, multi_scatter=True):
    """A camera on +z looking down -z at the whole domain, a fire-like
    temperature ramp and `lights` directional lights from above: settings for
    synthetic scenes (the reference's demo scenes are not distributed)."""
    rp = _abi.BlzRenderParams()
    rp.width, rp.height = width, height
    lo, hi = np.array(settings.domainBboxMin, float), np.array(settings.domainBboxMax, float)
    ctr, size = 0.5 * (lo + hi), float((hi - lo).max())
    rp.cam_focal, rp.cam_aperture = 1.0, 0.6
    _set3(rp.cam_u, (1, 0, 0))
    _set3(rp.cam_v, (0, 1, 0))
    _set3(rp.cam_w, (0, 0, 1))
    _set3(rp.cam_trans, (ctr[0], ctr[1], hi[2] + 1.4 * size))
    rp.p_step, rp.s_step = float(settings.dx), 2.0 * float(settings.dx)
    rp.cutoff = 1e-4
    rp.density_scale, rp.shadow_density_scale = 8.0 / size, 1.0
    _set3(rp.volume_color, (1.0, 1.0, 1.0))
    _set3(rp.scattering, (0.8, 0.8, 0.8))
    rp.absorption, rp.gain = 0.2, 0.5
    rp.emission_scale = 0.6
    rp.temp_range[0], rp.temp_range[1] = 0.05, 2.0
    keys = [0.0, 0.35, 0.7, 1.0]
    colors = [(0.0, 0.0, 0.0), (0.6, 0.1, 0.0), (1.0, 0.5, 0.1), (1.0, 0.9, 0.6)]
    rp.ramp_size = len(keys)
    for i, (k, c) in enumerate(zip(keys, colors)):
        rp.ramp_keys[i] = k
        _set3(rp.ramp_colors[i], c)
    rp.multi_scatter_scale = 0.5 if multi_scatter else 0.0
    rp.multi_scatter_density_mask[0], rp.multi_scatter_density_mask[1] = 0.1, 1.0
    _set3(rp.multi_scatter_color, (1.0, 0.6, 0.3))
    rp.multi_scatter_blur_iter = 3 if multi_scatter else 0
    rp.light_count = lights
    dirs = [(0.3, -1.0, -0.4), (-0.5, -0.6, 0.6), (0.0, -1.0, 0.0)]
    for i in range(lights):
        d = np.array(dirs[i % len(dirs)], float)
        _set3(rp.light_dir[i], d / np.linalg.norm(d))
        _set3(rp.light_color[i], (1.0, 0.95, 0.9))
        rp.light_intensity[i], rp.light_exposure[i] = 1.0, 0.5
    return rp


def render_file_name(scene, frame):
    """The reference's output path (RenderEngine.cu:371-379): renderFile minus
    its last 9 characters ("_####.exr"), then _%04d of the frame and the
    file's 3-letter extension, inside the scene's directory."""
    rf = scene.raw["renderFile"]
    return os.path.join(scene.scene_dir, f"{rf[:-9]}_{frame:04d}.{rf[-3:]}")


class RenderEngine:
    def __init__(self, tmr, settings, render_params, stream=None):
        self._lib = load()
        self.tmr = tmr
        self.grid = settings.to_params() if hasattr(settings, "to_params") else settings
        self.rp = render_params
        h = C.c_void_p()
        _check(self._lib, self._lib.blz_render_create(C.byref(self.rp), C.byref(self.grid), C.byref(h)), None)
        self._h = h
        if stream is not None:
            _check(self._lib, self._lib.blz_render_set_stream(self._h, C.c_void_p(stream)), self._h)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.blz_render_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def render(self, temp):
        """Renders a FluidSolver's temperature field, or a T field already in
        device memory (a device pointer, or an object with data_ptr())."""
        if hasattr(temp, "_h") and hasattr(temp, "getTempGrid"):
            rc = self._lib.blz_render_solver(self._h, temp._h)
        else:
            ptr = temp.data_ptr() if hasattr(temp, "data_ptr") else int(temp)
            rc = self._lib.blz_render(self._h, C.c_void_p(ptr))
        _check(self._lib, rc, self._h)
        return self.last_ms

    def image(self):
        """The frame buffer as a (height, width, 3) float32 array."""
        out = np.empty((self.rp.height, self.rp.width, 3), np.float32)
        _check(self._lib, self._lib.blz_render_get_image(self._h, out.ctypes.data_as(C.c_void_p), 0), self._h)
        return out

    def writeToDisk(self, path_or_scene):
        """Writes the frame buffer: to a path (.ppm, .png or .exr), or for a
        SceneFile to the reference's per-frame name for tmr.iter, creating
        its directory (RenderEngine.cu:367-383)."""
        path = path_or_scene
        if not isinstance(path_or_scene, (str, os.PathLike)):
            path = render_file_name(path_or_scene, self.tmr.iter)
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        _check(self._lib, self._lib.blz_render_write(self._h, os.fsencode(path)), self._h)
        return path

    def sample_temp(self, temp_ptr, pos_ptr, n, out_ptr):
        """Samples T through the renderer's texture (test hook; device pointers)."""
        _check(self._lib, self._lib.blz_render_sample_temp(self._h, C.c_void_p(temp_ptr), C.c_void_p(pos_ptr), int(n),
                                                           C.c_void_p(out_ptr)), self._h)

    @property
    def last_ms(self):
        return float(self._lib.blz_render_last_ms(self._h))

    @property
    def kernel_launches(self):
        return int(self._lib.blz_render_kernel_launches(self._h))
