"""ctypes mirror of include/blaze_b200.h (structs, constants, prototypes).

Shared by the product binding (``blaze_b200._lib``) and by the test-side
oracle binding, which takes the same ``blz_params`` struct.
"""
import ctypes as C

BLZ_OK = 0
BLZ_ERR_CUDA = -1
BLZ_ERR_ARG = -2
BLZ_ERR_TIMEOUT = -3
BLZ_ERR_NAN = -4
BLZ_ERR_NOCONV = -5
BLZ_ERR_ALLOC = -6
BLZ_ERR_STATE = -7

BLZ_BC_REF_COMPAT = 0
BLZ_BC_FREE_SURFACE = 1
BLZ_GS_RB3D = 0
BLZ_GS_PLANE = 1
BLZ_ADVECT_RK3 = 0
BLZ_ADVECT_EULER = 1
BLZ_ADVECT_RK2 = 2
BLZ_WARM_STEP_RESIDUAL = 0
BLZ_WARM_STEP_ENERGY = 1

FIELD_T, FIELD_U, FIELD_V, FIELD_W, FIELD_P, FIELD_RHS, FIELD_DENSITY = range(7)
FIELD_NAMES = {"T": FIELD_T, "U": FIELD_U, "V": FIELD_V, "W": FIELD_W, "P": FIELD_P, "RHS": FIELD_RHS,
               "DENSITY": FIELD_DENSITY}


class BlzParams(C.Structure):
    _fields_ = [
        ("width", C.c_int), ("height", C.c_int), ("depth", C.c_int),
        ("dx", C.c_float), ("dt", C.c_float),
        ("domain_min", C.c_float * 3), ("domain_max", C.c_float * 3),
        ("closed_bounds", C.c_int * 6),
        ("density", C.c_float), ("gravity", C.c_float), ("buoyancy", C.c_float),
        ("cooling_rate", C.c_float), ("vorticity_conf", C.c_float), ("drag", C.c_float),
        ("wind_dir", C.c_int),
        ("wind_amp", C.c_float), ("wind_speed", C.c_float),
        ("wind_turb_amp", C.c_float), ("wind_turb_scale", C.c_float),
        ("turbulence_amp", C.c_float), ("turbulence_scale", C.c_float),
        ("turb_mask_temp_ramp", C.c_float * 2), ("turb_mask_vel_ramp", C.c_float * 2),
        ("max_iter", C.c_int), ("tol", C.c_double), ("check_every", C.c_int),
        ("bc_mode", C.c_int), ("gs_order", C.c_int), ("reset_pressure", C.c_int),
        ("max_particles", C.c_int), ("temporal_block", C.c_int),
        ("device_loop", C.c_int), ("sweep_variant", C.c_int), ("advect_scheme", C.c_int),
        ("density_field", C.c_int), ("buoyancy_alpha", C.c_float), ("defect_correction", C.c_int),
    ]

    def dims(self):
        return self.width, self.height, self.depth

    def field_shape(self, f):
        """numpy shape (z, y, x) of a field in the reference layout."""
        W, H, D = self.dims()
        if isinstance(f, str):
            f = FIELD_NAMES[f]
        return {FIELD_T: (D, H, W), FIELD_U: (D, H, W + 1), FIELD_V: (D, H + 1, W),
                FIELD_W: (D + 1, H, W), FIELD_P: (D, H, W), FIELD_RHS: (D, H, W), FIELD_DENSITY: (D, H, W)}[f]

    def copy(self):
        p = BlzParams()
        C.pointer(p)[0] = self
        return p

    def as_dict(self):
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if hasattr(v, "__len__") else v
        return out


class BlzStepStats(C.Structure):
    _fields_ = [
        ("iterations", C.c_int), ("converged", C.c_int),
        ("residual", C.c_double), ("rhs_norm", C.c_double), ("rel_residual", C.c_double),
        ("ms_source", C.c_float), ("ms_forces", C.c_float), ("ms_divergence", C.c_float),
        ("ms_solve", C.c_float), ("ms_gradient", C.c_float), ("ms_advect", C.c_float),
        ("ms_total", C.c_float), ("ms_sweeps", C.c_float), ("residual_checks", C.c_int),
        ("sweep_variant", C.c_int), ("device_loop", C.c_int), ("ms_checks", C.c_float),
        ("ms_warm_start", C.c_float), ("warm_started", C.c_int), ("check_interval", C.c_int),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


BLZ_CONV_SLACK = 256
BLZ_SLAB_ALIGN = 16
BLZ_SLAB_HALO = 4


class BlzConvDesc(C.Structure):
    _fields_ = [("W", C.c_int), ("H", C.c_int), ("D", C.c_int), ("cin", C.c_int), ("cout", C.c_int),
                ("relu", C.c_int), ("out_f32", C.c_int)]


BLZ_MAX_LIGHTS = 10
BLZ_MAX_RAMP = 10


class BlzRenderParams(C.Structure):
    _fields_ = [
        ("width", C.c_int), ("height", C.c_int),
        ("cam_focal", C.c_float), ("cam_aperture", C.c_float),
        ("cam_u", C.c_float * 3), ("cam_v", C.c_float * 3), ("cam_w", C.c_float * 3),
        ("cam_trans", C.c_float * 3),
        ("p_step", C.c_float), ("s_step", C.c_float), ("cutoff", C.c_float),
        ("density_scale", C.c_float), ("shadow_density_scale", C.c_float), ("absorption", C.c_float),
        ("scattering", C.c_float * 3), ("volume_color", C.c_float * 3),
        ("gain", C.c_float), ("emission_scale", C.c_float), ("temp_range", C.c_float * 2),
        ("ramp_size", C.c_int), ("ramp_keys", C.c_float * BLZ_MAX_RAMP),
        ("ramp_colors", (C.c_float * 3) * BLZ_MAX_RAMP),
        ("multi_scatter_scale", C.c_float), ("multi_scatter_density_mask", C.c_float * 2),
        ("multi_scatter_color", C.c_float * 3), ("multi_scatter_blur_iter", C.c_int),
        ("light_count", C.c_int),
        ("light_dir", (C.c_float * 3) * BLZ_MAX_LIGHTS), ("light_color", (C.c_float * 3) * BLZ_MAX_LIGHTS),
        ("light_intensity", C.c_float * BLZ_MAX_LIGHTS), ("light_exposure", C.c_float * BLZ_MAX_LIGHTS),
    ]


# Noise functions (blz_noise): ids 0-8 are cuda-noise's basisFunction values.
NOISE_FUNCS = ["checker", "discrete", "linearvalue", "fadedvalue", "cubicvalue", "perlin", "simplex", "worley",
               "spots", "repeater_perlin", "repeater_perlin_bounded", "repeater_perlin_abs", "repeater_simplex",
               "repeater_simplex_abs", "repeater_simplex_bounded", "repeater", "fractal_simplex", "turbulence",
               "repeater_turbulence"]
BLZ_NOISE = {name: i for i, name in enumerate(NOISE_FUNCS)}
BLZ_SHAPE_STEP, BLZ_SHAPE_LINEAR, BLZ_SHAPE_QUADRATIC = 0, 1, 2


class BlzNoiseArgs(C.Structure):
    _fields_ = [
        ("func", C.c_int), ("seed", C.c_int), ("scale", C.c_float), ("scale_out", C.c_float),
        ("size", C.c_float), ("jitter", C.c_float), ("min_num", C.c_int), ("max_num", C.c_int),
        ("shape", C.c_int), ("octaves", C.c_int), ("lacunarity", C.c_float), ("decay", C.c_float),
        ("threshold", C.c_float), ("du", C.c_float), ("strength", C.c_float),
        ("basis", C.c_int), ("basis_out", C.c_int),
    ]


def noise_args(func, **kw):
    """A BlzNoiseArgs for function `func` (name or id); bases may be given by
    name.  Unset fields take the library's usual values (scale 1, octaves 4,
    lacunarity 2, decay 0.5, size 1, jitter 1, 4 points per cell)."""
    a = BlzNoiseArgs()
    a.func = BLZ_NOISE[func] if isinstance(func, str) else int(func)
    a.scale = a.scale_out = a.size = a.jitter = 1.0
    a.min_num = a.max_num = a.octaves = 4
    a.lacunarity, a.decay = 2.0, 0.5
    for k, v in kw.items():
        if k in ("basis", "basis_out") and isinstance(v, str):
            v = BLZ_NOISE[v]
        setattr(a, k, v)
    return a


# Every entry point declared in include/blaze_b200.h, with its ctypes signature.
_P = C.POINTER
EXPORTS = {
    "blz_default_params": (C.c_int, [_P(BlzParams)]),
    "blz_create": (C.c_int, [_P(BlzParams), _P(C.c_void_p)]),
    "blz_destroy": (C.c_int, [C.c_void_p]),
    "blz_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "blz_set_particles": (C.c_int, [C.c_void_p, _P(C.c_float), C.c_int]),
    "blz_set_particles_ex": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    "blz_add_source": (C.c_int, [C.c_void_p]),
    "blz_step": (C.c_int, [C.c_void_p, C.c_float, _P(BlzStepStats)]),
    "blz_forces": (C.c_int, [C.c_void_p, C.c_float]),
    "blz_project": (C.c_int, [C.c_void_p, _P(BlzStepStats)]),
    "blz_divergence": (C.c_int, [C.c_void_p]),
    "blz_solve": (C.c_int, [C.c_void_p, _P(BlzStepStats)]),
    "blz_gradient": (C.c_int, [C.c_void_p]),
    "blz_advect": (C.c_int, [C.c_void_p]),
    "blz_sweeps": (C.c_int, [C.c_void_p, C.c_int]),
    "blz_tight_solve": (C.c_int, [C.c_void_p, C.c_double, C.c_int, C.c_double, _P(C.c_int), _P(C.c_double)]),
    "blz_residual": (C.c_int, [C.c_void_p, _P(C.c_double), _P(C.c_double)]),
    "blz_slab_info": (C.c_int, [C.c_void_p, _P(C.c_int), _P(C.c_int), _P(C.c_longlong)]),
    "blz_slab_get_planes": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]),
    "blz_slab_set_planes": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]),
    "blz_slab_pass": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int]),
    "blz_slab_residual": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, _P(C.c_int), _P(C.c_int)]),
    "blz_reduce_partials": (C.c_int, [C.c_void_p, C.c_void_p, _P(C.c_double), _P(C.c_double)]),
    "blz_get_field": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int]),
    "blz_set_field": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int]),
    "blz_field_size": (C.c_size_t, [C.c_void_p, C.c_int]),
    "blz_field_ptr": (C.c_void_p, [C.c_void_p, C.c_int]),
    "blz_perlin": (C.c_int, [_P(C.c_float), C.c_int, C.c_float, C.c_int, _P(C.c_float)]),
    "blz_noise": (C.c_int, [_P(BlzNoiseArgs), C.c_void_p, C.c_longlong, C.c_void_p, C.c_int, C.c_void_p]),
    "blz_residual_noalloc": (C.c_int, [_P(BlzParams), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "blz_conv3d": (C.c_int, [_P(BlzConvDesc), C.c_void_p, C.c_void_p, _P(C.c_float), C.c_void_p, C.c_void_p]),
    "blz_unet_layer_info": (C.c_int, [C.c_int, _P(C.c_longlong)]),
    "blz_unet_create": (C.c_int, [C.c_int, C.c_int, C.c_int, _P(C.c_void_p)]),
    "blz_unet_destroy": (C.c_int, [C.c_void_p]),
    "blz_unet_num_params": (C.c_longlong, [C.c_void_p]),
    "blz_unet_kernel_launches": (C.c_longlong, [C.c_void_p]),
    "blz_unet_last_alpha": (C.c_float, [C.c_void_p]),
    "blz_unet_set_smoothing": (C.c_int, [C.c_void_p, C.c_int]),
    "blz_unet_set_step": (C.c_int, [C.c_void_p, C.c_int]),
    "blz_unet_set_params": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "blz_unet_get_params": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "blz_unet_get_grads": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "blz_unet_set_kappa": (C.c_int, [C.c_void_p, C.c_float]),
    "blz_unet_forward": (C.c_int, [C.c_void_p, _P(BlzParams), _P(C.c_int), C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p]),
    "blz_unet_loss_grad": (C.c_int, [C.c_void_p, _P(BlzParams), _P(C.c_int), C.c_void_p, C.c_void_p, C.c_void_p,
                                     _P(C.c_double), C.c_void_p]),
    "blz_unet_tensor_shape": (C.c_int, [C.c_void_p, C.c_int, _P(C.c_int)]),
    "blz_unet_get_tensor": (C.c_int, [C.c_void_p, C.c_int, _P(C.c_float), C.c_longlong]),
    "blz_unet_adam": (C.c_int, [C.c_void_p, C.c_float, C.c_float, C.c_float, C.c_float, C.c_void_p]),
    "blz_set_warm_start": (C.c_int, [C.c_void_p, C.c_void_p]),
    "blz_batch_create": (C.c_int, [_P(C.c_void_p), C.c_int, _P(C.c_void_p)]),
    "blz_batch_destroy": (C.c_int, [C.c_void_p]),
    "blz_batch_stream": (C.c_void_p, [C.c_void_p]),
    "blz_batch_set_sweep": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "blz_batch_add_source": (C.c_int, [C.c_void_p]),
    "blz_batch_step": (C.c_int, [C.c_void_p, _P(C.c_float), _P(BlzStepStats)]),
    "blz_batch_solve": (C.c_int, [C.c_void_p, _P(BlzStepStats)]),
    "blz_batch_kernel_launches": (C.c_longlong, [C.c_void_p]),
    "blz_batch_last_ms": (C.c_float, [C.c_void_p]),
    "blz_render_create": (C.c_int, [_P(BlzRenderParams), _P(BlzParams), _P(C.c_void_p)]),
    "blz_render_destroy": (C.c_int, [C.c_void_p]),
    "blz_render_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "blz_render": (C.c_int, [C.c_void_p, C.c_void_p]),
    "blz_render_solver": (C.c_int, [C.c_void_p, C.c_void_p]),
    "blz_render_get_image": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "blz_render_write": (C.c_int, [C.c_void_p, C.c_char_p]),
    "blz_image_write": (C.c_int, [C.c_char_p, C.c_void_p, C.c_int, C.c_int]),
    "blz_render_sample_temp": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "blz_render_last_ms": (C.c_float, [C.c_void_p]),
    "blz_render_kernel_launches": (C.c_longlong, [C.c_void_p]),
    "blz_render_last_error": (C.c_char_p, [C.c_void_p]),
    "blz_kernel_launches": (C.c_longlong, [C.c_void_p]),
    "blz_last_error": (C.c_char_p, [C.c_void_p]),
}


def bind(lib, exports=EXPORTS):
    for name, (res, args) in exports.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib
