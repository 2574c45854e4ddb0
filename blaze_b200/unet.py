"""Learned warm start of the pressure solve: Python handle over the
``blz_unet_*`` entry points of libblaze_b200.so.

    net = WarmStartUNet((256, 256, 256))
    net.load("blaze_b200/weights/plume256.npz")
    solver.set_warm_start(net)          # every later solve starts from the network

The network, its kernels and its training step live in the CUDA library
(csrc/unet.cu, csrc/unet_conv.cu); this module moves parameters between host
and device, reads and writes the weight files, and passes device pointers of
torch tensors.  No counterpart in the reference, which has no learned parts.
"""
import ctypes as C
import json
import os

import numpy as np

from . import _abi
from ._lib import check, load

KIND_CONV3, KIND_UP, KIND_HEAD = 0, 1, 2
LAYER_NAMES = ["e0a", "e0b", "e1a", "e1b", "e2a", "e2b", "e3a", "e3b",
               "d2a", "d2b", "d1a", "d1b", "d0a", "d0b", "u2", "u1", "u0", "head"]
TENSOR_NAMES = ["X0", "e0a", "cat0", "d0a", "d0b", "p1", "e1a", "cat1", "d1a", "d1b", "p2", "e2a", "cat2", "d2a",
                "d2b", "p3", "e3a", "e3b", "g_d0b", "g_d0a", "g_cat0", "g_e0b", "g_e0a", "g_p1", "g_d1b", "g_d1a",
                "g_cat1", "g_e1b", "g_e1a", "g_p2", "g_d2b", "g_d2a", "g_cat2", "g_e2b", "g_e2a", "g_p3", "g_e3b",
                "g_e3a"]
WEIGHTS_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights")


def layers():
    """The library's layer table: one dict per layer (kind, cin, cout, taps,
    weight and bias offsets into the flat parameter array)."""
    lib = load()
    out = []
    info = (C.c_longlong * 6)()
    for i, name in enumerate(LAYER_NAMES):
        check(lib.blz_unet_layer_info(i, info))
        out.append({"name": name, "kind": int(info[0]), "cin": int(info[1]), "cout": int(info[2]),
                    "taps": int(info[3]), "w_off": int(info[4]), "b_off": int(info[5])})
    return out


def num_params():
    last = layers()[-1]
    return last["b_off"] + last["cout"]


def init_params(seed=0):
    """He-normal weights for the ReLU layers, zero biases, a small head (PCG
    seeded numpy generator)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(num_params(), np.float32)
    for L in layers():
        n = L["taps"] * L["cout"] * L["cin"]
        if L["kind"] == KIND_CONV3:
            std = np.sqrt(2.0 / (27 * L["cin"]))
        elif L["kind"] == KIND_UP:
            std = np.sqrt(1.0 / L["cin"])
        else:
            std = 0.1 / np.sqrt(L["cin"])
        p[L["w_off"]:L["w_off"] + n] = rng.standard_normal(n).astype(np.float32) * std
    return p


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _stream_handle(stream):
    if stream is None:
        import torch
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)
    return C.c_void_p(stream)


class WarmStartUNet:
    """One network instance for a crop of dims (W, H, D), multiples of 8."""

    def __init__(self, dims, params=None, kappa=1.0):
        self._lib = load()
        self.dims = tuple(int(d) for d in dims)
        h = C.c_void_p()
        check(self._lib.blz_unet_create(*self.dims, C.byref(h)))
        self._h = h
        self.n_params = int(self._lib.blz_unet_num_params(h))
        self.kappa = float(kappa)
        self.meta = {}
        check(self._lib.blz_unet_set_kappa(h, C.c_float(self.kappa)))
        if params is not None:
            self.set_params(params)

    # -- lifetime ---------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._lib.blz_unet_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # -- parameters ---------------------------------------------------------------
    def set_params(self, params):
        if hasattr(params, "data_ptr"):
            assert params.numel() == self.n_params and params.is_cuda
            check(self._lib.blz_unet_set_params(self._h, _ptr(params), 1))
        else:
            a = np.ascontiguousarray(params, np.float32)
            assert a.size == self.n_params, (a.size, self.n_params)
            check(self._lib.blz_unet_set_params(self._h, a.ctypes.data_as(C.c_void_p), 0))

    def get_params(self):
        a = np.empty(self.n_params, np.float32)
        check(self._lib.blz_unet_get_params(self._h, a.ctypes.data_as(C.c_void_p), 0))
        return a

    def get_grads(self):
        a = np.empty(self.n_params, np.float32)
        check(self._lib.blz_unet_get_grads(self._h, a.ctypes.data_as(C.c_void_p), 0))
        return a

    def set_kappa(self, kappa):
        self.kappa = float(kappa)
        check(self._lib.blz_unet_set_kappa(self._h, C.c_float(self.kappa)))

    def kernel_launches(self):
        return int(self._lib.blz_unet_kernel_launches(self._h))

    def last_alpha(self):
        """Step alpha of the last warm start (p + alpha d)."""
        return float(self._lib.blz_unet_last_alpha(self._h))

    def set_step(self, mode):
        """_abi.BLZ_WARM_STEP_RESIDUAL or BLZ_WARM_STEP_ENERGY (blz_unet_set_step)."""
        check(self._lib.blz_unet_set_step(self._h, int(mode)))
        return self

    def set_smoothing(self, sweeps):
        """Sweeps of p and d before the warm start's step is chosen."""
        check(self._lib.blz_unet_set_smoothing(self._h, int(sweeps)))

    def tensor(self, name):
        """FP32 host copy of an internal tensor, padded (D+2, H+2, W+2, C)."""
        i = TENSOR_NAMES.index(name)
        shape = (C.c_int * 4)()
        check(self._lib.blz_unet_tensor_shape(self._h, i, shape))
        out = np.empty(tuple(shape), np.float32)
        check(self._lib.blz_unet_get_tensor(self._h, i, out.ctypes.data_as(C.POINTER(C.c_float)), out.size))
        return out

    # -- weight files ---------------------------------------------------------------
    def save(self, path, **meta):
        m = dict(self.meta)
        m.update(meta)
        np.savez(path, params=self.get_params(), kappa=np.float32(self.kappa),
                 dims=np.array(self.dims, np.int32), meta=np.array(json.dumps(m)))

    def load(self, path):
        with np.load(path, allow_pickle=False) as z:
            self.set_params(z["params"])
            self.set_kappa(float(z["kappa"]))
            self.meta = json.loads(str(z["meta"])) if "meta" in z else {}
        return self

    # -- compute (device arrays: torch CUDA float32 tensors, reference layout) --------
    def forward(self, params_blz, rhs, p, origin=(0, 0, 0), out=None, stream=None):
        """Raw network output delta over the crop at `origin` (torch tensor,
        shape (D, H, W) of the crop)."""
        import torch
        W, H, D = self.dims
        if out is None:
            out = torch.empty((D, H, W), dtype=torch.float32, device=rhs.device)
        org = (C.c_int * 3)(*origin)
        check(self._lib.blz_unet_forward(self._h, C.byref(params_blz), org, _ptr(rhs), _ptr(p), _ptr(out),
                                         _stream_handle(stream)))
        return out

    def loss_grad(self, params_blz, rhs, p, p_target, origin=(0, 0, 0), stream=None):
        """Loss of one sample and the parameter gradients (kept on the device).
        Returns (loss, mean target^2)."""
        org = (C.c_int * 3)(*origin)
        loss = (C.c_double * 2)()
        check(self._lib.blz_unet_loss_grad(self._h, C.byref(params_blz), org, _ptr(rhs), _ptr(p),
                                           _ptr(p_target), loss, _stream_handle(stream)))
        return float(loss[0]), float(loss[1])

    def adam(self, lr, beta1=0.9, beta2=0.999, eps=1e-8, stream=None):
        check(self._lib.blz_unet_adam(self._h, C.c_float(lr), C.c_float(beta1), C.c_float(beta2),
                                      C.c_float(eps), _stream_handle(stream)))


def weights_path(name):
    return os.path.join(WEIGHTS_DIR, name)


def _main(argv=None):
    """Times the network's forward pass on a random n^3 grid, or one training
    step (forward, loss and every gradient) with --train-step:
    python -m blaze_b200.unet --forward 256 --reps 5
    python -m blaze_b200.unet --forward 128 --train-step --reps 5"""
    import argparse
    import time
    import torch
    from .scenes import SceneSettings
    ap = argparse.ArgumentParser()
    ap.add_argument("--forward", type=int, default=128, help="grid edge (multiple of 8)")
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--train-step", action="store_true", help="time blz_unet_loss_grad instead")
    args = ap.parse_args(argv)
    n = args.forward
    g = SceneSettings(gridRes=(n, n, n), dx=1.0 / n, closedBounds=(1, 1, 1, 0, 1, 1), bc_mode=1).to_params()
    gen = torch.Generator(device="cuda").manual_seed(0)
    rhs = torch.randn((n, n, n), device="cuda", generator=gen)
    p = 0.1 * torch.randn((n, n, n), device="cuda", generator=gen)
    net = WarmStartUNet((n, n, n), init_params(0))
    out = torch.empty((n, n, n), device="cuda")
    pt = p + 0.05 * torch.randn((n, n, n), device="cuda", generator=gen)
    run = (lambda: net.loss_grad(g, rhs, p, pt)) if args.train_step else (lambda: net.forward(g, rhs, p, out=out))
    run()
    torch.cuda.synchronize()
    launches0 = net.kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.reps):
        run()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.reps
    key = "train_step_ms" if args.train_step else "forward_ms"
    print(json.dumps({"grid": n, key: ms, "launches_per_call": (net.kernel_launches() - launches0) // args.reps}))
    net.close()


if __name__ == "__main__":
    _main()
