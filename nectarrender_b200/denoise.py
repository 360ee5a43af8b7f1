"""The learned denoiser through the C ABI (nr_denoiser_*): a five-level U-Net
on the beauty, diffuse, world-normal and depth layers, trained and run on the
GPU.

It stands where the reference's OIDN stage stands (TransferStream applies
OIDN's "RT" filter to beauty with diffuse and world normal as guides,
nectar_render/csrc/data/include/data/stream.h:160-170, denoise.h:21-104).
Images are CUDA float32 tensors [B, 3, H, W] (depth [B, 1, H, W]; H, W
multiples of 16).
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import capi, library

LOSS_SQUARED, LOSS_ABSOLUTE = 0, 1
# layer_mask of renders whose layers feed the denoiser: beauty, diffuse,
# world normal and depth
DENOISE_LAYERS = (1 << 0) | (1 << 1) | (1 << 4) | (1 << 6)


def _f(t):
    return C.cast(t.data_ptr(), C.POINTER(C.c_float)) if t is not None else None


class Denoiser:
    def __init__(self, max_pixels: int, seed: int = 0):
        self.lib = library()
        self.h = C.c_void_p()
        self.max_pixels = max_pixels
        capi._check(self.lib.nr_denoiser_create(C.c_uint32(max_pixels), C.c_uint32(seed),
                                                C.byref(self.h)), "nr_denoiser_create")

    def __del__(self):
        if getattr(self, "h", None) and self.h.value:
            self.lib.nr_denoiser_destroy(self.h)
            self.h = None  # module globals may already be gone at exit

    @staticmethod
    def _stream():
        import torch
        return C.c_uint64(torch.cuda.current_stream().cuda_stream)

    def set_loss(self, kind: int) -> None:
        """LOSS_ABSOLUTE (the default) or LOSS_SQUARED, in log space."""
        capi._check(self.lib.nr_denoiser_set_loss(self.h, kind), "nr_denoiser_set_loss")

    def train_step(self, beauty, diffuse, normal, target, lr: float, depth=None) -> float:
        """One step (lr <= 0: gradients only); returns the loss before it."""
        B, _, H, W = beauty.shape
        loss = C.c_double()
        capi._check(self.lib.nr_denoiser_train_step(self.h, _f(beauty), _f(diffuse), _f(normal),
                                                    _f(depth), _f(target), B, H, W,
                                                    C.c_float(lr), C.byref(loss), self._stream()),
                    "nr_denoiser_train_step")
        return loss.value

    def infer(self, beauty, diffuse, normal, out=None, depth=None):
        import torch
        if out is None:
            out = torch.empty_like(beauty)
        B, _, H, W = beauty.shape
        capi._check(self.lib.nr_denoiser_infer(self.h, _f(beauty), _f(diffuse), _f(normal),
                                               _f(depth), _f(out), B, H, W, self._stream()),
                    "nr_denoiser_infer")
        return out

    def infer_device(self, beauty: int, diffuse: int, normal: int, out: int, B: int, H: int,
                     W: int, depth: int = 0) -> None:
        """infer() on raw device addresses (e.g. a render's layer pointers)."""
        cf = lambda a: C.cast(C.c_void_p(a), C.POINTER(C.c_float)) if a else None
        capi._check(self.lib.nr_denoiser_infer(self.h, cf(beauty), cf(diffuse), cf(normal),
                                               cf(depth), cf(out), B, H, W, self._stream()),
                    "nr_denoiser_infer")

    def layers(self) -> list[tuple[int, int]]:
        n = C.c_int32()
        self.lib.nr_denoiser_layers(self.h, C.byref(n), None)
        arr = (C.c_int32 * (2 * n.value))()
        self.lib.nr_denoiser_layers(self.h, C.byref(n), arr)
        return [(arr[2 * i], arr[2 * i + 1]) for i in range(n.value)]

    def _get(self, what: int) -> list[tuple[np.ndarray, np.ndarray]]:
        n = C.c_uint64()
        self.lib.nr_denoiser_param_count(self.h, C.byref(n))
        flat = np.zeros(n.value, np.float32)
        capi._check(self.lib.nr_denoiser_get_params(self.h, what,
                                                    flat.ctypes.data_as(C.POINTER(C.c_float))),
                    "nr_denoiser_get_params")
        out, o = [], 0
        for cin, cout in self.layers():
            k = 9 * cin * cout
            out.append((flat[o:o + k].reshape(9, cout, cin), flat[o + k:o + k + cout]))
            o += k + cout
        return out

    def params(self):
        return self._get(0)

    def grads(self):
        return self._get(1)

    def set_params(self, params) -> None:
        flat = np.concatenate([np.concatenate([w.ravel(), b.ravel()]) for w, b in params])
        flat = np.ascontiguousarray(flat, np.float32)
        capi._check(self.lib.nr_denoiser_set_params(self.h, flat.ctypes.data_as(C.POINTER(C.c_float))),
                    "nr_denoiser_set_params")


def render_layers(render: capi.Render):
    """(beauty, diffuse, normal, depth) of a render's accumulated layers as
    CUDA tensors [1, C, H, W] (copies of the device layers); depth is None
    unless the render keeps the depth layer (layer_mask DENOISE_LAYERS)."""
    import torch
    out = []
    for layer in (0, 1, 4):
        out.append(torch.from_numpy(render.layer(layer)).cuda()[None])
    try:
        z = render.layer_channels(6)
        out.append(torch.from_numpy(z).cuda()[None])
    except RuntimeError:
        out.append(None)
    return tuple(out)


def train(den: Denoiser, pairs, steps: int = 0, seconds: float = 0.0, lr: float = 2e-3,
          crop: int = 128, batch: int = 8, seed: int = 0, log=None):
    """Trains on `pairs` = [((beauty, diffuse, normal, depth), target)] of CUDA
    tensors [1, C, H, W] (depth may be None) with random crops; stops after `steps` steps or `seconds`
    of wall time. Returns (steps, seconds, last loss)."""
    import torch
    rng = np.random.default_rng(seed)
    t0 = time.perf_counter()
    k, loss = 0, float("nan")
    while (steps and k < steps) or (seconds and time.perf_counter() - t0 < seconds):
        bs, ds, ns, zs, ts = [], [], [], [], []
        for _ in range(batch):
            (b, d, n, z), t = pairs[rng.integers(len(pairs))]
            H, W = b.shape[2], b.shape[3]
            y, x = int(rng.integers(0, H - crop + 1)), int(rng.integers(0, W - crop + 1))
            sl = (slice(None), slice(None), slice(y, y + crop), slice(x, x + crop))
            bs.append(b[sl]); ds.append(d[sl]); ns.append(n[sl]); ts.append(t[sl])
            zs.append(z[sl] if z is not None else None)
        cat = lambda xs: torch.cat(xs).contiguous()
        depth = cat(zs) if all(z is not None for z in zs) else None
        loss = den.train_step(cat(bs), cat(ds), cat(ns), cat(ts), lr, depth=depth)
        k += 1
        if log and k % 50 == 0:
            log(k, loss)
    torch.cuda.synchronize()
    return k, time.perf_counter() - t0, loss
