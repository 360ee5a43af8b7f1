"""The neural radiance cache through the C ABI (nr_nrc_*): hash-grid
encoding + 64-wide MLP on the tcgen05 tensor cores, trained online.
Queries are CUDA float32 tensors [n, 16] (position, roughness, outgoing
direction, -, normal, -, diffuse albedo, -); radiance [n, 3]."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi, library

LEVELS, FEAT, LOG2T = 16, 2, 19
LAYERS = (64, 64, 64, 64, 16)  # output widths: four hidden layers, then the output


def _f(t):
    return C.cast(t.data_ptr(), C.POINTER(C.c_float))


class RadianceCache:
    def __init__(self, max_queries: int, lo, hi, seed: int = 0):
        self.lib = library()
        self.h = C.c_void_p()
        self.lo, self.hi = np.asarray(lo, np.float32), np.asarray(hi, np.float32)
        capi._check(self.lib.nr_nrc_create(C.c_uint32(max_queries),
                                           self.lo.ctypes.data_as(C.POINTER(C.c_float)),
                                           self.hi.ctypes.data_as(C.POINTER(C.c_float)),
                                           C.c_uint32(seed), C.byref(self.h)), "nr_nrc_create")

    def __del__(self):
        if getattr(self, "h", None) and self.h.value:
            self.lib.nr_nrc_destroy(self.h)
            self.h = None  # module globals may already be gone at exit

    @staticmethod
    def _stream():
        import torch
        return C.c_uint64(torch.cuda.current_stream().cuda_stream)

    def infer(self, queries, out=None):
        import torch
        n = queries.shape[0]
        if out is None:
            out = torch.empty((n, 3), dtype=torch.float32, device=queries.device)
        capi._check(self.lib.nr_nrc_infer(self.h, _f(queries), n, _f(out), self._stream()),
                    "nr_nrc_infer")
        return out

    def train(self, queries, target, lr: float, want_loss: bool = True):
        loss = C.c_double()
        capi._check(self.lib.nr_nrc_train(self.h, _f(queries), _f(target), queries.shape[0],
                                          C.c_float(lr), C.byref(loss) if want_loss else None,
                                          self._stream()), "nr_nrc_train")
        return loss.value if want_loss else None

    def get(self, what: int) -> np.ndarray:
        n = C.c_uint64()
        self.lib.nr_nrc_count(self.h, what, C.byref(n))
        out = np.zeros(n.value, np.float32)
        capi._check(self.lib.nr_nrc_get(self.h, what, out.ctypes.data_as(C.POINTER(C.c_float))),
                    "nr_nrc_get")
        return out

    def mlp_layers(self, flat):
        out, o = [], 0
        for nout in LAYERS:
            out.append(flat[o:o + nout * 64].reshape(nout, 64))
            o += nout * 64
        return out
