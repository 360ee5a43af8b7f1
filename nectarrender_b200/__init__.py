"""nectarrender_b200 — B200-native (sm_100a) back end for NectarRender's
path-tracing hot path.

Two native libraries live in this directory (built by ``build.py``):

* ``libnectar_b200.so`` — the CUDA kernels and the C ABI declared in
  ``include/nectar_b200.h``;
* ``_pathtracer*.so`` — a pybind11 module with the reference's Python API
  (``_pathtracer.scene.Scene``, ``_pathtracer.engine.RenderEngine``, ...)
  implemented on that C ABI.

There is no CPU fallback: without the built libraries, or without a CUDA
device, rendering raises.
"""
from __future__ import annotations

import ctypes
import importlib
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libnectar_b200.so"

_lib: ctypes.CDLL | None = None


def library() -> ctypes.CDLL:
    """The C-ABI library (ctypes handle); raises if it was not built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: run `python -m nectarrender_b200.build` "
                "(or __graft_entry__.build()) first")
        _lib = ctypes.CDLL(str(LIB_PATH))
        _lib.nr_last_error.restype = ctypes.c_char_p
    return _lib


def pathtracer():
    """The `_pathtracer` module (the reference's Python API on this back end)."""
    library()
    return importlib.import_module("nectarrender_b200._pathtracer")


def last_error() -> str:
    return library().nr_last_error().decode()


def device_count() -> int:
    return int(library().nr_device_count())
