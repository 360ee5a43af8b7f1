"""Helpers shared by the GPU tests."""
import numpy as np


def frac_close(a, b, rtol=1e-4, floor=1e-3):
    """Fraction of values with |a-b| <= rtol * max(|b|, floor)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float((np.abs(a - b) <= rtol * np.maximum(np.abs(b), floor)).mean())


def read_device_floats(ptr: int, shape) -> np.ndarray:
    """Copies float32 device memory at `ptr` (e.g. DataObject.device_ptr())
    into a host array with cudaMemcpy, as the reference's harnesses read its
    layers."""
    import ctypes
    out = np.zeros(shape, np.float32)
    cudart = ctypes.CDLL("libcudart.so.12")
    rc = cudart.cudaMemcpy(ctypes.c_void_p(out.ctypes.data), ctypes.c_void_p(ptr),
                           ctypes.c_size_t(out.nbytes), 2)  # cudaMemcpyDeviceToHost
    assert rc == 0, f"cudaMemcpy failed ({rc})"
    return out
