"""Helpers shared by the GPU tests."""
import numpy as np


def frac_close(a, b, rtol=1e-4, floor=1e-3):
    """Fraction of values with |a-b| <= rtol * max(|b|, floor)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float((np.abs(a - b) <= rtol * np.maximum(np.abs(b), floor)).mean())
