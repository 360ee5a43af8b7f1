"""The divergence classifier on planted records (no GPU): each class is
recognised from a pair of hand-made per-bounce records."""
import numpy as np

from nectarrender_b200 import scenes
from tests.divergence import NONE, classify_pixel


def _rec(n=3):
    r = np.zeros((n, 16), np.float32)
    r[:, 3:6] = (0.0, 0.0, -1.0)
    r[:, 9:12] = 0.5
    r.view(np.uint32)[:, 6] = 1
    r[:, 8] = 2.0
    r.view(np.uint32)[:, 15] = 1
    r.view(np.uint32)[-1, 15] = 0
    return r


def _spec():
    return scenes.cornell(res=8, spp=2)   # object 1: grey quad, 7: dielectric sphere r=0.3


def test_identical_records_are_rounding_of_the_last_bounce():
    a = _rec()
    assert classify_pixel(a, a.copy(), _spec())[0] == "rounding"


def test_a_small_ray_difference_is_rounding_and_a_large_one_drift():
    a, b = _rec(), _rec()
    b[1, 4] = np.nextafter(np.float32(0.0), np.float32(1.0)) * 1e3
    assert classify_pixel(a, b, _spec())[:2] == ("rounding", 1)
    b[1, 4] = 0.01
    assert classify_pixel(a, b, _spec())[0] == "drift"


def test_hits_tie_eps_and_bug():
    spec = _spec()
    a, b = _rec(), _rec()
    b.view(np.uint32)[1, 6] = 2
    assert classify_pixel(a, b, spec)[0] == "tie"            # same t, other object
    b[1, 8] = 3.0
    assert classify_pixel(a, b, spec)[0] == "hit"            # other object, other t
    sph = spec.objects[7]
    a[1, 0:3] = np.asarray(sph["position"]) + np.array([sph["radius"] + 1e-4, 0, 0])
    b[1, 0:3] = a[1, 0:3]
    b.view(np.uint32)[1, 6] = 7
    b[1, 8] = 0.5
    assert classify_pixel(a, b, spec)[0] == "eps"            # origin on the sphere's skin


def test_throughput_differences_by_material():
    spec = _spec()
    a, b = _rec(), _rec()
    b[0, 9] *= 1.0 + 5e-5
    assert classify_pixel(a, b, spec)[0] == "rounding"       # Lambertian quad
    b[0, 9] = a[0, 9] * (1.0 + 1e-3)
    assert classify_pixel(a, b, spec)[0] == "shade"
    a.view(np.uint32)[0, 6] = b.view(np.uint32)[0, 6] = 6    # the PBR sphere
    assert classify_pixel(a, b, spec)[0] == "ggx"
    b.view(np.uint32)[1:] = NONE                             # one path stops early
    a2 = a.copy()
    b2 = a.copy()
    b2.view(np.uint32)[0, 15] = 0
    assert classify_pixel(a2, b2, spec)[0] == "shade"        # stop decision on equal values
