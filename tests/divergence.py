"""Classification of per-sample differences between this back end and the
reference's CUDA build, from the per-bounce records of both
(nr_render_trace_log, and the reference's own trace_ray driven by
oracle.RefCUDA.trace_log): 16 floats per pixel and bounce — ray origin and
direction, hit object id and triangle as uint32 bits, world t, throughput and
beauty after the bounce, and whether the path goes on.

For every pixel whose sample misses the per-sample bar (1e-4 relative, floor
1e-3, on any beauty channel) the two records are walked from bounce 0 to the
FIRST bounce where anything differs. What differs there puts the pixel in
one class:

* ``rounding`` — the ray entering that bounce differs by at most `ray_tol`
  (relative to the largest coordinate), or the throughput and beauty of a
  non-PBR bounce by at most `value_tol` relative: fast-math device arithmetic
  rounded differently (another operation order, multiply and add fused at
  other places), amplified by the local conditioning of the step that made
  it (refraction near total internal reflection, cosine samples near the
  horizon). Everything after follows from it: the difference grows over the
  next bounces until a sky lookup or a discrete choice (which object a ray
  grazes, Russian roulette, reflect or refract) differs.
* ``ggx``      — same rays and hits, and the throughput of a PBR bounce
  differs by at most `ggx_tol` relative: the GGX distribution at low
  roughness magnifies a rounding difference in n.h by about 4 / alpha^2
  (alpha = roughness^2; 1e5 at roughness 0.08).
* ``tie``      — bit-identical rays hit different objects at the same world t
  (within 1e-6 relative): the closest-hit rule decides an exact tie (the
  reference keeps the first object visited at equal t across objects,
  graph.h:38, and the last triangle at equal t in a mesh, mesh.h:361).
* ``eps``      — bit-identical rays disagree about an object whose surface
  lies within 1.5 EPS of the ray origin: a root of the intersection within a
  few ulps of the interval bound EPS (hittable.h:326) is accepted on one side
  and rejected on the other. This is how a ray leaving a dielectric sphere by
  refraction meets the sphere again, since its origin is biased EPS outward
  along the front-face normal (hit_record.h:46).
* ``hit``      — bit-identical rays hit different objects at different t,
  away from the EPS bound: a traversal or intersection disagreement (a bug).
* ``shade``    — same rays and hits, but the bounce's throughput, beauty or
  stop decision differs beyond the tolerances above (a bug).
* ``drift``    — the first difference is a ray that differs beyond `ray_tol`.
"""
from __future__ import annotations

import numpy as np

NONE = np.uint32(0xFFFFFFFF)
EPS = 1e-4


def failing_pixels(ours_beauty, ref_beauty, rtol=1e-4, floor=1e-3):
    """(y, x) of the pixels with any beauty channel outside the bar."""
    a = np.asarray(ours_beauty, np.float64)
    b = np.asarray(ref_beauty, np.float64)
    bad = np.abs(a - b) > rtol * np.maximum(np.abs(b), floor)
    bad |= np.isnan(a) != np.isnan(b)
    return np.argwhere(bad.any(axis=0))


def _surface_distance(spec, obj_id, origin):
    """|distance from origin to the surface| of a sphere object of `spec`
    (world space, unrotated spheres scaled by radius), else None."""
    if spec is None or obj_id == NONE or obj_id >= len(spec.objects):
        return None
    o = spec.objects[int(obj_id)]
    base = o["wrapped_type"] or o["type"]
    if base != 2:  # spheres
        return None
    c = np.asarray(o["position"], np.float64)
    r = float(o["radius"]) * float(o["scale"][0])
    return abs(float(np.linalg.norm(np.asarray(origin, np.float64) - c)) - r)


def _is_pbr(spec, obj_id):
    if spec is None or obj_id == NONE or obj_id >= len(spec.objects):
        return False
    return spec.objects[int(obj_id)]["material"]["type"] == 2


def _rel(a, b, scale=None):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.maximum(np.abs(b), 1e-30) if scale is None else max(scale, 1e-30)
    d = np.abs(a - b) / den
    return float(np.max(np.where(np.isnan(d), np.inf, d)))


def classify_pixel(lo, lr, spec=None, ray_tol=2e-4, value_tol=1e-4, ggx_tol=2e-2):
    """(class, bounce, magnitude) for one pixel's records `lo` (ours) and
    `lr` (reference), each (bounces, 16) float32; magnitude is the relative
    size of the first difference."""
    uo, ur = lo.view(np.uint32), lr.view(np.uint32)
    nb = lo.shape[0]
    for b in range(nb):
        reached_o = not np.all(uo[b] == NONE)
        reached_r = not np.all(ur[b] == NONE)
        if reached_o != reached_r or not reached_o:
            # the records end together unless a stop decision differed at
            # b - 1, which the checks below catch first
            return "rounding", b, 0.0
        if not np.array_equal(uo[b, :6], ur[b, :6]):
            m = max(_rel(lo[b, :3], lr[b, :3], float(np.max(np.abs(lr[b, :3])))),
                    _rel(lo[b, 3:6], lr[b, 3:6], float(np.max(np.abs(lr[b, 3:6])))))
            return ("rounding" if m <= ray_tol else "drift"), b, m
        obj_o, obj_r = uo[b, 6], ur[b, 6]
        if obj_o != obj_r:
            to, tr = float(lo[b, 8]), float(lr[b, 8])
            if obj_o != NONE and obj_r != NONE and abs(to - tr) <= 1e-6 * max(abs(tr), 1e-6):
                return "tie", b, 0.0
            for obj in (obj_o, obj_r):
                dist = _surface_distance(spec, obj, lo[b, :3])
                if dist is not None and dist <= 1.5 * EPS:
                    return "eps", b, 0.0
            return "hit", b, abs(to - tr)
        if not np.array_equal(uo[b, 9:16], ur[b, 9:16]):
            m = _rel(lo[b, 9:15], lr[b, 9:15])
            if uo[b, 15] != ur[b, 15] and m == 0.0:
                return "shade", b, m
            if _is_pbr(spec, obj_o):
                return ("ggx" if m <= ggx_tol else "shade"), b, m
            return ("rounding" if m <= value_tol else "shade"), b, m
        if uo[b, 15] == 0:
            return "rounding", b, 0.0
    return "rounding", nb - 1, 0.0


def classify(ours_log, ref_log, ours_beauty, ref_beauty, spec=None, **tol):
    """Counts per class over the failing pixels, plus per-pixel details:
    {"failing": n, "pixels": total, "classes": {cls: n}, "by_bounce":
    {cls: [n per bounce]}, "examples": {cls: [(y, x, bounce), ...]}}."""
    fails = failing_pixels(ours_beauty, ref_beauty)
    return classify_records(ours_log[fails[:, 0], fails[:, 1]],
                            ref_log[fails[:, 0], fails[:, 1]], fails,
                            int(ours_beauty.shape[1] * ours_beauty.shape[2]), spec, **tol)


def classify_records(lo, lr, where, pixels, spec=None, **tol):
    """classify() over the records of the failing pixels only: lo, lr are
    (n, bounces, 16), `where` their (y, x)."""
    nb = lo.shape[1]
    out = {"pixels": int(pixels), "failing": int(len(lo)), "classes": {}, "by_bounce": {},
           "examples": {}, "largest_first_difference": {}}
    for k in range(len(lo)):
        cls, b, m = classify_pixel(lo[k], lr[k], spec, **tol)
        big = out["largest_first_difference"]
        big[cls] = max(big.get(cls, 0.0), m)
        out["classes"][cls] = out["classes"].get(cls, 0) + 1
        out["by_bounce"].setdefault(cls, [0] * nb)[max(b, 0)] += 1
        ex = out["examples"].setdefault(cls, [])
        if len(ex) < 8:
            ex.append((int(where[k][0]), int(where[k][1]), int(b)))
    return out
