"""Classification of per-sample differences between this back end and the
reference's CUDA build, from the per-bounce records of both
(nr_render_trace_log and the reference's trace_ray driven by
oracle.RefCUDA.trace_log: 16 floats per pixel and bounce — ray origin and
direction, hit object id and triangle as uint32 bits, world t, throughput
and beauty after the bounce, and whether the path goes on).

For every pixel whose sample misses the per-sample bar (1e-4 relative, floor
1e-3, on any beauty channel), the first bounce where the two paths part is
found: the bounce where the hit objects differ, or where one path stops and
the other goes on. The pixel is then put in one class:

* ``tie``    — the two rays at that bounce are bit-identical, they hit
  different objects at the same world t (within 1e-6 relative): the
  closest-hit rule decides an exact tie (the reference keeps the first
  object visited at equal t across objects, graph.h:38);
* ``ulp``    — the rays or throughputs entering that bounce already differ,
  by at most `ulp_rel` relative: last-bit differences of fast-math device
  arithmetic (contraction into fused multiply-adds at other places, other
  operation order) carried along the path until they flip a discrete
  decision — which object a ray grazes, Russian roulette, reflect or refract;
* ``value``  — the paths never part (same objects, same stop), the beauty
  differs only through accumulated rounding;
* ``hit``    — bit-identical rays hit different objects at different t: a
  traversal or intersection disagreement, which would be a bug;
* ``drift``  — the inputs to the parting bounce differ by more than
  `ulp_rel`: larger than rounding can explain.
"""
from __future__ import annotations

import numpy as np

NONE = np.uint32(0xFFFFFFFF)


def failing_pixels(ours_beauty, ref_beauty, rtol=1e-4, floor=1e-3):
    """(y, x) of the pixels with any beauty channel outside the bar."""
    a = np.asarray(ours_beauty, np.float64)
    b = np.asarray(ref_beauty, np.float64)
    bad = np.abs(a - b) > rtol * np.maximum(np.abs(b), floor)
    bad |= np.isnan(a) != np.isnan(b)
    return np.argwhere(bad.any(axis=0))


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.maximum(np.abs(a), np.abs(b)), 1e-30)))


def classify_pixel(lo, lr, ulp_rel=1e-4):
    """(class, bounce) for one pixel's logs `lo` (ours) and `lr` (reference),
    each (bounces, 16) float32."""
    uo, ur = lo.view(np.uint32), lr.view(np.uint32)
    nb = lo.shape[0]
    prev_atten_o = np.ones(3)
    prev_atten_r = np.ones(3)
    for b in range(nb):
        reached_o = not np.all(uo[b] == NONE)
        reached_r = not np.all(ur[b] == NONE)
        if not reached_o and not reached_r:
            return "value", b
        if reached_o != reached_r:
            # one path ended at the previous bounce: a stop decision differed
            return ("ulp" if _rel(prev_atten_o, prev_atten_r) <= ulp_rel else "drift"), b - 1
        rays_equal = bool(np.all(uo[b, :6] == ur[b, :6]))
        obj_o, obj_r = uo[b, 6], ur[b, 6]
        if obj_o != obj_r:
            if rays_equal:
                to, tr = float(lo[b, 8]), float(lr[b, 8])
                if obj_o != NONE and obj_r != NONE and abs(to - tr) <= 1e-6 * max(abs(tr), 1e-6):
                    return "tie", b
                return "hit", b
            ray_rel = _rel(lo[b, :6], lr[b, :6])
            return ("ulp" if ray_rel <= ulp_rel else "drift"), b
        go_o, go_r = uo[b, 15], ur[b, 15]
        if go_o != go_r:
            # same hit, one path stops: Russian roulette or a scatter that
            # failed on one side only, decided by the incoming values
            inputs = max(_rel(lo[b, :6], lr[b, :6]), _rel(prev_atten_o, prev_atten_r))
            return ("ulp" if inputs <= ulp_rel else "drift"), b
        prev_atten_o, prev_atten_r = lo[b, 9:12], lr[b, 9:12]
        if go_o == 0:
            return "value", b
    return "value", nb - 1


def classify(ours_log, ref_log, ours_beauty, ref_beauty, ulp_rel=1e-4):
    """Counts per class over the failing pixels, plus per-pixel details:
    {"failing": n, "pixels": total, "classes": {cls: n}, "by_bounce":
    {cls: [n per bounce]}, "examples": {cls: [(y, x, bounce), ...]}}."""
    fails = failing_pixels(ours_beauty, ref_beauty)
    nb = ours_log.shape[2]
    out = {"pixels": int(ours_beauty.shape[1] * ours_beauty.shape[2]), "failing": int(len(fails)),
           "classes": {}, "by_bounce": {}, "examples": {}}
    for y, x in fails:
        cls, b = classify_pixel(ours_log[y, x], ref_log[y, x], ulp_rel)
        out["classes"][cls] = out["classes"].get(cls, 0) + 1
        out["by_bounce"].setdefault(cls, [0] * nb)[max(b, 0)] += 1
        ex = out["examples"].setdefault(cls, [])
        if len(ex) < 8:
            ex.append((int(y), int(x), int(b)))
    return out
