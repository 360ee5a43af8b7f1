"""Launch-shape tuner for the wavefront integrator.

Picks, by timing on the scene that will be rendered, the knobs that change
speed but never the image:

  * ``mesh_leaf`` / ``tlas_leaf`` - primitives per 8-wide BVH leaf (1..3) of
    the mesh trees and of the top-level tree;
  * ``mesh_width`` / ``tlas_width`` - children per wide BVH node (4 or 8)
    of the same trees;
  * ``extend_variant`` - traversal kernel and the CTAs per SM its register
    budget targets: 4, 5, 6, 8 (nested two-level traversal; 128, 96, 80 or
    64 registers per thread) and 14, 15, 16, 18 (flattened traversal with lane
    refill, same budgets), 64 / 74 / 84 (14 with a per-iteration warp vote
    between primitive tests and node work); 100 * a + b runs a for the
    camera rays of bounce 0 and b for the later bounces;
  * ``samples_per_wave`` - sample indices in flight per wave, i.e. the length
    of the path queues (paths = W*H*samples_per_wave);
  * ``shade_variant`` - register budget of the shading kernel (5 or 6 CTAs
    per SM, or 128 registers);
  * ``sort_materials`` - shade each bounce's queue grouped by material type
    (1) or in queue order (-1);
  * ``schedule`` - wavefront or the per-pixel megakernel.

Every candidate renders the same samples (the parity tests cover each knob;
knobs that reshape a tree can only change which primitive wins an exact tie),
so the record only trades time. A record is keyed by the scene's signature
and can be saved and reused with :func:`load` / :func:`save`.
"""
from __future__ import annotations

import itertools
import json
from dataclasses import asdict, dataclass, field
from pathlib import Path

from . import capi
from .scenes import SceneSpec

VARIANTS = (5, 14, 514, 564, 574, 584, 414, 474)


@dataclass
class Tuning:
    mesh_leaf: int = 1
    tlas_leaf: int = 1
    mesh_width: int = 8
    tlas_width: int = 8
    extend_variant: int = 574
    samples_per_wave: int = 0
    shade_variant: int = 6
    sort_materials: int = 1
    schedule: int = capi.SCHEDULE_WAVEFRONT
    ms_per_sample: float = 0.0
    table: list = field(default_factory=list)

    def render_overrides(self) -> dict:
        return {"extend_variant": self.extend_variant, "samples_per_wave": self.samples_per_wave,
                "shade_variant": self.shade_variant, "sort_materials": self.sort_materials,
                "schedule": self.schedule}

    def scene_overrides(self) -> dict:
        return {"mesh_leaf": self.mesh_leaf, "tlas_leaf": self.tlas_leaf,
                "mesh_width": self.mesh_width, "tlas_width": self.tlas_width}


def signature(spec: SceneSpec) -> str:
    """Identifies the workload a record was tuned on."""
    cam = spec.camera
    return json.dumps({"res": [int(cam["resolution"][0]), int(cam["resolution"][1])],
                       "depth": spec.ray_depth, "objects": len(spec.objects), "name": spec.name,
                       "meshes": [Path(m).name for m in spec.meshes]}, sort_keys=True)


def _time(scene: capi.Scene, spec: SceneSpec, over: dict, samples: int, reps: int) -> float:
    r = capi.Render(scene, spec, **over)
    r.samples(1, samples)  # warm-up: allocates the queues, loads the kernels
    best = float("inf")
    for _ in range(reps):
        r.samples(1, samples)
        best = min(best, r.last_ms())
    return best / samples


def tune(spec: SceneSpec, samples: int = 4, reps: int = 2, leaves=((1, 1), (2, 1), (3, 1), (1, 2)),
         variants=VARIANTS, waves=(0, 2, 4, 8), shades=(5, 6), sorts=(1, -1),
         megakernel: bool = True, widths=((8, 8), (4, 8))) -> Tuning:
    """Times every candidate on `spec` (device time of `samples` sample
    indices, best of `reps`) and returns the fastest as a :class:`Tuning`."""
    table = []
    best = None
    for (mesh_leaf, tlas_leaf), (mesh_width, tlas_width) in itertools.product(leaves, widths):
        scene = capi.Scene(spec, mesh_leaf=mesh_leaf, tlas_leaf=tlas_leaf, mesh_width=mesh_width,
                           tlas_width=tlas_width)
        cands = [dict(extend_variant=v, samples_per_wave=w, shade_variant=sv, sort_materials=so,
                      schedule=capi.SCHEDULE_WAVEFRONT)
                 for v, w, sv, so in itertools.product(variants, waves, shades, sorts)]
        if megakernel:
            cands.append(dict(extend_variant=0, samples_per_wave=0, shade_variant=0,
                              sort_materials=-1, schedule=capi.SCHEDULE_MEGAKERNEL))
        for over in cands:
            ms = _time(scene, spec, over, samples, reps)
            row = dict(mesh_leaf=mesh_leaf, tlas_leaf=tlas_leaf, mesh_width=mesh_width,
                       tlas_width=tlas_width, ms_per_sample=ms, **over)
            table.append(row)
            if best is None or ms < best["ms_per_sample"]:
                best = row
        del scene
    t = Tuning(**{k: best[k] for k in ("mesh_leaf", "tlas_leaf", "mesh_width", "tlas_width",
                                       "extend_variant",
                                       "samples_per_wave", "shade_variant", "sort_materials",
                                       "schedule", "ms_per_sample")})
    t.table = table
    return t


def save(path: str | Path, spec: SceneSpec, t: Tuning) -> None:
    p = Path(path)
    records = json.loads(p.read_text()) if p.exists() else {}
    records[signature(spec)] = asdict(t)
    p.write_text(json.dumps(records, indent=1))


def load(path: str | Path, spec: SceneSpec) -> Tuning | None:
    p = Path(path)
    if not p.exists():
        return None
    rec = json.loads(p.read_text()).get(signature(spec))
    return Tuning(**rec) if rec else None
