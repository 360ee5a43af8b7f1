"""Regenerates the golden fixtures in tests/golden/ from the reference's own
integrator compiled for the host (oracle/_ref/libref_cpu.so, built by
oracle/Makefile from the reference sources). Run in a container where the
reference sources exist:

    python tests/golden/make_golden.py

Fixtures:
  cornell24.npz     Cornell scene 24x24: raw layers and primary ids of
                    samples 1 and 2, running mean of samples 1..3, the n-rooks
                    pattern (4 samples, seed 0) and Philox draws
  mesh_small.npz    displaced icosphere (2 subdivisions) + 8 spheres + 32x16
                    HDRI at 20x20: raw layers of sample 1, running mean of
                    samples 1..2, parsed OBJ arrays, HDR floats, SAH cost
  icosphere_l2.obj, sky_32x16.hdr   the input files of mesh_small
  viewport24.npz    Cornell scene 24x24: viewport preview layers with and
                    without the axis grid, 8 picking rays, the selection
                    outline (radius 2) of the object under the centre
"""
from __future__ import annotations

import shutil
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

import oracle  # noqa: E402
from nectarrender_b200 import scenes  # noqa: E402


def cornell_spec():
    return scenes.cornell(res=24, spp=3)


def mesh_spec():
    spec = scenes.mesh_stress(levels=2, res_h=20, res_w=20, spp=2, depth=12, n_spheres=8,
                              hdri_size=(32, 16), scene_seed=7)
    return spec


def local_mesh_spec():
    """mesh_spec() reading the committed input files."""
    spec = mesh_spec()
    spec.meshes = [str(HERE / "icosphere_l2.obj")]
    spec.sky = dict(spec.sky, path=str(HERE / "sky_32x16.hdr"))
    return spec


def viewport_fixture(ref):
    spec = cornell_spec()
    h = ref.open_scene(spec, draw_rtl=1)
    out = {}
    for grid in (0, 1):
        b, d, n = h.viewport(bool(grid))
        out[f"beauty_grid{grid}"], out[f"diffuse_grid{grid}"], out[f"normal_grid{grid}"] = b, d, n
    uv = np.random.default_rng(1).uniform(0.02, 0.98, size=(8, 2)).astype(np.float32)
    picks = [h.pick(float(u), float(v)) for u, v in uv]
    out["pick_uv"] = uv
    out["pick_hit"] = np.array([int(p["hit"]) for p in picks], np.int32)
    out["pick_obj"] = np.array([p["object_id"] for p in picks], np.int32)
    out["pick_t"] = np.array([p["t"] for p in picks], np.float32)
    oid = h.pick(0.5, 0.5)["object_id"]
    out["mask_object"] = np.array(oid)
    out["mask_r2"] = h.selection_mask(oid, 2)
    np.savez_compressed(HERE / "viewport24.npz", **out)


def main():
    ref = oracle.RefCPU()
    viewport_fixture(ref)
    spec = cornell_spec()
    out = {}
    for s in (1, 2):
        b, d, n, p, _ = ref.render(spec, s, mode=0)
        out[f"s{s}_beauty"], out[f"s{s}_diffuse"], out[f"s{s}_normal"], out[f"s{s}_primary"] = b, d, n, p
    b, d, n, _, b64 = ref.render(spec, 1, count=3, mode=1, fp64=True)
    out.update(acc_beauty=b, acc_diffuse=d, acc_normal=n, acc_beauty64=b64)
    out["n_rooks_4_0"] = ref.n_rooks(4, 0)
    out["philox_0_5"] = ref.uniforms(0, 5, 64)
    out["philox_54321_1000"] = ref.uniforms(54321, 1000, 64)
    np.savez_compressed(HERE / "cornell24.npz", **out)

    spec = mesh_spec()
    shutil.copy(spec.meshes[0], HERE / "icosphere_l2.obj")
    shutil.copy(spec.sky["path"], HERE / "sky_32x16.hdr")
    spec = local_mesh_spec()
    out = {}
    b, d, n, p, _ = ref.render(spec, 1, mode=0)
    out.update(s1_beauty=b, s1_diffuse=d, s1_normal=n, s1_primary=p)
    b, d, n, _, b64 = ref.render(spec, 1, count=2, mode=1, fp64=True)
    out.update(acc_beauty=b, acc_diffuse=d, acc_normal=n, acc_beauty64=b64)
    P, N, T, UV, tris = ref.load_obj(spec.meshes[0])
    out.update(obj_P=P, obj_N=N, obj_T=T, obj_UV=UV, obj_tris=tris)
    out["hdr"] = ref.load_hdr(spec.sky["path"])
    sah, nodes = ref.mesh_sah(spec)
    out["sah"] = np.array([sah])
    out["sah_nodes"] = np.array([nodes])
    np.savez_compressed(HERE / "mesh_small.npz", **out)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
