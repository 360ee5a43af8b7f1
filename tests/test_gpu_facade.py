"""GPU twin of tests/test_facade.py: the scenes that the reference's Python
facade builds over this back end (committed as tests/golden/facade_scenes.json
by tests/golden/make_facade_scenes.py) rendered through `_pathtracer`'s
RenderEngine and compared per sample with the reference's CUDA build, plus
the SceneInterface's outline, selection and transform edits and the
host.memory queries. Tolerance: per-sample radiance within 1e-4 relative
(floor 1e-3), as a fraction of values (a path that takes another branch after
a last-ulp difference differs wholesale)."""
import copy
import json
from pathlib import Path

import numpy as np
import pytest

import nectarrender_b200 as nb
import oracle
from nectarrender_b200 import capi, scenes
from tests.gpu_util import frac_close, read_device_floats

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden" / "facade_scenes.json"


def spec_of(name, spp=2):
    spec = scenes.spec_from_json(json.loads(GOLDEN.read_text())[name])
    spec.camera["samples_per_pixel"] = spp
    return spec


def engine_layers(spec):
    """Renders samples 1..spp-1 through RenderEngine; returns the running
    means of beauty, diffuse and world normal read from device_ptr()."""
    pt = nb.pathtracer()
    scene, cam, keep = scenes.to_pathtracer(spec, pt)
    eng = pt.engine.RenderEngine(cam, spec.ray_depth, spec.seed)
    eng.set_scene(scene)
    eng.render()
    H, W = (int(x) for x in spec.camera["resolution"])
    L = eng.layers()
    out = [read_device_floats(d.device_ptr(), (3, H, W)) for d in (L.beauty, L.diffuse, L.world_normal)]
    return eng, keep, out


@pytest.fixture(scope="module")
def refcuda():
    if not oracle.REF_CUDA_SO.exists():
        pytest.skip("reference CUDA build not present")
    return oracle.RefCUDA()


@pytest.mark.parametrize("name", ["cornell512", "config_py"])
def test_facade_scene_first_sample_vs_reference_cuda(name, refcuda):
    spec = spec_of(name, spp=2)          # renders sample index 1 only
    eng, keep, (b, d, n) = engine_layers(spec)
    rb, rd, rn, _ = refcuda.render(spec, 1, count=1, mode=1)
    assert np.isfinite(b).all()
    assert frac_close(b, rb) >= 0.995
    assert frac_close(d, rd) >= 0.995
    assert frac_close(n, rn) >= 0.999


def test_facade_cornell_running_mean_vs_reference_cuda(refcuda):
    spec = spec_of("cornell512", spp=5)  # samples 1..4
    eng, keep, (b, d, n) = engine_layers(spec)
    rb, rd, rn, _ = refcuda.render(spec, 1, count=4, mode=1)
    assert frac_close(b, rb) >= 0.99
    assert frac_close(n, rn) >= 0.999


def test_scene_interface_outline_selection_and_transform():
    spec = spec_of("config_py", spp=2)
    spec.camera["resolution"] = (64.0, 64.0)
    pt = nb.pathtracer()
    eng, keep, (b0, _, _) = engine_layers(spec)
    si = eng.get_scene_interface()
    nodes = list(si.get_scene_outline().nodes)
    assert [x.type_name for x in nodes] == ["Quad"] * 5 + ["Cube"] * 2 + ["ObjectLight"]
    assert [x.object_id for x in nodes] == list(range(8))
    assert [x.material_id for x in nodes] == list(range(1, 9))   # id 0: default material
    assert all(x.parent_id == 0 and x.name == x.type_name for x in nodes)
    si.select_scene_node(nodes[5])
    assert si.is_enabled() and si.get_hit_record().object_id == 5
    t = si.get_transform()
    assert (t.position().x(), t.position().y(), t.position().z()) == pytest.approx((0.2, -0.35, 0.2))
    assert si.get_material().material_type() == pt.material.MaterialType.Lambertian
    # move the cube: the next render rebuilds the scene and restarts at sample 1
    V3 = pt.core.vector.Vector3
    moved = pt.core.Transform(V3(0.1, -0.35, 0.25), V3(0.0, 35.0, 0.0), V3(0.3))
    si.set_transform(moved)
    eng.render()
    H, W = 64, 64
    b1 = read_device_floats(eng.layers().beauty.device_ptr(), (3, H, W))
    assert not np.array_equal(b0, b1)
    spec2 = copy.deepcopy(spec)
    spec2.objects[5]["position"] = (float(np.float32(0.1)), float(np.float32(-0.35)),
                                    float(np.float32(0.25)))
    r = capi.Render(capi.Scene(spec2))
    r.render_all()
    np.testing.assert_array_equal(b1, r.layer(0))


def test_host_memory_queries():
    pt = nb.pathtracer()
    info = pt.host.memory.get_cuda_meminfo()
    assert info.total > 0 and info.used + info.free == info.total
    assert pt.host.memory.get_cuda_memory_total() == info.total
