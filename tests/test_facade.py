"""The reference's own Python facade (nectar_render/python) imported over
this back end's `_pathtracer` module: every facade module imports, the
factories build the small configuration and the reference's config.py scene,
and the scene specs read back from those objects equal the committed
fixture that the GPU twin renders (tests/test_gpu_facade.py). The facade is
read from the reference project where it lies; without it these tests skip."""
import json
import sys
from pathlib import Path

import numpy as np
import pytest

import nectarrender_b200 as nb
from nectarrender_b200 import scenes

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
import make_facade_scenes as mfs  # noqa: E402

GOLDEN = Path(__file__).resolve().parent / "golden" / "facade_scenes.json"


@pytest.fixture(scope="module")
def facade():
    root = mfs.reference_root()
    if not (root / "nectar_render" / "python" / "__init__.py").exists():
        pytest.skip("reference project not present")
    return mfs.import_facade(root)


def test_every_facade_module_imports(facade):
    import importlib
    for m in ["core", "cuda", "data", "hittable", "host", "material", "progress", "engine",
              "engine.camera", "engine.engine", "engine.lights", "engine.scene"]:
        importlib.import_module("nectar_render.python." + m)
    # names the facade re-exports at package level
    for name in ["Scene", "SceneInterface", "SceneNode", "SceneOutline", "Camera", "CameraParams",
                 "Skylight", "RenderEngine", "EngineType", "CUDAMemInfo", "CUDAProfiler",
                 "Hittable", "Volumetric", "HitRecord", "Material", "Texture", "Vector3", "Color"]:
        assert getattr(facade, name) is not None, name
    assert facade.SceneNode is nb.pathtracer().scene.SceneNode


def test_facade_scenes_match_the_fixture(facade):
    specs = mfs.facade_specs(mfs.reference_root())
    golden = json.loads(GOLDEN.read_text())
    assert set(specs) == set(golden)
    for k, spec in specs.items():
        assert scenes.spec_to_json(spec) == golden[k], k


def _f32(x):
    if isinstance(x, (list, tuple)):
        return [_f32(v) for v in x]
    if isinstance(x, float):
        return float(np.float32(x))
    if isinstance(x, dict):
        return {k: _f32(v) for k, v in x.items()}
    return x


def test_facade_cornell_is_the_small_configuration(facade):
    scene, cam = mfs.cornell_through_facade(facade)
    got = scenes.spec_to_json(scenes.from_pathtracer(scene, cam, 8, 0))
    want = scenes.spec_to_json(scenes.cornell(res=512, spp=64, depth=8, seed=0))
    assert _f32(got["objects"]) == _f32(want["objects"])
    assert _f32(got["camera"]) == _f32(want["camera"])
    assert got["sky"] == want["sky"] and got["ray_depth"] == 8 and got["seed"] == 0


def test_spec_round_trip_through_pathtracer(facade):
    golden = json.loads(GOLDEN.read_text())
    pt = nb.pathtracer()
    for k, d in golden.items():
        spec = scenes.spec_from_json(d)
        scene, cam, keep = scenes.to_pathtracer(spec, pt)
        back = scenes.spec_to_json(scenes.from_pathtracer(scene, cam, spec.ray_depth, spec.seed,
                                                          name=spec.name))
        assert back == d, k


def test_config_py_scene_content(facade):
    spec = scenes.spec_from_json(json.loads(GOLDEN.read_text())["config_py"])
    types = [o["type"] for o in spec.objects]
    assert types == [scenes.QUAD] * 5 + [scenes.CUBE] * 2 + [scenes.LIGHT]
    assert spec.objects[5]["rotation"] == (0.0, 35.0, 0.0)
    assert spec.camera["aperture"] > 0           # thin-lens camera (defocus)
    assert (spec.ray_depth, spec.seed) == (5, 42)


def test_outline_and_memory_without_a_device(facade):
    pt = nb.pathtracer()
    spec = scenes.cornell(res=16, spp=2)
    scene, cam, keep = scenes.to_pathtracer(spec, pt)
    eng = facade.RenderEngine(cam, 8, 0)
    si = eng.get_scene_interface()
    outline = si.get_scene_outline()          # nothing set yet: empty outline
    assert list(outline.nodes) == []
    with pytest.raises(RuntimeError, match="Object index not valid"):
        si.get_transform()
    if nb.device_count() == 0:
        with pytest.raises(RuntimeError, match="no CUDA device"):
            facade.CUDAProfiler.get_cuda_meminfo()
        with pytest.raises(RuntimeError, match="no CUDA device"):
            eng.set_scene(scene)
