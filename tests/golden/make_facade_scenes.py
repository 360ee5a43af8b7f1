"""Regenerates tests/golden/facade_scenes.json: scenes built through the
reference's own Python facade (nectar_render/python, imported from the
reference project over this back end's `_pathtracer` module) and read back
as scene specs. Run where the reference project exists:

    NECTAR_REFERENCE=<reference project root> python tests/golden/make_facade_scenes.py

(default root: /root/reference). Scenes:
  config_py   the reference's own config.py scene and camera (five quads,
              two rotated cubes, a ceiling object light, a thin-lens camera
              with aperture 0.01), with its MAX_DEPTH and SEED
  cornell512  the small configuration (512x512, 64 samples, depth 8, seed 0)
              built with the facade's Hittable/Material/Camera/Scene
"""
from __future__ import annotations

import json
import os
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from nectarrender_b200 import scenes  # noqa: E402


def reference_root() -> Path:
    return Path(os.environ.get("NECTAR_REFERENCE", "/root/reference"))


def import_facade(root: Path):
    """Imports nectar_render.python with `_pathtracer` bound to this back end."""
    import nectarrender_b200 as nb
    sys.modules["_pathtracer"] = nb.pathtracer()
    if str(root) not in sys.path:
        sys.path.insert(0, str(root))
    import nectar_render.python as facade
    return facade


def cornell_through_facade(nr):
    """The small configuration with the facade's factories (SURVEY config 1:
    grey 0.73 / red / green quads, spheres r=0.3, ceiling light radiance 15,
    fov 40 degrees, 512x512, 64 samples, depth 8, seed 0)."""
    C, V3, H, M = nr.Color, nr.Vector3, nr.Hittable, nr.Material
    grey, red, green = C(0.73, 0.73, 0.73), C(0.65, 0.05, 0.05), C(0.12, 0.45, 0.15)
    hittables = [
        H.QUAD(V3(0.0, -0.5, 0.0), V3(0.0, 0.0, 0.0), V3(1.0), M.LAMBERTIAN(grey)),
        H.QUAD(V3(0.0, 0.5, 0.0), V3(0.0, 180.0, 0.0), V3(1.0), M.LAMBERTIAN(grey)),
        H.QUAD(V3(0.5, 0.0, 0.0), V3(0.0, 0.0, 90.0), V3(1.0), M.LAMBERTIAN(red)),
        H.QUAD(V3(-0.5, 0.0, 0.0), V3(0.0, 0.0, -90.0), V3(1.0), M.LAMBERTIAN(green)),
        H.QUAD(V3(0.0, 0.0, -0.5), V3(-90.0, 0.0, 0.0), V3(1.0), M.LAMBERTIAN(grey)),
        H.SPHERE(V3(-0.22, -0.2, -0.15), 0.3, M.LAMBERTIAN(C(0.8, 0.8, 0.8))),
        H.SPHERE(V3(0.22, -0.2, -0.2), 0.3, M.PBR(albedo=C(0.9, 0.9, 0.9), roughness=0.1,
                                                  metallic=1.0)),
        H.SPHERE(V3(0.02, -0.25, 0.22), 0.3, M.DIELECTRIC(ior=1.5)),
    ]
    lights = [H.OBJECT_LIGHT(H.QUAD(V3(0.0, 0.499, 0.0), V3(0.0, 180.0, 0.0), V3(0.2)), 15.0,
                             C.white())]
    sky = nr.Skylight()
    scene = nr.Scene(hittables, lights, sky)
    cam = nr.Camera(resolution=(512, 512), position=(0.0, 0.0, 2.0), rotation=(0.0, 0.0, 0.0),
                    num_samples=65, focal_length=1.0, focus_distance=1.0, aperture=0.0,
                    sensor_width=scenes.FOV40_SENSOR, shutter_speed=1.0)
    return scene, cam


def facade_specs(root: Path) -> dict[str, scenes.SceneSpec]:
    nr = import_facade(root)
    out = {}
    scene, cam = cornell_through_facade(nr)
    out["cornell512"] = scenes.from_pathtracer(scene, cam, 8, 0, name="cornell512 (facade)")
    sys.path.insert(0, str(root))
    import config  # the reference's config.py: builds CAMERA and SCENE at import
    out["config_py"] = scenes.from_pathtracer(config.SCENE, config.CAMERA, config.MAX_DEPTH,
                                              config.SEED, name="config.py (facade)")
    return out


def main():
    specs = facade_specs(reference_root())
    data = {k: scenes.spec_to_json(v) for k, v in specs.items()}
    text = "{\n" + ",\n".join(f"{json.dumps(k)}: {json.dumps(v)}" for k, v in data.items()) + "\n}\n"
    (HERE / "facade_scenes.json").write_text(text)
    print("wrote", HERE / "facade_scenes.json")


if __name__ == "__main__":
    main()
