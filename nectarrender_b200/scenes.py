"""Seeded synthetic scenes for the benchmark configurations.

No public dataset or asset is involved: every scene is generated from a seed.
The reference's API only loads meshes and HDRIs from files
(``Hittable.mesh(path)``, ``Skylight.hdri(path)``), so the generators write
Wavefront OBJ and Radiance ``.hdr`` files and both this back end and the
reference read those same files.

A scene is described by plain dicts (``SceneSpec``) that map one to one onto
the reference's factories; ``to_pathtracer`` turns a spec into objects of the
``_pathtracer`` API, and ``oracle`` turns it into the checker's C structs.

* ``cornell``   — the small configuration: a 5-quad box (grey 0.73, red,
  green), an emissive ceiling quad of radiance 15 passed as a light, three
  r=0.3 spheres (Lambertian 0.8, metal PBR roughness 0.1, dielectric 1.5),
  pinhole camera with a 40 degree field of view, no sky.
* ``mesh_stress`` — the BVH/mesh stress configuration: an icosphere
  subdivided ``levels`` times (8 gives 1,310,720 triangles), radially
  displaced by 4-octave value noise of amplitude 0.05, one PBR material;
  256 spheres with radii U(0.05, 0.3) and materials drawn uniformly from
  Lambertian/PBR/dielectric; a 2048x1024 equirectangular HDRI with a
  log-normal sky (mu=0, sigma=1) and a sun disk of radiance 1e4.
* ``medium_stress`` — the radiance-cache configuration: ``mesh_stress`` plus
  a 2x2x2 box of isotropic medium (sigma_t 0.5, albedo 0.9), depth 32.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

# generated assets are cached outside the source tree
ASSETS = Path(os.environ.get("NR_ASSET_DIR", "/tmp/nectarrender_b200_assets"))

# nr_hittable / nr_material enums (include/nectar_b200.h)
QUAD, SPHERE, CUBE, MESH, MEDIUM, LIGHT = 1, 2, 3, 4, 5, 6
LAMBERTIAN, PBR, DIELECTRIC, EMISSIVE, ISOTROPIC = 1, 2, 3, 4, 5
SKY_NULL, SKY_SIMPLE, SKY_HDRI = 0, 1, 2

FOV40_SENSOR = 2.0 * math.tan(math.radians(20.0))  # sensor_width / focal_length


@dataclass
class SceneSpec:
    objects: list[dict]            # hittables followed by lights
    camera: dict                   # CameraParams fields
    ray_depth: int = 8
    seed: int = 0
    sky: dict = field(default_factory=lambda: {"type": SKY_NULL})
    meshes: list[str] = field(default_factory=list)   # OBJ paths, indexed by object["mesh"]
    name: str = ""
    # uint8 planar CHW images (C >= 3) of IMAGE textures: a material's texture
    # slot is an RGB tuple (a constant colour) or {"image": index, "scale": s}
    images: list = field(default_factory=list)


def _mat(type_, **kw) -> dict:
    m = {"type": type_, "ior": 1.5, "brightness": 35.0, "tint": (1.0, 1.0, 1.0),
         "tex": [(1.0, 1.0, 1.0)] * 5}
    m.update(kw)
    return m


def lambertian(rgb) -> dict:
    return _mat(LAMBERTIAN, tex=[tuple(rgb)] + [(0.0, 0.0, 0.0)] * 4)


def pbr(albedo=(1, 1, 1), roughness=0.8, metallic=0.0, emission=(0, 0, 0), normal=(0.5, 0.5, 1.0)):
    # Material.pbr defaults (bind_material.h:118-125)
    return _mat(PBR, tex=[tuple(albedo), (roughness,) * 3, (metallic,) * 3, tuple(emission), tuple(normal)])


def dielectric(tint=(1.0, 1.0, 1.0), ior=1.5):
    return _mat(DIELECTRIC, tint=tuple(tint), ior=ior, tex=[(0.0, 0.0, 0.0)] * 5)


def emissive(rgb=(1.0, 1.0, 1.0), brightness=35.0):
    return _mat(EMISSIVE, brightness=brightness, tex=[tuple(rgb)] + [(0.0, 0.0, 0.0)] * 4)


def isotropic(rgb=(1.0, 1.0, 1.0)):
    return _mat(ISOTROPIC, tex=[tuple(rgb)] + [(0.0, 0.0, 0.0)] * 4)


def obj(type_, material, position=(0, 0, 0), rotation=(0, 0, 0), scale=(1, 1, 1), radius=1.0,
        mesh=-1, wrapped=0, density=1.0) -> dict:
    return {"type": type_, "wrapped_type": wrapped, "material": material, "mesh": mesh,
            "position": tuple(map(float, position)), "rotation": tuple(map(float, rotation)),
            "scale": tuple(map(float, scale)), "radius": float(radius), "density": float(density)}


def camera(res_h, res_w, position, rotation, spp, focal=1.0, sensor=FOV40_SENSOR, aperture=0.0,
           focus_distance=1.0, shutter_speed=1.0) -> dict:
    return {"resolution": (float(res_h), float(res_w)), "position": tuple(map(float, position)),
            "rotation": tuple(map(float, rotation)), "samples_per_pixel": int(spp),
            "focal_length": float(focal), "focus_distance": float(focus_distance),
            "aperture": float(aperture), "sensor_width": float(sensor),
            "shutter_speed": float(shutter_speed)}


# ---------------------------------------------------------------------------
# small configuration

def cornell(res: int = 512, spp: int = 64, depth: int = 8, seed: int = 0) -> SceneSpec:
    """Box of five quads (config.py:19-76 layout) with three spheres and a
    ceiling light. `spp` samples are rendered: the reference renders
    samples_per_pixel - 1 of them, so samples_per_pixel = spp + 1."""
    grey, red, green = (0.73, 0.73, 0.73), (0.65, 0.05, 0.05), (0.12, 0.45, 0.15)
    objs = [
        obj(QUAD, lambertian(grey), (0, -0.5, 0), (0, 0, 0)),      # bottom
        obj(QUAD, lambertian(grey), (0, 0.5, 0), (0, 180, 0)),     # top
        obj(QUAD, lambertian(red), (0.5, 0, 0), (0, 0, 90)),       # right
        obj(QUAD, lambertian(green), (-0.5, 0, 0), (0, 0, -90)),   # left
        obj(QUAD, lambertian(grey), (0, 0, -0.5), (-90, 0, 0)),    # back
        obj(SPHERE, lambertian((0.8, 0.8, 0.8)), (-0.22, -0.2, -0.15), radius=0.3),
        obj(SPHERE, pbr((0.9, 0.9, 0.9), roughness=0.1, metallic=1.0), (0.22, -0.2, -0.2), radius=0.3),
        obj(SPHERE, dielectric(ior=1.5), (0.02, -0.25, 0.22), radius=0.3),
        # lights come last (scene.h:36)
        obj(LIGHT, emissive((1, 1, 1), 15.0), (0, 0.499, 0), (0, 180, 0), (0.2, 0.2, 0.2), wrapped=QUAD),
    ]
    cam = camera(res, res, (0, 0, 2), (0, 0, 0), spp + 1)
    return SceneSpec(objects=objs, camera=cam, ray_depth=depth, seed=seed, name=f"cornell{res}")


def cornell_cubes(res: int = 64, spp: int = 4, depth: int = 8, seed: int = 0, aperture: float = 0.08,
                  focus_distance: float = 2.0) -> SceneSpec:
    """The Cornell box with its spheres replaced by rotated cubes (Lambertian,
    rough metal, glass) and a camera with a finite aperture (thin-lens
    defocus, camera.h): the cube's six quads under an arbitrary rotation and
    the lens sampling, which the other test scenes do not exercise."""
    spec = cornell(res=res, spp=spp, depth=depth, seed=seed)
    light = spec.objects[-1]
    spec.objects = spec.objects[:5] + [
        obj(CUBE, lambertian((0.8, 0.8, 0.8)), (-0.22, -0.3, -0.15), (15, 30, 5), (0.3, 0.4, 0.3)),
        obj(CUBE, pbr((0.9, 0.7, 0.4), roughness=0.35, metallic=0.8), (0.22, -0.3, -0.2), (-10, -40, 20),
            (0.25, 0.25, 0.25)),
        obj(CUBE, dielectric(ior=1.5), (0.02, -0.28, 0.22), (30, 45, 0), (0.2, 0.2, 0.2)),
        light,
    ]
    spec.camera["aperture"] = float(aperture)
    spec.camera["focus_distance"] = float(focus_distance)
    spec.name = f"cornell_cubes{res}"
    return spec


def image_tex(index: int, scale: float = 1.0) -> dict:
    """An IMAGE texture slot: spec.images[index] at texture_scale `scale`."""
    return {"image": int(index), "scale": float(scale)}


def cornell_textured(res: int = 64, spp: int = 4, depth: int = 8, seed: int = 0) -> SceneSpec:
    """The Cornell box with image textures: a checker albedo on the back
    wall (scale 0.5, so the uvs wrap), a PBR sphere and a PBR cube whose
    albedo, roughness, metallic and normal come from images (the normal map
    tilts the shading normal through the tangent frame), and the ceiling
    light's emission from an image, generated from a fixed seed."""
    spec = cornell(res=res, spp=spp, depth=depth, seed=seed)
    rng = np.random.default_rng(7)
    n = 16
    yy, xx = np.mgrid[0:n, 0:n]
    checker = ((xx // 4 + yy // 4) % 2).astype(np.float64)
    albedo = np.stack([40 + 200 * checker, 60 + 150 * (1 - checker), 90 + 0 * checker]).astype(np.uint8)
    rough = np.repeat((40 + 180 * rng.random((1, n, n))).astype(np.uint8), 3, axis=0)
    metal = np.repeat((255 * (rng.random((1, n, n)) > 0.5)).astype(np.uint8), 3, axis=0)
    # tangent-space normals: a bumpy field around +z, stored as n * 0.5 + 0.5
    ang = rng.random((2, n, n)) * 0.6 - 0.3
    nz = np.sqrt(np.maximum(1.0 - ang[0] ** 2 - ang[1] ** 2, 0.0))
    normal = np.clip(np.stack([ang[0], ang[1], nz]) * 127.5 + 127.5, 0, 255).astype(np.uint8)
    colour = (40 + 200 * rng.random((3, n, n))).astype(np.uint8)
    spec.images = [albedo, rough, metal, normal, colour]
    back = dict(spec.objects[4])
    back["material"] = _mat(LAMBERTIAN, tex=[image_tex(0, 0.5)] + [(0.0, 0.0, 0.0)] * 4)
    textured_pbr = _mat(PBR, tex=[image_tex(4), image_tex(1), image_tex(2), (0.0, 0.0, 0.0), image_tex(3)])
    light = dict(spec.objects[-1])  # the ceiling light's emission from an image too
    light["material"] = dict(light["material"], tex=[image_tex(4)] + list(light["material"]["tex"][1:]))
    spec.objects = spec.objects[:4] + [back] + [
        obj(SPHERE, textured_pbr, (-0.22, -0.2, -0.15), radius=0.3),
        obj(CUBE, textured_pbr, (0.22, -0.3, -0.2), (10, -35, 5), (0.3, 0.3, 0.3)),
        obj(SPHERE, dielectric(ior=1.5), (0.02, -0.25, 0.22), radius=0.3),
        light,
    ]
    spec.name = f"cornell_textured{res}"
    return spec


# ---------------------------------------------------------------------------
# mesh stress configuration

def icosphere(levels: int) -> tuple[np.ndarray, np.ndarray]:
    """Unit icosphere: 20*4^levels faces, 10*4^levels + 2 vertices."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t],
                  [0, -1, -t], [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]],
                 dtype=np.float64)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9],
                  [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2],
                  [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10],
                  [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    for _ in range(levels):
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        e.sort(axis=1)
        uniq, inv = np.unique(e, axis=0, return_inverse=True)
        mid = v[uniq[:, 0]] + v[uniq[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = len(v)
        v = np.concatenate([v, mid])
        nf = len(f)
        a, b, c = (inv[:nf] + base), (inv[nf:2 * nf] + base), (inv[2 * nf:] + base)
        f = np.concatenate([np.stack([f[:, 0], a, c], 1), np.stack([f[:, 1], b, a], 1),
                            np.stack([f[:, 2], c, b], 1), np.stack([a, b, c], 1)])
    return v, f


def value_noise(p: np.ndarray, seed: int, octaves: int = 4, base_freq: float = 2.0) -> np.ndarray:
    """Sum of `octaves` trilinearly interpolated lattice noises in [-1, 1]
    (frequency doubling, amplitude halving), normalised to [-1, 1]."""
    rng = np.random.default_rng(seed)
    table = rng.uniform(-1.0, 1.0, size=4096)
    perm = rng.permutation(4096)

    def lattice(ix, iy, iz):
        h = perm[(ix * 73856093 ^ iy * 19349663 ^ iz * 83492791) & 4095]
        return table[h]

    out = np.zeros(len(p))
    amp, freq, norm = 1.0, base_freq, 0.0
    for _ in range(octaves):
        q = p * freq
        i = np.floor(q).astype(np.int64)
        fr = q - i
        s = fr * fr * (3.0 - 2.0 * fr)
        acc = 0.0
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    w = ((s[:, 0] if dx else 1 - s[:, 0]) * (s[:, 1] if dy else 1 - s[:, 1])
                         * (s[:, 2] if dz else 1 - s[:, 2]))
                    acc = acc + w * lattice(i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz)
        out += amp * acc
        norm += amp
        amp *= 0.5
        freq *= 2.0
    return out / norm


def write_obj(path: Path, v: np.ndarray, f: np.ndarray, n: np.ndarray | None = None,
              uv: np.ndarray | None = None) -> None:
    """OBJ with positions, optional normals and optional texture coordinates
    (with uv, faces are written v/vt/vn, or v/vt without normals)."""
    v32 = v.astype(np.float32)
    lines = ["# nectarrender_b200 generated mesh"]
    lines += [f"v {a:.9g} {b:.9g} {c:.9g}" for a, b, c in v32]
    if uv is not None:
        lines += [f"vt {a:.9g} {b:.9g}" for a, b in uv.astype(np.float32)]
        if n is not None:
            lines += [f"vn {a:.9g} {b:.9g} {c:.9g}" for a, b, c in n.astype(np.float32)]
            lines += [f"f {a}/{a}/{a} {b}/{b}/{b} {c}/{c}/{c}" for a, b, c in (f + 1)]
        else:
            lines += [f"f {a}/{a} {b}/{b} {c}/{c}" for a, b, c in (f + 1)]
    elif n is not None:
        lines += [f"vn {a:.9g} {b:.9g} {c:.9g}" for a, b, c in n.astype(np.float32)]
        lines += [f"f {a}//{a} {b}//{b} {c}//{c}" for a, b, c in (f + 1)]
    else:
        lines += [f"f {a} {b} {c}" for a, b, c in (f + 1)]
    path.write_text("\n".join(lines) + "\n")


def displaced_icosphere(levels: int, seed: int, amplitude: float = 0.05):
    v, f = icosphere(levels)
    d = value_noise(v, seed)
    v = v * (1.0 + amplitude * d)[:, None]
    # area-weighted vertex normals of the displaced surface
    fn = np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 0]])
    n = np.zeros_like(v)
    for k in range(3):
        np.add.at(n, f[:, k], fn)
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    return v, f, n


def write_hdr(path: Path, rgb: np.ndarray) -> None:
    """Radiance RGBE, flat scanlines, -Y H +X W orientation."""
    h, w, _ = rgb.shape
    m = rgb.max(axis=2)
    e = np.zeros_like(m, dtype=np.int32)
    mant = np.zeros_like(m)
    pos = m > 1e-32
    mant[pos], e[pos] = np.frexp(m[pos])
    scale = np.where(pos, mant * 256.0 / np.where(pos, m, 1.0), 0.0)
    out = np.zeros((h, w, 4), dtype=np.uint8)
    out[..., :3] = np.clip(rgb * scale[..., None], 0, 255).astype(np.uint8)
    out[..., 3] = np.where(pos, e + 128, 0).astype(np.uint8)
    with open(path, "wb") as fh:
        fh.write(b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n")
        fh.write(f"-Y {h} +X {w}\n".encode())
        fh.write(out.tobytes())


def procedural_hdri(width: int, height: int, seed: int, sun_radiance: float = 1e4) -> np.ndarray:
    """Log-normal sky exp(z), z a smooth unit-variance random field (mu=0,
    sigma=1), slightly blue, plus a sun disk of 0.6 degree radius."""
    rng = np.random.default_rng(seed)
    coarse = rng.standard_normal((height // 64 + 2, width // 64 + 2))
    yy = np.linspace(0, coarse.shape[0] - 1.001, height)
    xx = np.linspace(0, coarse.shape[1] - 1.001, width)
    y0, x0 = np.floor(yy).astype(int), np.floor(xx).astype(int)
    ty, tx = (yy - y0)[:, None], (xx - x0)[None, :]
    z = ((coarse[y0][:, x0] * (1 - tx) + coarse[y0][:, x0 + 1] * tx) * (1 - ty)
         + (coarse[y0 + 1][:, x0] * (1 - tx) + coarse[y0 + 1][:, x0 + 1] * tx) * ty)
    z = (z - z.mean()) / z.std()
    sky = np.exp(z)[..., None] * np.array([0.75, 0.85, 1.0])
    # sun: direction at elevation 40 deg, azimuth 30 deg, in the sampler's (u, v) convention
    u = (np.arange(width) + 0.5) / width
    v = (np.arange(height) + 0.5) / height
    phi = (u - 0.5) * 2 * np.pi
    theta = v * np.pi
    dx = np.sin(theta)[:, None] * np.cos(phi)[None, :]
    dz = np.sin(theta)[:, None] * np.sin(phi)[None, :]
    dy = np.cos(theta)[:, None] * np.ones((1, width))
    el, az = math.radians(40.0), math.radians(30.0)
    s = np.array([math.cos(el) * math.cos(az), math.sin(el), math.cos(el) * math.sin(az)])
    cosang = dx * s[0] + dy * s[1] + dz * s[2]
    sun = cosang > math.cos(math.radians(0.6))
    sky[sun] = sun_radiance
    return sky.astype(np.float32)


def uv_sphere(n_lat: int = 24, n_lon: int = 48):
    """Latitude-longitude unit sphere with texture coordinates (u along the
    longitude, v along the latitude; the seam and the poles duplicate
    vertices) and normals: (v, f, n, uv)."""
    lat = np.linspace(0.0, math.pi, n_lat + 1)
    lon = np.linspace(0.0, 2.0 * math.pi, n_lon + 1)
    th, ph = np.meshgrid(lat, lon, indexing="ij")
    v = np.stack([np.sin(th) * np.cos(ph), np.cos(th), np.sin(th) * np.sin(ph)], -1).reshape(-1, 3)
    uv = np.stack([ph / (2.0 * math.pi), 1.0 - th / math.pi], -1).reshape(-1, 2)
    idx = np.arange((n_lat + 1) * (n_lon + 1)).reshape(n_lat + 1, n_lon + 1)
    a, b = idx[:-1, :-1].ravel(), idx[:-1, 1:].ravel()
    c, d = idx[1:, :-1].ravel(), idx[1:, 1:].ravel()
    f = np.concatenate([np.stack([a, c, b], 1), np.stack([b, c, d], 1)])
    # drop the zero-area triangles at the poles
    area = np.linalg.norm(np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 0]]), axis=1)
    return v, f[area > 1e-9], v.copy(), uv


def cornell_textured_mesh(res: int = 64, spp: int = 4, depth: int = 8, seed: int = 0) -> SceneSpec:
    """The textured Cornell box with a uv-mapped sphere mesh (OBJ with vt
    and vn) carrying the image-textured PBR material: mesh texture
    coordinates, the tangents the mesh loader derives from them, and normal
    maps on a mesh."""
    spec = cornell_textured(res=res, spp=spp, depth=depth, seed=seed)
    ASSETS.mkdir(parents=True, exist_ok=True)
    obj_path = ASSETS / "uv_sphere_24x48.obj"
    if not obj_path.exists():
        v, f, n, uv = uv_sphere()
        tmp = obj_path.with_suffix(f".{os.getpid()}.tmp")  # unique per writer process
        write_obj(tmp, v, f, n, uv)
        tmp.replace(obj_path)
    spec.meshes = [str(obj_path)]
    textured_pbr = spec.objects[5]["material"]
    light = spec.objects[-1]
    spec.objects = spec.objects[:5] + [
        obj(MESH, textured_pbr, (-0.2, -0.22, -0.1), (20, 30, 0), (0.28, 0.28, 0.28), mesh=0),
        spec.objects[6],
        light,
    ]
    spec.name = f"cornell_textured_mesh{res}"
    return spec


def mesh_stress(levels: int = 8, res_h: int = 1080, res_w: int = 1920, spp: int = 256,
                depth: int = 12, seed: int = 0, n_spheres: int = 256,
                hdri_size: tuple[int, int] = (2048, 1024), scene_seed: int = 0) -> SceneSpec:
    ASSETS.mkdir(parents=True, exist_ok=True)
    obj_path = ASSETS / f"icosphere_l{levels}_s{scene_seed}.obj"
    hdr_path = ASSETS / f"sky_{hdri_size[0]}x{hdri_size[1]}_s{scene_seed}.hdr"
    if not obj_path.exists():
        v, f, n = displaced_icosphere(levels, scene_seed)
        tmp = obj_path.with_suffix(f".{os.getpid()}.tmp")  # unique per writer process
        write_obj(tmp, v, f, n)
        tmp.replace(obj_path)
    if not hdr_path.exists():
        tmp = hdr_path.with_suffix(f".{os.getpid()}.tmp")
        write_hdr(tmp, procedural_hdri(hdri_size[0], hdri_size[1], scene_seed))
        tmp.replace(hdr_path)
    rng = np.random.default_rng(scene_seed + 1)
    mesh_mat = pbr(tuple(rng.uniform(0.2, 0.9, 3)), roughness=float(rng.uniform(0.05, 0.6)),
                   metallic=float(rng.integers(0, 2)))
    objs = [obj(MESH, mesh_mat, (0, 0, 0), (0, 0, 0), (1, 1, 1), mesh=0)]
    placed: list[tuple[np.ndarray, float]] = []
    while len(placed) < n_spheres:
        r = float(rng.uniform(0.05, 0.3))
        p = rng.uniform([-3.2, -1.6, -3.0], [3.2, 1.6, 1.6])
        if np.linalg.norm(p) < 1.06 + r:
            continue
        if any(np.linalg.norm(p - q) < r + s for q, s in placed):
            continue
        placed.append((p, r))
    for p, r in placed:
        kind = int(rng.integers(0, 3))
        if kind == 0:
            m = lambertian(tuple(rng.uniform(0.1, 0.9, 3)))
        elif kind == 1:
            m = pbr(tuple(rng.uniform(0.1, 0.9, 3)), roughness=float(rng.uniform(0.05, 0.6)),
                    metallic=float(rng.integers(0, 2)))
        else:
            m = dielectric(ior=float(rng.uniform(1.3, 1.7)))
        objs.append(obj(SPHERE, m, p, radius=r))
    # The reference maps resolution[0] to image rows and uses it as the
    # horizontal extent of the sensor (camera.h:176-178 vs :269-272): with
    # resolution (H, W) = (1080, 1920) the visible window is offset to the
    # upper right of the optical axis, so the camera is turned to centre it.
    cam_pos = np.array([0.0, 0.2, 4.2])
    uvw_x = FOV40_SENSOR
    uvw_y = -FOV40_SENSOR * (res_w / res_h)
    u_c = ((res_w - 1) / 2 - (res_h - 1) / 2) * (uvw_x / res_h)
    v_c = ((res_h - 1) / 2 - (res_w - 1) / 2) * (uvw_y / res_w)
    yaw = math.degrees(math.atan2(u_c, 1.0))
    pitch = -math.degrees(math.atan2(v_c, 1.0)) - math.degrees(math.atan2(cam_pos[1], cam_pos[2]))
    cam = camera(res_h, res_w, cam_pos, (pitch, yaw, 0.0), spp + 1)
    sky = {"type": SKY_HDRI, "path": str(hdr_path), "rotation": 0.0, "intensity": 1.0}
    return SceneSpec(objects=objs, camera=cam, ray_depth=depth, seed=seed, sky=sky,
                     meshes=[str(obj_path)], name=f"mesh_stress_l{levels}_{res_h}x{res_w}")


def medium_stress(levels: int = 8, res_h: int = 1080, res_w: int = 1920, spp: int = 256,
                  depth: int = 32, seed: int = 0, n_spheres: int = 256,
                  hdri_size: tuple[int, int] = (2048, 1024), scene_seed: int = 0) -> SceneSpec:
    """The mesh-stress scene inside a 2x2x2 box of isotropic homogeneous
    medium (sigma_t = 0.5, albedo 0.9) centred on the mesh, depth 32: the
    radiance-cache configuration."""
    spec = mesh_stress(levels, res_h, res_w, spp, depth, seed, n_spheres, hdri_size, scene_seed)
    spec.objects.append(obj(MEDIUM, isotropic((0.9, 0.9, 0.9)), (0, 0, 0), (0, 0, 0), (2, 2, 2),
                            wrapped=CUBE, density=0.5))
    spec.name = f"medium_stress_l{levels}_{res_h}x{res_w}"
    return spec


def batch_set(n: int = 64, seed: int = 0) -> list[SceneSpec]:
    """The batched configuration: n independent scenes from the Cornell and
    mesh-stress generators, triangle counts log-uniform in 10k-2M (rounded
    to the nearest icosphere subdivision, levels 5-8), resolutions 256-1024
    a side in steps of 16, 16-256 samples, depth 4-16. Meshes of one level
    share their OBJ file (and the level-8 one is the mesh-stress workload's);
    the spheres, camera, samples and depth differ per scene."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        res_h, res_w = (int(rng.integers(16, 65)) * 16 for _ in range(2))
        spp = int(rng.integers(1, 17)) * 16
        depth = int(rng.integers(4, 17))
        if i % 4 == 0:
            s = cornell(res=res_h, spp=spp, depth=depth, seed=int(rng.integers(1 << 16)))
        else:
            tris = math.exp(rng.uniform(math.log(1e4), math.log(2e6)))
            level = int(min(8, max(5, round(math.log(tris / 20.0, 4)))))
            s = mesh_stress(levels=level, res_h=res_h, res_w=res_w, spp=spp, depth=depth,
                            n_spheres=int(rng.integers(8, 129)), hdri_size=(512, 256),
                            scene_seed=0, seed=int(rng.integers(1 << 16)))
        s.name = f"batch{seed}_{i}"
        out.append(s)
    return out


# ---------------------------------------------------------------------------
# spec -> _pathtracer objects (the reference's Python API)

def to_pathtracer(spec: SceneSpec, pt=None):
    """Builds (scene, camera) with the reference's API on this back end."""
    if pt is None:
        from . import pathtracer
        pt = pathtracer()
    V3, C = pt.core.vector.Vector3, pt.core.vector.Color
    M, H, T = pt.material.Material, pt.hittable.Hittable, pt.material.texture.Texture

    def material(d):
        t = d["type"]
        if any(isinstance(c, dict) for c in d["tex"]):
            raise NotImplementedError("image texture slots of a spec go through capi.Scene "
                                      "(Texture.from_image reads image files)")
        tex = [T.from_color(C(*c)) for c in d["tex"]]
        if t == LAMBERTIAN:
            return M.lambertian(tex[0])
        if t == PBR:
            return M.pbr(*tex)
        if t == DIELECTRIC:
            return M.dielectric(C(*d["tint"]), d["ior"])
        if t == EMISSIVE:
            return M.emissive(tex[0], d["brightness"])
        if t == ISOTROPIC:
            return M.isotropic(tex[0])
        return M()

    def shape(o, t, mat):
        p, r, s = V3(*o["position"]), V3(*o["rotation"]), V3(*o["scale"])
        if t == QUAD:
            return H.quad(p, r, s, mat)
        if t == CUBE:
            return H.cube(p, r, s, mat)
        if t == SPHERE:
            return H.sphere(p, o["radius"], mat)
        if t == MESH:
            return H.mesh(spec.meshes[o["mesh"]], p, r, s, mat)
        raise ValueError(t)

    hittables, lights = [], []
    for o in spec.objects:
        t = o["type"]
        if t in (LIGHT, MEDIUM):
            bound = shape(o, o["wrapped_type"], M())
            d = o["material"]
            if t == LIGHT:
                h = H.object_light(bound, d["brightness"], T.from_color(C(*d["tex"][0])))
                lights.append(h)
            else:
                h = H.constant_medium(bound, o["density"], T.from_color(C(*d["tex"][0])))
                hittables.append(h)
        else:
            hittables.append(shape(o, t, material(o["material"])))
    L = pt.light.Skylight
    if spec.sky["type"] == SKY_SIMPLE:
        sky = L.simple(C(*spec.sky["start"]), C(*spec.sky["end"]))
    elif spec.sky["type"] == SKY_HDRI:
        sky = L.hdri(spec.sky["path"])
        sky.config_hdri().rotation = spec.sky.get("rotation", 0.0)
        sky.config_hdri().intensity = spec.sky.get("intensity", 1.0)
    else:
        sky = L()
    scene = pt.scene.Scene(hittables, lights, sky)
    c = spec.camera
    params = pt.engine.camera.CameraParams(
        pt.core.vector.Vector2(*c["resolution"]), V3(*c["position"]), V3(*c["rotation"]),
        c["samples_per_pixel"], c["focal_length"], c["focus_distance"], c["aperture"],
        c["sensor_width"], c["shutter_speed"])
    cam = pt.engine.camera.Camera(params)
    return scene, cam, (hittables, lights, sky)


def from_pathtracer(scene, camera, ray_depth: int, seed: int, name: str = "") -> SceneSpec:
    """The SceneSpec of a scene built with the `_pathtracer` factories
    (``Scene(hittables, lights, skylight)``, ``Camera(params)``), read back
    through ``Scene.describe()``; the inverse of ``to_pathtracer``. Values
    are the stored float32 ones."""
    meshes: list[str] = []
    objects = []
    desc = scene.describe()
    for d in desc["objects"]:
        m = d["material"]
        tex = [tuple(t) if not isinstance(t, str) else t for t in m["tex"]]
        mat = {"type": m["type"], "ior": m["ior"], "brightness": m["brightness"],
               "tint": tuple(m["tint"]), "tex": tex}
        base = d["wrapped_type"] or d["type"]
        mesh = -1
        if base == MESH:
            if d["mesh_path"] not in meshes:
                meshes.append(d["mesh_path"])
            mesh = meshes.index(d["mesh_path"])
        objects.append(obj(d["type"], mat, d["position"], d["rotation"], d["scale"], d["radius"],
                           mesh=mesh, wrapped=d["wrapped_type"], density=d["density"]))
    s = desc["sky"]
    if s["type"] == SKY_SIMPLE:
        sky = {"type": SKY_SIMPLE, "start": tuple(s["start"]), "end": tuple(s["end"])}
    elif s["type"] == SKY_HDRI:
        sky = {"type": SKY_HDRI, "path": s["path"], "rotation": s["rotation"],
               "intensity": s["intensity"]}
    else:
        sky = {"type": SKY_NULL}
    p = camera.parameters()
    cam = {"resolution": (p.resolution.x(), p.resolution.y()),
           "position": (p.position.x(), p.position.y(), p.position.z()),
           "rotation": (p.rotation.x(), p.rotation.y(), p.rotation.z()),
           "samples_per_pixel": int(p.samples_per_pixel), "focal_length": p.focal_length,
           "focus_distance": p.focus_distance, "aperture": p.aperture,
           "sensor_width": p.sensor_width, "shutter_speed": p.shutter_speed}
    return SceneSpec(objects=objects, camera=cam, ray_depth=int(ray_depth), seed=int(seed),
                     sky=sky, meshes=meshes, name=name)


def spec_to_json(spec: SceneSpec) -> dict:
    """A JSON-ready dict of a spec (tuples and arrays become lists)."""
    import dataclasses
    return json_ready(dataclasses.asdict(spec))


def json_ready(x):
    if isinstance(x, np.ndarray):
        return x.tolist()
    if isinstance(x, dict):
        return {k: json_ready(v) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return [json_ready(v) for v in x]
    return x


def spec_from_json(d: dict) -> SceneSpec:
    """Inverse of spec_to_json (lists become tuples where the spec has tuples)."""
    def tup(v):
        return tuple(tup(x) for x in v) if isinstance(v, list) else v
    objects = []
    for o in d["objects"]:
        o = {k: tup(v) if k != "material" else v for k, v in o.items()}
        m = dict(o["material"])
        m["tint"] = tuple(m["tint"])
        m["tex"] = [tuple(t) if isinstance(t, list) else t for t in m["tex"]]
        o["material"] = m
        objects.append(o)
    cam = {k: tup(v) for k, v in d["camera"].items()}
    sky = {k: tup(v) for k, v in d["sky"].items()}
    images = [np.asarray(im, np.uint8) for im in d.get("images", [])]
    return SceneSpec(objects=objects, camera=cam, ray_depth=d["ray_depth"], seed=d["seed"],
                     sky=sky, meshes=list(d["meshes"]), name=d.get("name", ""), images=images)


def scene_set(n: int = 16, seed: int = 0, max_level: int = 6) -> list[SceneSpec]:
    """A seeded set of small scenes of mixed size for the multi-scene
    workload: Cornell boxes and mesh-stress scenes (icosphere levels 3 to
    max_level), resolutions 256 to 512 in steps of 16, 16 to 64 samples,
    depth 4 to 16."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        res = int(rng.integers(16, 33)) * 16
        spp = int(rng.choice([16, 32, 64]))
        depth = int(rng.integers(4, 17))
        if i % 4 == 0:
            s = cornell(res=res, spp=spp, depth=depth, seed=int(rng.integers(1 << 16)))
        else:
            s = mesh_stress(levels=int(rng.integers(3, max_level + 1)), res_h=res,
                            res_w=int(rng.integers(16, 33)) * 16, spp=spp, depth=depth,
                            n_spheres=int(rng.integers(8, 65)), hdri_size=(256, 128),
                            scene_seed=100 + i)
        s.name = f"set{seed}_{i}"
        out.append(s)
    return out
