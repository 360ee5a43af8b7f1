"""Checker libraries for the path-tracing hot path — TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package, and only to check or time against it; the product never calls
it.

* ``Oracle``  — liboracle.so, the CPU restatement of the reference integrator
  (oracle.cpp), pinned against the reference itself;
* ``RefCPU``  — _ref/libref_cpu.so, the reference's own integrator headers
  compiled for the host (built here by oracle/Makefile from the reference
  sources, shipped as a binary);
* ``RefCUDA`` — _ref/libref_cuda.so, the reference's CUDA path compiled for
  sm_100a.

Parity is pinned: the restatement is compared bit for bit with RefCPU on the
same seeded scenes and with fixtures generated from it
(tests/test_oracle_golden.py), and RefCPU/RefCUDA are the reference code.

Nothing here loads the product library (libnectar_b200.so): the descriptor
structs below are plain ctypes layouts, and render settings are filled from
this module's own copy of the defaults, so timing a checker never maps the
product. The reference sources are located by the NECTAR_REFERENCE
environment variable (the reference project root); without it only the
prebuilt checkers are used.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

# plain ctypes layouts of include/nectar_b200.h (importing them loads no library)
from nectarrender_b200.capi import CameraDesc, MaterialDesc, ObjectDesc, RenderConfig
from nectarrender_b200.capi import camera_desc, material_desc, object_desc
from nectarrender_b200.scenes import SKY_HDRI, SKY_SIMPLE, SceneSpec

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_CPU_SO = HERE / "_ref" / "libref_cpu.so"
REF_CUDA_SO = HERE / "_ref" / "libref_cuda.so"

# nr_render_config_default (include/nectar_b200.h); tests check that the two agree
RENDER_CONFIG_DEFAULTS = {"ray_depth": 8, "seed": 54321, "rr_enabled": 1, "rr_start_bounce": 3,
                          "rr_survival": 0.95, "mode": 0, "schedule": 1, "fp64_accumulate": 0,
                          "layer_mask": (1 << 0) | (1 << 1) | (1 << 4), "extend_variant": 0,
                          "samples_per_wave": 0, "use_graphs": 1, "tail_max_paths": 0,
                          "shade_variant": 0, "sort_materials": 0, "max_traversal_steps": 0,
                          "traversal_stack_limit": 0}


def render_config(spec: SceneSpec, **over) -> RenderConfig:
    """The render settings of `spec` over the library defaults."""
    cfg = RenderConfig()
    for k, v in RENDER_CONFIG_DEFAULTS.items():
        setattr(cfg, k, v)
    cfg.ray_depth = spec.ray_depth
    cfg.seed = spec.seed
    for k, v in over.items():
        setattr(cfg, k, v)
    return cfg


def reference_sources(root: str | os.PathLike | None = None) -> Path | None:
    """The reference's csrc tree under `root` (default: $NECTAR_REFERENCE), or
    None where it is absent."""
    root = root if root is not None else os.environ.get("NECTAR_REFERENCE")
    if not root:
        return None
    src = Path(root) / "nectar_render" / "csrc"
    return src if src.exists() else None


def build(reference_root: str | os.PathLike | None = None) -> None:
    """make -C oracle: the restatement, and the reference's CPU and CUDA
    builds where the reference sources exist under `reference_root` (default:
    $NECTAR_REFERENCE)."""
    targets = [str(ORACLE_SO)]
    src = reference_sources(reference_root)
    extra = []
    if src is not None:
        targets += [str(REF_CPU_SO), str(REF_CUDA_SO)]
        extra = [f"REF={src}"]
    r = subprocess.run(["make", "-C", str(HERE), *extra, *targets], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout[-4000:] + r.stderr[-4000:])


class OrMesh(C.Structure):
    _fields_ = [("obj_path", C.c_char_p), ("positions", C.POINTER(C.c_float)),
                ("normals", C.POINTER(C.c_float)), ("tangents", C.POINTER(C.c_float)),
                ("uvs", C.POINTER(C.c_float)), ("n_vertices", C.c_uint32),
                ("triangles", C.POINTER(C.c_uint32)), ("n_triangles", C.c_uint32)]


class OrImage(C.Structure):
    _fields_ = [("chw", C.POINTER(C.c_uint8)), ("C", C.c_uint32), ("H", C.c_uint32), ("W", C.c_uint32)]


class OrScene(C.Structure):
    _fields_ = [("materials", C.POINTER(MaterialDesc)), ("n_materials", C.c_uint32),
                ("objects", C.POINTER(ObjectDesc)), ("n_objects", C.c_uint32),
                ("meshes", C.POINTER(OrMesh)), ("n_meshes", C.c_uint32),
                ("sky_type", C.c_int32), ("sky_start", C.c_float * 3), ("sky_end", C.c_float * 3),
                ("hdri", C.POINTER(C.c_float)), ("hdri_C", C.c_uint32), ("hdri_H", C.c_uint32),
                ("hdri_W", C.c_uint32), ("hdri_rotation", C.c_float), ("hdri_intensity", C.c_float),
                ("hdri_path", C.c_char_p), ("images", C.POINTER(OrImage)), ("n_images", C.c_uint32)]


class OrRequest(C.Structure):
    _fields_ = [("first", C.c_uint32), ("count", C.c_uint32), ("mode", C.c_int32),
                ("draw_rtl", C.c_int32), ("row_begin", C.c_uint32), ("row_end", C.c_uint32),
                ("threads", C.c_int32), ("beauty", C.POINTER(C.c_float)),
                ("diffuse", C.POINTER(C.c_float)), ("normal", C.POINTER(C.c_float)),
                ("primary", C.POINTER(C.c_uint32)), ("beauty64", C.POINTER(C.c_double))]


def _f(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class _Lib:
    prefix = ""
    path: Path

    def __init__(self):
        if not self.path.exists():
            raise FileNotFoundError(f"{self.path} not built (oracle/Makefile)")
        self.lib = C.CDLL(str(self.path))
        getattr(self.lib, self.prefix + "mesh_sah").restype = C.c_double
        self._keep: list = []

    def load_obj(self, path: str):
        fn = getattr(self.lib, self.prefix + "load_obj")
        cap_v, cap_t = 1 << 23, 1 << 23
        nv, nt = C.c_uint32(), C.c_uint32()
        P = np.zeros(3 * cap_v, np.float32)
        N, T = np.zeros_like(P), np.zeros_like(P)
        UV = np.zeros(2 * cap_v, np.float32)
        tris = np.zeros(3 * cap_t, np.uint32)
        rc = fn(path.encode(), _f(P), _f(N), _f(T), _f(UV), tris.ctypes.data_as(C.POINTER(C.c_uint32)),
                C.byref(nv), C.byref(nt), cap_v, cap_t)
        if rc != 0:
            raise RuntimeError(f"load_obj failed ({rc}) for {path}")
        v, t = nv.value, nt.value
        return (P[:3 * v].copy(), N[:3 * v].copy(), T[:3 * v].copy(), UV[:2 * v].copy(),
                tris[:3 * t].copy())

    def load_hdr(self, path: str):
        fn = getattr(self.lib, self.prefix + "load_hdr")
        cap = 64 << 20
        buf = np.zeros(cap, np.float32)
        c, h, w = C.c_uint32(), C.c_uint32(), C.c_uint32()
        rc = fn(path.encode(), _f(buf), C.byref(c), C.byref(h), C.byref(w), C.c_uint64(cap))
        if rc != 0:
            raise RuntimeError(f"load_hdr failed ({rc}) for {path}")
        return buf[:c.value * h.value * w.value].reshape(c.value, h.value, w.value).copy()

    def or_scene(self, spec: SceneSpec) -> OrScene:
        keep = []
        mats = [MaterialDesc()]
        d0 = mats[0]
        d0.type = 1
        d0.tex[0].rgb = (C.c_float * 3)(1.0, 0.0, 1.0)
        d0.tex[0].scale = 1.0
        objs = []
        for i, o in enumerate(spec.objects):
            mats.append(material_desc(o["material"]))
            objs.append(object_desc(o, i + 1))
        mat_arr = (MaterialDesc * len(mats))(*mats)
        obj_arr = (ObjectDesc * len(objs))(*objs)
        meshes = []
        for p in spec.meshes:
            P, N, T, UV, tris = self.load_obj(p)
            keep += [P, N, T, UV, tris]
            m = OrMesh(p.encode(), _f(P), _f(N), _f(T), _f(UV), len(P) // 3,
                       tris.ctypes.data_as(C.POINTER(C.c_uint32)), len(tris) // 3)
            meshes.append(m)
        mesh_arr = (OrMesh * max(1, len(meshes)))(*meshes)
        s = OrScene()
        s.materials, s.n_materials = mat_arr, len(mats)
        s.objects, s.n_objects = obj_arr, len(objs)
        s.meshes, s.n_meshes = mesh_arr, len(meshes)
        s.sky_type = spec.sky["type"]
        if spec.sky["type"] == SKY_SIMPLE:
            s.sky_start = (C.c_float * 3)(*spec.sky["start"])
            s.sky_end = (C.c_float * 3)(*spec.sky["end"])
        if spec.sky["type"] == SKY_HDRI:
            img = self.load_hdr(spec.sky["path"])
            keep.append(img)
            s.hdri = _f(img)
            s.hdri_C, s.hdri_H, s.hdri_W = img.shape
            s.hdri_rotation = spec.sky.get("rotation", 0.0)
            s.hdri_intensity = spec.sky.get("intensity", 1.0)
            s.hdri_path = spec.sky["path"].encode()
        imgs = []
        for im in spec.images:
            im = np.ascontiguousarray(im, np.uint8)
            keep.append(im)
            imgs.append(OrImage(im.ctypes.data_as(C.POINTER(C.c_uint8)), *im.shape))
        img_arr = (OrImage * max(1, len(imgs)))(*imgs)
        s.images, s.n_images = img_arr, len(imgs)
        keep += [mat_arr, obj_arr, mesh_arr, img_arr]
        self._keep = keep
        return s

    def render(self, spec: SceneSpec, first: int, count: int = 1, mode: int = 1,
               rows: tuple[int, int] | None = None, threads: int = 0, draw_rtl: int = 1,
               fp64: bool = False, cfg: RenderConfig | None = None):
        """mode 0: raw layers of sample `first`; mode 1: running mean of
        samples [first, first+count). Returns (beauty, diffuse, normal,
        primary, beauty64) as numpy arrays."""
        s = self.or_scene(spec)
        cam = camera_desc(spec.camera)
        cfg = cfg or render_config(spec)
        H, W = int(spec.camera["resolution"][0]), int(spec.camera["resolution"][1])
        b = np.zeros((3, H, W), np.float32)
        d, n = np.zeros_like(b), np.zeros_like(b)
        p = np.full((H, W), 0xffffffff, np.uint32)
        b64 = np.zeros((3, H, W), np.float64) if fp64 else None
        r0, r1 = rows or (0, H)
        req = OrRequest(first, count, mode, draw_rtl, r0, r1, threads, _f(b), _f(d), _f(n),
                        p.ctypes.data_as(C.POINTER(C.c_uint32)),
                        b64.ctypes.data_as(C.POINTER(C.c_double)) if fp64 else None)
        rc = getattr(self.lib, self.prefix + "render")(C.byref(s), C.byref(cam), C.byref(cfg),
                                                        C.byref(req))
        if rc != 0:
            raise RuntimeError(f"{self.prefix}render failed ({rc})")
        return b, d, n, p, b64

    def open_scene(self, spec: SceneSpec, draw_rtl: int = 1) -> "SceneHandle":
        """Builds the checker's scene once (files parsed, BVH built on the host)."""
        return SceneHandle(self, spec, draw_rtl)

    def mesh_sah(self, spec: SceneSpec, mesh: int = 0) -> tuple[float, int]:
        P, N, T, UV, tris = self.load_obj(spec.meshes[mesh])
        m = OrMesh(spec.meshes[mesh].encode(), _f(P), _f(N), _f(T), _f(UV), len(P) // 3,
                   tris.ctypes.data_as(C.POINTER(C.c_uint32)), len(tris) // 3)
        nn = C.c_uint64()
        v = getattr(self.lib, self.prefix + "mesh_sah")(C.byref(m), C.byref(nn))
        return float(v), int(nn.value)

    def uniforms(self, seed: int, sub: int, count: int) -> np.ndarray:
        out = np.zeros(count, np.float32)
        getattr(self.lib, self.prefix + "uniforms")(seed, sub, count, _f(out))
        return out


class SceneHandle:
    def __init__(self, lib: "_Lib", spec: SceneSpec, draw_rtl: int):
        self.lib, self.spec = lib, spec
        self.draw_rtl = draw_rtl
        s = lib.or_scene(spec)
        self._keep = lib._keep
        create = getattr(lib.lib, lib.prefix + "scene_create")
        create.restype = C.c_void_p
        self.h = create(C.byref(s), draw_rtl)
        if not self.h:
            raise RuntimeError("scene_create failed")

    def viewport(self, show_axis_grid: bool = True, seed: int | None = None):
        """(beauty, diffuse, normal) of the viewport preview (oracle only)."""
        spec = self.spec
        cam = camera_desc(spec.camera)
        H, W = int(spec.camera["resolution"][0]), int(spec.camera["resolution"][1])
        b = np.zeros((3, H, W), np.float32)
        d, n = np.zeros_like(b), np.zeros_like(b)
        rc = getattr(self.lib.lib, self.lib.prefix + "scene_viewport")(C.c_void_p(self.h), C.byref(cam),
                                                spec.seed if seed is None else seed,
                                                int(show_axis_grid), _f(b), _f(d), _f(n))
        if rc != 0:
            raise RuntimeError(f"oracle_scene_viewport failed ({rc})")
        return b, d, n

    def pick(self, u: float, v: float, seed: int | None = None) -> dict:
        from nectarrender_b200.capi import PickResult
        r = PickResult()
        cam = camera_desc(self.spec.camera)
        rc = getattr(self.lib.lib, self.lib.prefix + "scene_pick")(C.c_void_p(self.h), C.byref(cam),
                                            self.spec.seed if seed is None else seed,
                                            C.c_float(u), C.c_float(v), C.byref(r))
        if rc != 0:
            raise RuntimeError(f"oracle_scene_pick failed ({rc})")
        return {"hit": bool(r.hit), "object_id": r.object_id, "material_id": r.material_id,
                "t": r.t, "p": tuple(r.p), "n": tuple(r.n), "uv": tuple(r.uv),
                "front_face": bool(r.front_face)}

    def selection_mask(self, object_id: int, radius: int = 2, seed: int | None = None):
        spec = self.spec
        cam = camera_desc(spec.camera)
        H, W = int(spec.camera["resolution"][0]), int(spec.camera["resolution"][1])
        out = np.zeros((H, W), np.uint8)
        rc = getattr(self.lib.lib, self.lib.prefix + "scene_selection_mask")(C.c_void_p(self.h), C.byref(cam),
                                                      spec.seed if seed is None else seed,
                                                      int(object_id), int(radius),
                                                      out.ctypes.data_as(C.POINTER(C.c_uint8)))
        if rc != 0:
            raise RuntimeError(f"oracle_scene_selection_mask failed ({rc})")
        return out

    def render(self, first: int, count: int = 1, mode: int = 1, rows=None, threads: int = 0,
               fp64: bool = False, cfg: RenderConfig | None = None, spec: SceneSpec | None = None):
        spec = spec or self.spec
        cam = camera_desc(spec.camera)
        cfg = cfg or render_config(spec)
        H, W = int(spec.camera["resolution"][0]), int(spec.camera["resolution"][1])
        b = np.zeros((3, H, W), np.float32)
        d, n = np.zeros_like(b), np.zeros_like(b)
        p = np.full((H, W), 0xffffffff, np.uint32)
        b64 = np.zeros((3, H, W), np.float64) if fp64 else None
        r0, r1 = rows or (0, H)
        req = OrRequest(first, count, mode, self.draw_rtl, r0, r1, threads, _f(b), _f(d), _f(n),
                        p.ctypes.data_as(C.POINTER(C.c_uint32)),
                        b64.ctypes.data_as(C.POINTER(C.c_double)) if fp64 else None)
        fn = getattr(self.lib.lib, self.lib.prefix + "scene_render")
        rc = fn(C.c_void_p(self.h), C.byref(cam), C.byref(cfg), C.byref(req))
        if rc != 0:
            raise RuntimeError(f"scene_render failed ({rc})")
        return b, d, n, p, b64

    def __del__(self):
        if getattr(self, "h", None):
            getattr(self.lib.lib, self.lib.prefix + "scene_destroy")(C.c_void_p(self.h))
            self.h = None


class Oracle(_Lib):
    prefix = "oracle_"
    path = ORACLE_SO

    def n_rooks(self, n: int, seed: int, draw_rtl: int = 1) -> np.ndarray:
        out = np.zeros(2 * n, np.float32)
        self.lib.oracle_n_rooks(n, seed, draw_rtl, _f(out))
        return out.reshape(n, 2)


def display(img: np.ndarray, cfg) -> tuple[np.ndarray, np.ndarray]:
    """Oracle display transform of a (3, H, W) float image: (uint8, float)."""
    lib = Oracle().lib
    img = np.ascontiguousarray(img, dtype=np.float32)
    hw = img.shape[1] * img.shape[2]
    o8 = np.zeros(img.shape, np.uint8)
    of = np.zeros(img.shape, np.float32)
    lib.oracle_display(_f(img), hw, C.byref(cfg), o8.ctypes.data_as(C.POINTER(C.c_uint8)), _f(of))
    return o8, of


class RefCPU(_Lib):
    prefix = "refcpu_"
    path = REF_CPU_SO

    def n_rooks(self, n: int, seed: int) -> np.ndarray:
        out = np.zeros(2 * n, np.float32)
        self.lib.refcpu_n_rooks(n, seed, _f(out))
        return out.reshape(n, 2)

    def load_image_uint8(self, path: str) -> np.ndarray:
        """The reference's image-texture loader: its planes (C, H, W) as it
        builds them from the decoded file."""
        C_, H_, W_ = C.c_uint32(), C.c_uint32(), C.c_uint32()
        cap = 1 << 26
        buf = np.zeros(cap, np.uint8)
        rc = self.lib.refcpu_load_image_uint8(path.encode(), buf.ctypes.data_as(C.POINTER(C.c_uint8)),
                                              C.byref(C_), C.byref(H_), C.byref(W_), C.c_uint64(cap))
        if rc != 0:
            raise RuntimeError(f"refcpu_load_image_uint8 failed ({rc})")
        n = C_.value * H_.value * W_.value
        return buf[:n].reshape(C_.value, H_.value, W_.value).copy()

    def render(self, spec, first, count=1, mode=1, rows=None, threads=0, draw_rtl=1, fp64=False,
               cfg=None):
        # the reference's host build evaluates multi-draw arguments right to left
        return super().render(spec, first, count, mode, rows, threads, 1, fp64, cfg)


class RefCUDA(_Lib):
    """The reference's CUDA path (sm_100a build of trace.cu, data.cu, cuda.cu,
    scene.cpp) driven through its own host API."""
    prefix = "refcuda_"
    path = REF_CUDA_SO

    def __init__(self):
        if not self.path.exists():
            raise FileNotFoundError(f"{self.path} not built (oracle/Makefile)")
        self.lib = C.CDLL(str(self.path))
        self._keep = []
        self.cpu = RefCPU()  # file readers for the scene description

    def load_obj(self, path):
        return self.cpu.load_obj(path)

    def load_hdr(self, path):
        return self.cpu.load_hdr(path)

    def probe_draw_order(self) -> tuple[int, int]:
        a, b = C.c_int(), C.c_int()
        rc = self.lib.refcuda_probe_draw_order(C.byref(a), C.byref(b))
        if rc != 0:
            raise RuntimeError(f"draw-order probe failed ({rc})")
        return a.value, b.value

    def time_steps(self, spec, first: int, warmup: int, steps: int, spp_per_step: int,
                   cfg=None) -> list[float]:
        """Device ms of each of `steps` timed steps of the reference's render
        loop (trace_full, accumulate, clear and a synchronise per sample;
        `spp_per_step` sample indices per step, from `first`), after `warmup`
        untimed steps, with L2 overwritten between steps."""
        s = self.or_scene(spec)
        cam = camera_desc(spec.camera)
        cfg = cfg or render_config(spec)
        H, W = int(spec.camera["resolution"][0]), int(spec.camera["resolution"][1])
        if H % 16 or W % 16:
            raise ValueError(f"reference CUDA build needs both sizes a multiple of 16, got {H}x{W}")
        if first + (warmup + steps) * spp_per_step > spec.camera["samples_per_pixel"]:
            raise ValueError("sample indices beyond samples_per_pixel")
        out = (C.c_double * steps)()
        rc = self.lib.refcuda_time_steps(C.byref(s), C.byref(cam), C.byref(cfg), first, warmup, steps,
                                         spp_per_step, out)
        if rc != 0:
            raise RuntimeError(f"refcuda_time_steps failed ({rc})")
        return list(out)

    def trace_log(self, spec, sample: int, max_bounces: int, cfg=None):
        """(log, beauty): the per-bounce record of sample index `sample` from
        the reference's own trace_ray (layout of nr_render_trace_log,
        (H, W, max_bounces, 16) float32) and the raw beauty of the sample."""
        s = self.or_scene(spec)
        cam = camera_desc(spec.camera)
        cfg = cfg or render_config(spec)
        H, W = int(spec.camera["resolution"][0]), int(spec.camera["resolution"][1])
        if H % 16 or W % 16:
            raise ValueError(f"reference CUDA build needs both sizes a multiple of 16, got {H}x{W}")
        log = np.zeros((H, W, max_bounces, 16), np.float32)
        b = np.zeros((3, H, W), np.float32)
        rc = self.lib.refcuda_trace_log(C.byref(s), C.byref(cam), C.byref(cfg), sample, max_bounces,
                                        _f(log), _f(b))
        if rc != 0:
            raise RuntimeError(f"refcuda_trace_log failed ({rc})")
        return log, b

    def render(self, spec, first, count=1, mode=1, rows=None, threads=0, draw_rtl=1, fp64=False,
               cfg=None):
        """Returns (beauty, diffuse, normal, elapsed_ms) of the reference's
        CUDA render loop over samples [first, first+count)."""
        s = self.or_scene(spec)
        cam = camera_desc(spec.camera)
        cfg = cfg or render_config(spec)
        H, W = int(spec.camera["resolution"][0]), int(spec.camera["resolution"][1])
        if H % 16 or W % 16:
            # the reference's 16x16-block kernels have no bounds guard
            raise ValueError(f"reference CUDA build needs both sizes a multiple of 16, got {H}x{W}")
        b = np.zeros((3, H, W), np.float32)
        d, n = np.zeros_like(b), np.zeros_like(b)
        req = OrRequest(first, count, mode, 0, 0, H, 0, _f(b), _f(d), _f(n), None, None)
        ms = C.c_double()
        rc = self.lib.refcuda_render(C.byref(s), C.byref(cam), C.byref(cfg), C.byref(req), C.byref(ms))
        if rc != 0:
            raise RuntimeError(f"refcuda_render failed ({rc})")
        return b, d, n, ms.value
