"""ctypes view of the C ABI in include/nectar_b200.h.

`Scene` and `Render` wrap the opaque handles; every call checks the status
code and raises RuntimeError with nr_last_error() on failure. This is the
plain-pointer boundary a non-Python host would bind;
the pybind11 module `_pathtracer` sits on the same functions.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import library
from .scenes import SKY_HDRI, SKY_SIMPLE, SceneSpec

c_float3 = C.c_float * 3


class TextureDesc(C.Structure):
    _fields_ = [("type", C.c_int32), ("image", C.c_int32), ("scale", C.c_float), ("rgb", c_float3)]


class MaterialDesc(C.Structure):
    _fields_ = [("type", C.c_int32), ("ior", C.c_float), ("brightness", C.c_float),
                ("tint", c_float3), ("tex", TextureDesc * 5)]


class ObjectDesc(C.Structure):
    _fields_ = [("type", C.c_int32), ("wrapped_type", C.c_int32), ("material", C.c_int32),
                ("mesh", C.c_int32), ("position", c_float3), ("rotation", c_float3),
                ("scale", c_float3), ("radius", C.c_float), ("density", C.c_float)]


class CameraDesc(C.Structure):
    _fields_ = [("resolution", C.c_float * 2), ("position", c_float3), ("rotation", c_float3),
                ("samples_per_pixel", C.c_uint32), ("focal_length", C.c_float),
                ("focus_distance", C.c_float), ("aperture", C.c_float),
                ("sensor_width", C.c_float), ("shutter_speed", C.c_float)]


class RenderConfig(C.Structure):
    _fields_ = [("ray_depth", C.c_uint32), ("seed", C.c_uint32), ("rr_enabled", C.c_int32),
                ("rr_start_bounce", C.c_uint32), ("rr_survival", C.c_float), ("mode", C.c_int32),
                ("schedule", C.c_int32), ("fp64_accumulate", C.c_int32), ("layer_mask", C.c_uint32),
                ("extend_variant", C.c_int32), ("samples_per_wave", C.c_uint32),
                ("use_graphs", C.c_int32), ("tail_max_paths", C.c_uint32),
                ("shade_variant", C.c_int32), ("sort_materials", C.c_int32),
                ("max_traversal_steps", C.c_uint32), ("traversal_stack_limit", C.c_uint32)]


class StreamConfig(C.Structure):
    _fields_ = [("linear_to_gamma", C.c_int32), ("apply_white_balance", C.c_int32),
                ("wb_temperature", C.c_float), ("wb_tint", C.c_float),
                ("apply_tonemapping", C.c_int32), ("tm_method", C.c_int32),
                ("tm_white_point", C.c_float), ("tm_alpha", C.c_float)]


class SceneStats(C.Structure):
    _fields_ = [("n_objects", C.c_uint32), ("n_materials", C.c_uint32), ("n_lights", C.c_uint32),
                ("n_triangles", C.c_uint64), ("binary_nodes", C.c_uint64),
                ("wide_nodes", C.c_uint64), ("sah_cost_binary", C.c_double),
                ("build_ms", C.c_double), ("device_bytes", C.c_uint64)]


KERNEL_CLASSES = ("generate", "extend", "shade", "rotate", "accumulate", "megakernel")


class KernelProfile(C.Structure):
    _fields_ = [("ms", C.c_double * 6), ("launches", C.c_uint32 * 6)]


class PickResult(C.Structure):
    _fields_ = [("hit", C.c_int32), ("object_id", C.c_uint32), ("material_id", C.c_uint32),
                ("t", C.c_float), ("p", c_float3), ("n", c_float3), ("uv", C.c_float * 2),
                ("front_face", C.c_int32)]


class TraceCounters(C.Structure):
    _fields_ = [("rays", C.c_uint64), ("node_visits", C.c_uint64), ("tri_tests", C.c_uint64),
                ("obj_tests", C.c_uint64), ("paths", C.c_uint64)]


# symbols declared in include/nectar_b200.h
# nr_render_config.schedule
SCHEDULE_MEGAKERNEL = 0
SCHEDULE_WAVEFRONT = 1
# nr_render_config.mode
MODE_REFERENCE = 0
MODE_PERF = 1

EXPORTS = [
    "nr_abi_version", "nr_last_error", "nr_device_count", "nr_device_memory_info",
    "nr_device_draw_order",
    "nr_set_draw_order", "nr_scene_create", "nr_scene_destroy",
    "nr_scene_add_material", "nr_scene_add_image", "nr_scene_add_mesh", "nr_scene_get_mesh",
    "nr_scene_load_obj", "nr_scene_load_obj_device",
    "nr_scene_add_object", "nr_scene_set_sky_null", "nr_scene_set_sky_simple",
    "nr_scene_set_sky_hdri", "nr_scene_load_hdr", "nr_scene_set_hdri_params",
    "nr_scene_set_tuning", "nr_scene_set_bvh_width", "nr_scene_build",
    "nr_scene_get_stats", "nr_scene_get_bounds", "nr_scene_get_sky_tables", "nr_scene_get_binary_bvh", "nr_render_config_default",
    "nr_render_create", "nr_render_destroy", "nr_render_reset", "nr_render_samples",
    "nr_render_samples_static", "nr_render_samples_batch", "nr_render_set_profiling",
    "nr_render_get_profile",
    "nr_render_graph_stats", "nr_render_set_fused_display", "nr_host_alloc", "nr_host_free", "nr_render_viewport", "nr_render_pick", "nr_render_selection_mask",
    "nr_conv3x3_forward_device", "nr_conv3x3_wgrad_device",
    "nr_denoiser_create", "nr_denoiser_destroy", "nr_denoiser_set_loss",
    "nr_denoiser_train_step", "nr_denoiser_infer",
    "nr_denoiser_param_count", "nr_denoiser_get_params", "nr_denoiser_set_params",
    "nr_denoiser_layers", "nr_nrc_create", "nr_nrc_destroy", "nr_nrc_infer", "nr_nrc_train",
    "nr_nrc_count", "nr_nrc_get", "nr_nrc_set", "nr_render_set_nrc", "nr_render_nrc_stats",
    "nr_render_sample_layers", "nr_render_trace_log", "nr_render_layer_device_ptr", "nr_render_read_layer",
    "nr_render_read_beauty_fp64", "nr_render_read_beauty_fp64_sum", "nr_render_readback", "nr_render_display_float",
    "nr_render_dims", "nr_render_set_counters", "nr_render_get_counters", "nr_render_last_ms",
    "nr_render_stream", "nr_accumulate_device", "nr_display_device",
]


def device_draw_order() -> int:
    """0: multi-draw constructor arguments consume draws left to right (the
    reference's CUDA build), 1: right to left (its host build)."""
    return int(library().nr_device_draw_order())


def _check(rc: int, what: str) -> None:
    if rc != 0:
        raise RuntimeError(f"{what}: {library().nr_last_error().decode()} (status {rc})")


def material_desc(d: dict) -> MaterialDesc:
    m = MaterialDesc()
    m.type = d["type"]
    m.ior = d.get("ior", 1.5)
    m.brightness = d.get("brightness", 35.0)
    m.tint = c_float3(*d.get("tint", (1.0, 1.0, 1.0)))
    for k in range(5):
        t = TextureDesc()
        slot = d["tex"][k]
        if isinstance(slot, dict):  # IMAGE: an index into the spec's images
            t.type, t.image, t.scale = 1, int(slot["image"]), float(slot.get("scale", 1.0))
            t.rgb = c_float3(0.0, 0.0, 0.0)
        else:
            t.type, t.image, t.scale = 0, -1, 1.0
            t.rgb = c_float3(*slot)
        m.tex[k] = t
    return m


def object_desc(o: dict, material: int) -> ObjectDesc:
    d = ObjectDesc()
    d.type = o["type"]
    d.wrapped_type = o.get("wrapped_type", 0)
    d.material = material
    d.mesh = o.get("mesh", -1)
    d.position = c_float3(*o["position"])
    d.rotation = c_float3(*o["rotation"])
    d.scale = c_float3(*o["scale"])
    d.radius = o.get("radius", 1.0)
    d.density = o.get("density", 1.0)
    return d


def camera_desc(c: dict) -> CameraDesc:
    d = CameraDesc()
    d.resolution = (C.c_float * 2)(*c["resolution"])
    d.position = c_float3(*c["position"])
    d.rotation = c_float3(*c["rotation"])
    d.samples_per_pixel = c["samples_per_pixel"]
    d.focal_length = c["focal_length"]
    d.focus_distance = c["focus_distance"]
    d.aperture = c["aperture"]
    d.sensor_width = c["sensor_width"]
    d.shutter_speed = c["shutter_speed"]
    return d


def render_config(spec: SceneSpec, **over) -> RenderConfig:
    cfg = RenderConfig()
    library().nr_render_config_default(C.byref(cfg))
    cfg.ray_depth = spec.ray_depth
    cfg.seed = spec.seed
    for k, v in over.items():
        setattr(cfg, k, v)
    return cfg


def stream_config(gamma=True, white_balance=False, tonemap=True, method=0, temperature=6800.0,
                  tint=1.0, white_point=1.0, alpha=1.0) -> StreamConfig:
    s = StreamConfig()
    s.linear_to_gamma = int(gamma)
    s.apply_white_balance = int(white_balance)
    s.wb_temperature = temperature
    s.wb_tint = tint
    s.apply_tonemapping = int(tonemap)
    s.tm_method = method
    s.tm_white_point = white_point
    s.tm_alpha = alpha
    return s


class Scene:
    """An nr_scene built from a SceneSpec (registry semantics of the
    reference: one material per hittable, lights after hittables)."""

    def __init__(self, spec: SceneSpec, build: bool = True, mesh_leaf: int = 1, tlas_leaf: int = 1,
                 obj_on_device: bool = False, mesh_width: int = 8, tlas_width: int = 8):
        """obj_on_device: assemble the OBJ meshes' vertices on the GPU
        (nr_scene_load_obj_device; the same meshes as the host reader).
        mesh_width / tlas_width: children per wide BVH node (4..8)."""
        self.lib = library()
        self.spec = spec
        self.h = C.c_void_p()
        _check(self.lib.nr_scene_create(C.byref(self.h)), "nr_scene_create")
        _check(self.lib.nr_scene_set_tuning(self.h, mesh_leaf, tlas_leaf), "nr_scene_set_tuning")
        _check(self.lib.nr_scene_set_bvh_width(self.h, mesh_width, tlas_width),
               "nr_scene_set_bvh_width")
        load = self.lib.nr_scene_load_obj_device if obj_on_device else self.lib.nr_scene_load_obj
        for path in spec.meshes:
            mid = C.c_uint32()
            _check(load(self.h, path.encode(), C.byref(mid)), "nr_scene_load_obj")
        for im in spec.images:
            im = np.ascontiguousarray(im, np.uint8)
            _check(self.lib.nr_scene_add_image(self.h, im.ctypes.data_as(C.POINTER(C.c_uint8)), im.shape[0],
                                               im.shape[1], im.shape[2], None), "nr_scene_add_image")
        for o in spec.objects:
            mid = C.c_uint32()
            _check(self.lib.nr_scene_add_material(self.h, C.byref(material_desc(o["material"])),
                                                  C.byref(mid)), "nr_scene_add_material")
            _check(self.lib.nr_scene_add_object(self.h, C.byref(object_desc(o, mid.value)), None),
                   "nr_scene_add_object")
        sky = spec.sky
        if sky["type"] == SKY_SIMPLE:
            _check(self.lib.nr_scene_set_sky_simple(self.h, c_float3(*sky["start"]),
                                                    c_float3(*sky["end"])), "sky")
        elif sky["type"] == SKY_HDRI:
            _check(self.lib.nr_scene_load_hdr(self.h, sky["path"].encode(),
                                              C.c_float(sky.get("rotation", 0.0)),
                                              C.c_float(sky.get("intensity", 1.0))), "sky")
        if build:
            self.build()

    def build(self) -> None:
        _check(self.lib.nr_scene_build(self.h), "nr_scene_build")

    def stats(self) -> dict:
        s = SceneStats()
        _check(self.lib.nr_scene_get_stats(self.h, C.byref(s)), "nr_scene_get_stats")
        return {k: getattr(s, k) for k, _ in SceneStats._fields_}

    def bounds(self) -> tuple[np.ndarray, np.ndarray]:
        """World-space box around every object (lo, hi)."""
        lo, hi = np.zeros(3, np.float32), np.zeros(3, np.float32)
        _check(self.lib.nr_scene_get_bounds(self.h, _fptr(lo), _fptr(hi)), "nr_scene_get_bounds")
        return lo, hi

    def mesh(self, mesh_id: int = 0):
        """(positions, normals, tangents, uvs, triangles) as stored after parsing."""
        nv, nt = C.c_uint32(), C.c_uint32()
        _check(self.lib.nr_scene_get_mesh(self.h, mesh_id, None, None, None, None, None,
                                          C.byref(nv), C.byref(nt)), "nr_scene_get_mesh")
        P = np.zeros(3 * nv.value, np.float32)
        N, T = np.zeros_like(P), np.zeros_like(P)
        UV = np.zeros(2 * nv.value, np.float32)
        tris = np.zeros(3 * nt.value, np.uint32)
        _check(self.lib.nr_scene_get_mesh(self.h, mesh_id, _fptr(P), _fptr(N), _fptr(T), _fptr(UV),
                                          tris.ctypes.data_as(C.POINTER(C.c_uint32)),
                                          C.byref(nv), C.byref(nt)), "nr_scene_get_mesh")
        return P, N, T, UV, tris

    def binary_bvh(self, mesh_id: int = 0) -> tuple[np.ndarray, np.ndarray]:
        n = C.c_uint64()
        _check(self.lib.nr_scene_get_binary_bvh(self.h, mesh_id, None, C.byref(n), None), "bvh")
        nodes = np.zeros((n.value, 8), dtype=np.float32)
        order = np.zeros(n.value, dtype=np.uint32)
        _check(self.lib.nr_scene_get_binary_bvh(
            self.h, mesh_id, nodes.ctypes.data_as(C.POINTER(C.c_float)), C.byref(n),
            order.ctypes.data_as(C.POINTER(C.c_uint32))), "bvh")
        return nodes, order

    def __del__(self):
        if getattr(self, "h", None) and self.h.value:
            self.lib.nr_scene_destroy(self.h)
            self.h = None  # module globals may already be gone at exit


def _fptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_float))


def render_batch(renders, first, count) -> None:
    """nr_render_samples_batch over Render objects (first/count: lists)."""
    n = len(renders)
    hs = (C.c_void_p * n)(*[r.h.value for r in renders])
    fa = (C.c_uint32 * n)(*first)
    ca = (C.c_uint32 * n)(*count)
    _check(library().nr_render_samples_batch(hs, n, fa, ca), "nr_render_samples_batch")


class Render:
    def __init__(self, scene: Scene, spec: SceneSpec | None = None, **cfg_over):
        self.lib = library()
        self.scene = scene
        spec = spec or scene.spec
        self.cam = camera_desc(spec.camera)
        self.cfg = render_config(spec, **cfg_over)
        self.h = C.c_void_p()
        _check(self.lib.nr_render_create(scene.h, C.byref(self.cam), C.byref(self.cfg),
                                         C.byref(self.h)), "nr_render_create")
        dims = (C.c_uint32(), C.c_uint32(), C.c_uint32())
        self.lib.nr_render_dims(self.h, *map(C.byref, dims))
        self.C, self.H, self.W = (d.value for d in dims)
        self.spp = spec.camera["samples_per_pixel"]

    def samples(self, first: int, count: int) -> None:
        _check(self.lib.nr_render_samples(self.h, first, count), "nr_render_samples")

    def render_all(self) -> None:
        """The reference's render(): sample indices 1 .. spp-1."""
        self.samples(1, self.spp - 1)

    def sample_layers(self, sample_idx: int):
        b = np.zeros((3, self.H, self.W), np.float32)
        d = np.zeros_like(b)
        n = np.zeros_like(b)
        p = np.zeros((self.H, self.W), np.uint32)
        _check(self.lib.nr_render_sample_layers(self.h, sample_idx, _fptr(b), _fptr(d), _fptr(n),
                                                p.ctypes.data_as(C.POINTER(C.c_uint32))),
               "nr_render_sample_layers")
        return b, d, n, p

    def trace_log(self, sample_idx: int, max_bounces: int):
        """(log, beauty) of nr_render_trace_log: log is (H, W, max_bounces,
        16) float32, beauty the raw (3, H, W) sample."""
        log = np.zeros((self.H, self.W, max_bounces, 16), np.float32)
        b = np.zeros((3, self.H, self.W), np.float32)
        _check(self.lib.nr_render_trace_log(self.h, sample_idx, max_bounces, _fptr(log), _fptr(b)),
               "nr_render_trace_log")
        return log, b

    def layer(self, layer: int = 0) -> np.ndarray:
        out = np.zeros((3, self.H, self.W), np.float32)
        _check(self.lib.nr_render_read_layer(self.h, layer, _fptr(out)), "nr_render_read_layer")
        return out

    def layer_channels(self, layer: int) -> np.ndarray:
        """An enabled layer of any channel count (the depth layer has one)."""
        c = 1 if layer in (5, 6) else 3
        out = np.zeros((c, self.H, self.W), np.float32)
        _check(self.lib.nr_render_read_layer(self.h, layer, _fptr(out)), "nr_render_read_layer")
        return out

    def beauty_fp64(self) -> np.ndarray:
        out = np.zeros((3, self.H, self.W), np.float64)
        _check(self.lib.nr_render_read_beauty_fp64(self.h, out.ctypes.data_as(C.POINTER(C.c_double))),
               "nr_render_read_beauty_fp64")
        return out

    def beauty_fp64_sum(self) -> tuple[np.ndarray, int]:
        """(FP64 sum of beauty over the samples since the last reset, their count)."""
        out = np.zeros((3, self.H, self.W), np.float64)
        n = C.c_uint64()
        _check(self.lib.nr_render_read_beauty_fp64_sum(
            self.h, out.ctypes.data_as(C.POINTER(C.c_double)), C.byref(n)),
            "nr_render_read_beauty_fp64_sum")
        return out, int(n.value)

    def readback(self, layer: int = 0, cfg: StreamConfig | None = None) -> np.ndarray:
        out = np.zeros((3, self.H, self.W), np.uint8)
        cfg = cfg or stream_config()
        _check(self.lib.nr_render_readback(self.h, layer, C.byref(cfg),
                                           out.ctypes.data_as(C.POINTER(C.c_uint8))), "readback")
        return out

    def display_float(self, layer: int = 0, cfg: StreamConfig | None = None) -> np.ndarray:
        out = np.zeros((3, self.H, self.W), np.float32)
        cfg = cfg or stream_config()
        _check(self.lib.nr_render_display_float(self.h, layer, C.byref(cfg), _fptr(out)), "display")
        return out

    def counters(self, on: bool = True) -> None:
        self.lib.nr_render_set_counters(self.h, int(on))

    def last_counters(self) -> dict:
        c = TraceCounters()
        self.lib.nr_render_get_counters(self.h, C.byref(c))
        return {k: getattr(c, k) for k, _ in TraceCounters._fields_}

    def profiling(self, on: bool = True) -> None:
        _check(self.lib.nr_render_set_profiling(self.h, int(on)), "nr_render_set_profiling")

    def last_profile(self) -> dict:
        """{kernel class: (device ms, launches)} of the last samples() call."""
        p = KernelProfile()
        _check(self.lib.nr_render_get_profile(self.h, C.byref(p)), "nr_render_get_profile")
        return {k: (p.ms[i], p.launches[i]) for i, k in enumerate(KERNEL_CLASSES)}

    def viewport(self, show_axis_grid: bool = True) -> None:
        _check(self.lib.nr_render_viewport(self.h, int(show_axis_grid)), "nr_render_viewport")

    def pick(self, u: float, v: float) -> dict:
        r = PickResult()
        _check(self.lib.nr_render_pick(self.h, C.c_float(u), C.c_float(v), C.byref(r)),
               "nr_render_pick")
        return {"hit": bool(r.hit), "object_id": r.object_id, "material_id": r.material_id,
                "t": r.t, "p": tuple(r.p), "n": tuple(r.n), "uv": tuple(r.uv),
                "front_face": bool(r.front_face)}

    def selection_mask(self, object_id: int, outline_radius: int = 2) -> np.ndarray:
        out = np.zeros((self.H, self.W), np.uint8)
        _check(self.lib.nr_render_selection_mask(self.h, object_id, outline_radius,
                                                 out.ctypes.data_as(C.POINTER(C.c_uint8))),
               "nr_render_selection_mask")
        return out

    def set_nrc(self, cache, terminate_bounce: int = 2, train_one_in: int = 32,
                lr: float = 1e-2, batch: int = 16384, min_steps: int = 4) -> None:
        """Attach a nectarrender_b200.nrc.RadianceCache (None detaches)."""
        self._nrc = cache  # keep it alive while attached
        _check(self.lib.nr_render_set_nrc(self.h, cache.h if cache else None, terminate_bounce,
                                          train_one_in, C.c_float(lr), batch, min_steps),
               "nr_render_set_nrc")

    def nrc_stats(self) -> tuple[int, int]:
        q, t = C.c_uint64(), C.c_uint64()
        _check(self.lib.nr_render_nrc_stats(self.h, C.byref(q), C.byref(t)), "nr_render_nrc_stats")
        return q.value, t.value

    def graph_stats(self) -> tuple[int, int]:
        """(wave graphs captured, graph replays) of this render so far."""
        cap, rep = C.c_uint32(), C.c_uint64()
        _check(self.lib.nr_render_graph_stats(self.h, C.byref(cap), C.byref(rep)), "graph_stats")
        return cap.value, rep.value

    def last_ms(self) -> float:
        v = C.c_double()
        self.lib.nr_render_last_ms(self.h, C.byref(v))
        return v.value

    def reset(self) -> None:
        _check(self.lib.nr_render_reset(self.h), "nr_render_reset")

    def __del__(self):
        if getattr(self, "h", None) and self.h.value:
            self.lib.nr_render_destroy(self.h)
            self.h = None  # module globals may already be gone at exit
