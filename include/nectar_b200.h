/*
 * nectar_b200.h — C ABI of the B200 path-tracing back end.
 *
 * This is the drop-in boundary for NectarRender's path-tracing hot path. The
 * reference exposes that path through its pybind11 module `_pathtracer`
 * (nectar_render/csrc/bindings/bindings.cpp:16-30); the classes it binds are
 * backed here by plain C entry points with opaque handles, plain pointers and
 * sizes, and integer status codes. The pybind11 module shipped in
 * nectarrender_b200/csrc/pathtracer_module.cpp re-creates the reference's
 * Python names on top of these functions.
 *
 * Conventions
 *  - Every function returns NR_OK (0) or a negative NR_ERR_* code; the last
 *    error message of the calling thread is available from nr_last_error().
 *    The reference throws std::runtime_error in the same situations
 *    (e.g. nectar_render/csrc/engine/include/engine/camera.h:317-319,
 *    nectar_render/csrc/hittable/include/hittable/registry.h:113-117).
 *  - Images are planar CHW float32, index c*H*W + y*W + x, exactly the AOV
 *    layout of nectar_render/csrc/data/include/data/render_layers.h:28-55 and
 *    nectar_render/csrc/data/include/data/utils.h:9-21.
 *  - Resolution follows the reference's camera: resolution[0] is the image
 *    height H and resolution[1] its width W when buffers are sized
 *    (camera.h:176-178), while the pixel-to-sensor mapping uses
 *    resolution[0] as its horizontal extent (camera.h:269-272). Square images
 *    are therefore the only fully consistent case, exactly as in the reference.
 *  - No function allocates on, or touches, a GPU until nr_scene_build /
 *    nr_render_create. Without a usable CUDA device these return
 *    NR_ERR_NO_DEVICE; there is no CPU fallback.
 */
#ifndef NECTAR_B200_H
#define NECTAR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NR_ABI_VERSION 1

/* status codes ------------------------------------------------------------ */
#define NR_OK 0
#define NR_ERR_INVALID (-1)   /* bad argument or handle                       */
#define NR_ERR_CUDA (-2)      /* a CUDA runtime call failed                   */
#define NR_ERR_LIMIT (-3)     /* a registry/capacity limit was exceeded       */
#define NR_ERR_IO (-4)        /* a file could not be read or parsed           */
#define NR_ERR_NO_DEVICE (-5) /* no usable CUDA device                        */
#define NR_ERR_STATE (-6)     /* call out of order (e.g. render before build) */
#define NR_ERR_DEVICE (-7)    /* a kernel reported an error word (overflow)   */

/* limits of the reference registries -------------------------------------- */
#define NR_MAX_OBJECTS 1024   /* registry.h:104  MAX_REGISTRY_ENTRIES          */
#define NR_MAX_MATERIALS 4096 /* material/registry.h:11 MAX_MATERIAL_COUNT     */

/* enums: values mirror the reference enums ------------------------------- */
/* HittableType, nectar_render/csrc/hittable/include/hittable/hittable.h:13-15 */
enum {
  NR_HITTABLE_NULL = 0,
  NR_HITTABLE_QUAD = 1,
  NR_HITTABLE_SPHERE = 2,
  NR_HITTABLE_CUBE = 3,
  NR_HITTABLE_MESH = 4,
  NR_HITTABLE_CONSTANT_MEDIUM = 5,
  NR_HITTABLE_OBJECT_LIGHT = 6
};
/* MaterialType, nectar_render/csrc/material/include/material/material.h:374-376 */
enum {
  NR_MATERIAL_NULL = 0,
  NR_MATERIAL_LAMBERTIAN = 1,
  NR_MATERIAL_PBR = 2,
  NR_MATERIAL_DIELECTRIC = 3,
  NR_MATERIAL_EMISSIVE = 4,
  NR_MATERIAL_ISOTROPIC = 5
};
/* TextureType, nectar_render/csrc/material/include/material/texture.h:6 */
enum { NR_TEXTURE_CONSTANT = 0, NR_TEXTURE_IMAGE = 1 };
/* SkylightType, nectar_render/csrc/light/include/skylight.h:131 */
enum { NR_SKY_NULL = 0, NR_SKY_SIMPLE = 1, NR_SKY_HDRI = 2 };
/* LayerType, nectar_render/csrc/data/include/data/render_layers.h:11-14 */
enum {
  NR_LAYER_BEAUTY = 0,
  NR_LAYER_DIFFUSE = 1,
  NR_LAYER_SPECULAR = 2,
  NR_LAYER_OBJECT_NORMAL = 3,
  NR_LAYER_WORLD_NORMAL = 4,
  NR_LAYER_SHADOW = 5,
  NR_LAYER_DEPTH = 6,
  NR_LAYER_EMISSION = 7,
  NR_LAYER_OBJECT_ID = 8
};
/* TonemapMethod, nectar_render/csrc/data/include/data/stream.h:12 */
enum { NR_TONEMAP_REINHARD = 0, NR_TONEMAP_REINHARD_EXTENDED = 1, NR_TONEMAP_ACES = 2 };

/* Integrator modes.
 * NR_MODE_REFERENCE reproduces the reference sampler draw for draw
 *   (nectar_render/csrc/engine/src/trace.cu:11-79 and brdf.cu:4-35).
 * NR_MODE_PERF keeps every BSDF but adds next-event estimation with
 *   power-heuristic MIS toward lights[0] and toward the HDRI (importance
 *   sampled through an alias table). It converges to the same image. */
enum { NR_MODE_REFERENCE = 0, NR_MODE_PERF = 1 };

/* Integrator schedules: one persistent megakernel with path regeneration, or
 * the wavefront pipeline (generate / extend / shade / shadow / accumulate). */
enum { NR_SCHEDULE_MEGAKERNEL = 0, NR_SCHEDULE_WAVEFRONT = 1 };

/* scene description --------------------------------------------------------- */

/* One texture slot: Texture::from_color / Texture::from_image (texture.h:145-177). */
typedef struct nr_texture_desc {
  int32_t type;  /* NR_TEXTURE_CONSTANT or NR_TEXTURE_IMAGE                   */
  int32_t image; /* image id from nr_scene_add_image (IMAGE only)             */
  float scale;   /* texture_scale (IMAGE only)                                */
  float rgb[3];  /* constant_color (CONSTANT only)                            */
} nr_texture_desc;

/* One material (Material::lambertian/pbr/dielectric/emissive/isotropic,
 * material.h:453-532). Texture slots: LAMBERTIAN, EMISSIVE, ISOTROPIC use
 * tex[0]; PBR uses albedo, roughness, metallic, emission, normal in tex[0..4]. */
typedef struct nr_material_desc {
  int32_t type;     /* NR_MATERIAL_*                     */
  float ior;        /* DIELECTRIC                        */
  float brightness; /* EMISSIVE                          */
  float tint[3];    /* DIELECTRIC                        */
  nr_texture_desc tex[5];
} nr_material_desc;

/* One hittable (Hittable::quad/cube/sphere/mesh/object_light/constant_medium,
 * hittable.h:148-277). For OBJECT_LIGHT and CONSTANT_MEDIUM, wrapped_type and
 * the transform/radius/mesh fields describe the bound object, whose transform
 * the wrapper inherits (hittable.h:231-233, 261-263). */
typedef struct nr_object_desc {
  int32_t type;         /* NR_HITTABLE_*                                  */
  int32_t wrapped_type; /* bound object type for OBJECT_LIGHT / MEDIUM    */
  int32_t material;     /* material id; 0 = default purple Lambertian     */
  int32_t mesh;         /* mesh id for MESH (or a wrapped MESH)           */
  float position[3];
  float rotation[3]; /* Euler degrees, R = Rz*Ry*Rx (matrix.h:94-96)      */
  float scale[3];
  float radius;  /* SPHERE (or wrapped SPHERE)                             */
  float density; /* CONSTANT_MEDIUM                                        */
} nr_object_desc;

/* CameraParams (nectar_render/csrc/engine/include/engine/camera.h:351-405). */
typedef struct nr_camera_desc {
  float resolution[2];
  float position[3];
  float rotation[3];
  uint32_t samples_per_pixel;
  float focal_length;
  float focus_distance;
  float aperture;
  float sensor_width;
  float shutter_speed;
} nr_camera_desc;

/* TraceConfig (nectar_render/csrc/engine/include/engine/trace.h:10-19) plus
 * this back end's schedule, mode and accumulator options. */
typedef struct nr_render_config {
  uint32_t ray_depth;
  uint32_t seed;
  int32_t rr_enabled;       /* do_rr_termination                            */
  uint32_t rr_start_bounce; /* rr_start_bounce                              */
  float rr_survival;        /* rr_survival_chance                           */
  int32_t mode;             /* NR_MODE_*                                    */
  int32_t schedule;         /* NR_SCHEDULE_*                                */
  int32_t fp64_accumulate;  /* also keep an FP64 sum of the beauty layer    */
  uint32_t layer_mask;      /* bit i enables LayerType i (default 0x13).
                               DEPTH (bit 6, one channel) holds the running
                               mean of the first hit's world distance (0 on
                               a miss), written by the wavefront schedule;
                               the reference allocates it but never writes
                               it. The other optional layers stay zero, as
                               in the reference (engine/src/trace.cu:47-79) */
  int32_t extend_variant;   /* wavefront traversal kernel: 4, 5, 6, 8 = nested
                               two-level traversal with that many CTAs per
                               SM; 14..18 = flattened traversal with lane
                               refill; 64, 74, 84 = 14 with each iteration
                               running one kind of work (primitive tests or
                               the rest) chosen by a warp vote; 100*a + b =
                               a for bounce 0, b after; 0 = default (574).
                               Every variant finds the same hits.           */
  uint32_t samples_per_wave;/* wavefront: sample indices per wave (0 = ~8M paths) */
  int32_t use_graphs;       /* wavefront: replay each wave as a CUDA graph (1) */
  uint32_t tail_max_paths;  /* wavefront, reference mode: from bounce 4 on, a
                               queue of at most this many paths is finished
                               by one per-path launch (0 = 131072,
                               0xFFFFFFFF = never)                          */
  int32_t shade_variant;    /* wavefront shading kernel register budget: 5 or
                               6 CTAs of 128 threads per SM, any other value
                               128 registers; 0 = default (6)               */
  int32_t sort_materials;   /* wavefront: from bounce 1 on, shade the queue
                               grouped by material type (misses first): the
                               extend kernel counts the keys, one pass sorts
                               the queue; 1 = on, negative = off, 0 = default
                               (on)                                         */
  uint32_t max_traversal_steps;   /* bound on the steps of one BVH traversal;
                                     reaching it ends that query and sets
                                     error bit 8 (the call returns
                                     NR_ERR_DEVICE): 0 = default (2^20)     */
  uint32_t traversal_stack_limit; /* bound on the entries of a traversal
                                     stack (below each kernel's own depth);
                                     a push past it is dropped and sets
                                     error bit 1: 0 = no extra bound        */
} nr_render_config;

/* StreamConfig display fields (nectar_render/csrc/data/include/data/stream.h:13-30). */
typedef struct nr_stream_config {
  int32_t linear_to_gamma;
  int32_t apply_white_balance;
  float wb_temperature;
  float wb_tint;
  int32_t apply_tonemapping;
  int32_t tm_method;
  float tm_white_point;
  float tm_alpha;
} nr_stream_config;

/* Statistics of a built scene. */
typedef struct nr_scene_stats {
  uint32_t n_objects;
  uint32_t n_materials;
  uint32_t n_lights;
  uint64_t n_triangles;
  uint64_t binary_nodes;     /* binary SAH tree nodes, all meshes + top level */
  uint64_t wide_nodes;       /* 8-wide compressed nodes after collapse        */
  double sah_cost_binary;    /* SAH cost of the largest mesh's binary tree     */
  double build_ms;           /* device time of the last nr_scene_build         */
  uint64_t device_bytes;     /* scene bytes resident in HBM                    */
} nr_scene_stats;

/* Per-launch counters for the roofline (filled when counters are enabled). */
typedef struct nr_trace_counters {
  uint64_t rays;        /* extension + shadow ray queries                    */
  uint64_t node_visits; /* wide-node fetches (80 B each)                     */
  uint64_t tri_tests;   /* triangle records fetched (48 B each)              */
  uint64_t obj_tests;   /* instance/primitive records fetched                */
  uint64_t paths;       /* pixel-samples completed                           */
} nr_trace_counters;

/* Device time per kernel class of the last nr_render_samples call, from CUDA
 * events recorded between consecutive launches on the render stream (filled
 * when profiling is enabled). Index: NR_KERNEL_*. */
enum {
  NR_KERNEL_GENERATE = 0,   /* camera rays of a wave                         */
  NR_KERNEL_EXTEND = 1,     /* closest-hit traversal of a queue              */
  NR_KERNEL_SHADE = 2,      /* materials, sky, RR, next queue                */
  NR_KERNEL_ROTATE = 3,     /* queue swap and wave bookkeeping               */
  NR_KERNEL_ACCUMULATE = 4, /* running mean into the layers                  */
  NR_KERNEL_MEGAKERNEL = 5, /* per-pixel schedule                            */
  NR_KERNEL_CLASSES = 6
};
typedef struct nr_kernel_profile {
  double ms[NR_KERNEL_CLASSES];
  uint32_t launches[NR_KERNEL_CLASSES];
} nr_kernel_profile;

typedef struct nr_scene nr_scene;
typedef struct nr_render nr_render;

/* library ------------------------------------------------------------------ */
int nr_abi_version(void);
const char* nr_last_error(void);
/* Number of CUDA devices visible (0 without a GPU; never fails). */
int nr_device_count(void);
/* Device memory of the current device in bytes: used = total - free
 * (replaces get_cuda_meminfo / CUDAMemInfo,
 * nectar_render/csrc/host/include/host/utils.h:34-38, bound as
 * _pathtracer.host.memory). NR_ERR_NO_DEVICE without a GPU, where the
 * reference ignores cudaMemGetInfo's status. */
int nr_device_memory_info(uint64_t* used, uint64_t* free_bytes, uint64_t* total);
/* Order in which NR_MODE_REFERENCE consumes random draws for the reference's
 * constructor calls that take several draws as arguments (Vector3::random,
 * Quad::random, random_in_unit_disk; C++ leaves it unspecified): 0 = left to
 * right, as the reference's CUDA device code does (measured on sm_100a),
 * 1 = right to left, as its host-compiled code does. */
int nr_device_draw_order(void);
int nr_set_draw_order(int right_to_left);

/* scene (replaces Scene / HittablesRegistry / MaterialRegisty:
 * nectar_render/csrc/scene/include/scene.h:15-77,
 * nectar_render/csrc/hittable/include/hittable/registry.h:101-265,
 * nectar_render/csrc/material/include/material/registry.h:8-103) ---------- */
int nr_scene_create(nr_scene** out);
int nr_scene_destroy(nr_scene* scene);
/* Material id 0 always exists: the default purple Lambertian
 * (material/registry.h:23-25, material.h:650-652). */
int nr_scene_add_material(nr_scene* scene, const nr_material_desc* desc, uint32_t* out_id);
/* uint8 planar CHW image for IMAGE textures (texture.h:8-26). */
int nr_scene_add_image(nr_scene* scene, const uint8_t* chw, uint32_t C, uint32_t H, uint32_t W,
                       uint32_t* out_id);
/* Mesh from arrays (Mesh::set_geometry, mesh.h:169-175): positions/normals/
 * tangents are float[3*n_vertices], uvs float[2*n_vertices] (NULL = zeros),
 * triangles uint32[3*n_triangles]. */
int nr_scene_add_mesh(nr_scene* scene, const float* positions, const float* normals,
                      const float* tangents, const float* uvs, uint32_t n_vertices,
                      const uint32_t* triangles, uint32_t n_triangles, uint32_t* out_id);
/* Reads back mesh `mesh_id` as stored (after OBJ parsing): pass NULL
 * arrays to query n_vertices / n_triangles first. Needs no GPU. */
int nr_scene_get_mesh(const nr_scene* scene, uint32_t mesh_id, float* positions, float* normals,
                      float* tangents, float* uvs, uint32_t* triangles, uint32_t* n_vertices,
                      uint32_t* n_triangles);
/* Wavefront OBJ file (parse_obj_file, mesh.h:39-141): triangulated faces,
 * vertices deduplicated on the (v, vt, vn) index triple, smooth normals when
 * the file has none, per-vertex tangents from uv gradients. */
int nr_scene_load_obj(nr_scene* scene, const char* path, uint32_t* out_id);
/* Same mesh as nr_scene_load_obj, bit for bit, with the vertex assembly
 * (deduplication of the v/vt/vn triples in order of first use, missing
 * normals, tangents) done on the current GPU: the file is parsed on the host,
 * the assembly runs as hash-table, scan, sort and per-vertex kernels. The
 * reference assembles on the host (tinyobjloader + mesh.h:57-116). Fails with
 * NR_ERR_LIMIT when the v, vt and vn index ranges need more than 63 bits
 * together, NR_ERR_NO_DEVICE without a GPU. */
int nr_scene_load_obj_device(nr_scene* scene, const char* path, uint32_t* out_id);
/* Appends a hittable; OBJECT_LIGHT objects are also lights. Scene(hittables,
 * lights, sky) appends lights after the hittables (scene.h:31-39). */
int nr_scene_add_object(nr_scene* scene, const nr_object_desc* desc, uint32_t* out_id);
int nr_scene_set_sky_null(nr_scene* scene);
/* Skylight::simple (skylight.h:211-222). */
int nr_scene_set_sky_simple(nr_scene* scene, const float start_rgb[3], const float end_rgb[3]);
/* Skylight::hdri from float planar CHW data (skylight.h:54-69, texture.h:28-47). */
int nr_scene_set_sky_hdri(nr_scene* scene, const float* chw, uint32_t C, uint32_t H, uint32_t W,
                          float rotation_deg, float intensity);
/* Skylight::hdri(path) from a Radiance RGBE .hdr file (stbi_loadf semantics). */
int nr_scene_load_hdr(nr_scene* scene, const char* path, float rotation_deg, float intensity);
/* HDRISkylightConfig rotation/intensity (skylight.h:14-21) after creation. */
int nr_scene_set_hdri_params(nr_scene* scene, float rotation_deg, float intensity);
/* Leaf sizes of the 8-wide trees (1..3 primitives; defaults: meshes 1,
 * top level 1). Takes effect at the next nr_scene_build. */
int nr_scene_set_tuning(nr_scene* scene, uint32_t mesh_leaf_max, uint32_t tlas_leaf_max);
/* Children per wide node (4..8; default 8) of the mesh trees and of the top
 * level: the node layout stays the 8-wide compressed one, a narrower tree
 * uses fewer of its slots (more, smaller nodes, a deeper tree). Takes effect at the next
 * nr_scene_build. No counterpart in the reference (its trees are binary). */
int nr_scene_set_bvh_width(nr_scene* scene, uint32_t mesh_width, uint32_t tlas_width);
/* Uploads the scene and builds every BVH on the GPU (Scene::build,
 * nectar_render/csrc/scene/src/scene.cpp:68-76). Must precede nr_render_create. */
int nr_scene_build(nr_scene* scene);
int nr_scene_get_stats(const nr_scene* scene, nr_scene_stats* out);
/* World-space box around every object of a built scene (the union of the
 * top-level leaf boxes); the radiance cache's grid spans it. No counterpart
 * in the reference. */
int nr_scene_get_bounds(const nr_scene* scene, float lo[3], float hi[3]);
/* The HDRI importance-sampling tables of a built scene (NR_MODE_PERF; no
 * counterpart in the reference), built on the GPU: texel probabilities
 * [H][W], a row alias table (acceptance probabilities and alias rows, [H])
 * and one column alias table per row ([H][W]); a texel is drawn as row, then
 * column. W and H are 0 without an HDRI; null outputs are skipped; the
 * tables are left unread when the HDRI carries no energy. */
int nr_scene_get_sky_tables(const nr_scene* scene, float* texel_pdf, float* row_prob,
                            uint32_t* row_alias, float* col_prob, uint32_t* col_alias,
                            int32_t* W, int32_t* H);
/* Binary SAH tree of mesh `mesh_id` as built on the GPU, for checks:
 * nodes as float[8] {lo.xyz, hi.xyz, left|prim, right|count} bit patterns
 * (int32 stored in the float slots). Pass NULL to query the count. */
int nr_scene_get_binary_bvh(const nr_scene* scene, uint32_t mesh_id, float* nodes8,
                            uint64_t* n_nodes, uint32_t* prim_order);

/* render (replaces RenderEngine + RenderLayers + trace_full:
 * nectar_render/csrc/engine/include/engine/engine.h:274-380,
 * nectar_render/csrc/engine/src/engine.cpp:42-74,
 * nectar_render/csrc/engine/src/trace.cu:47-94,
 * nectar_render/csrc/data/include/data/render_layers.h:57-190) ----------- */
int nr_render_config_default(nr_render_config* cfg);
int nr_render_create(nr_scene* scene, const nr_camera_desc* camera, const nr_render_config* cfg,
                     nr_render** out);
int nr_render_destroy(nr_render* render);
/* Clears the accumulated layers; the next sample index is 1 (engine.cpp:216-220). */
int nr_render_reset(nr_render* render);
/* Renders sample indices [first, first+count) and folds each into the running
 * mean avg*(n-1)/n + s/n with n = sample index (data.cu:28-50). The reference
 * render() loop is first = 1, count = samples_per_pixel - 1 (engine.cpp:43). */
int nr_render_samples(nr_render* render, uint32_t first, uint32_t count);

/* Renders several scenes at once: renders[i] gets sample indices
 * [first[i], first[i] + count[i]) as nr_render_samples would, but every
 * render's launches are queued on its own stream before any is waited for,
 * so small scenes share the GPU instead of running one after another (the
 * reference renders a scene set with one RenderEngine at a time). A render
 * may appear once per batch. */
int nr_render_samples_batch(nr_render* const* renders, uint32_t n, const uint32_t* first,
                            const uint32_t* count);

/* Fuses the display transform into accumulation: with c set, every later
 * render call's accumulate pass also writes the beauty layer's display bytes
 * (uint8 CHW, the same values nr_render_readback computes for config c), and
 * nr_render_readback of the beauty layer with an identical config only
 * copies them to the host. c = NULL turns it off. No counterpart in the
 * reference, whose accumulate (data.cu:28-50) and process_stream
 * (stream.cu:146-159) are separate kernels. */
int nr_render_set_fused_display(nr_render* render, const nr_stream_config* c);

/* Page-locked host memory for readback buffers (the reference's
 * TransferStream reads back into pinned memory, stream.h:154-182): device to
 * host copies into it run at full link speed. Free with nr_host_free. */
int nr_host_alloc(uint64_t bytes, void** out);
int nr_host_free(void* p);

/* nr_render_samples_static: no counterpart in the reference.
 * Renders exactly like nr_render_samples (same sample indices, same layers,
 * same results; always the wavefront schedule) but allocates no device memory
 * during the call. nr_render_samples allocates its wave state (W*H*samples
 * per wave paths of ~124 B, about 1 GB at 1920x1080) on its first call; this
 * entry point carves that state out of a fixed library-owned device buffer of
 * NR_STATIC_WAVE_BYTES instead. It is for callers that cannot allocate while
 * rendering: a process whose free device memory is already reserved by
 * another allocator (e.g. a framework's caching allocator), or an interactive
 * caller that cannot take the device-wide synchronisation cudaMalloc and
 * cudaFree imply. Everything else the call uses was allocated by
 * nr_render_create.
 *  - Limit: W*H <= NR_STATIC_WAVE_PATHS pixels (e.g. 512x512); larger renders
 *    fail with NR_ERR_LIMIT before any work. A wave holds
 *    NR_STATIC_WAVE_PATHS / (W*H) sample indices (at most the render's
 *    samples_per_wave setting).
 *  - Mode: NR_MODE_REFERENCE renders only; a render created with another
 *    mode fails with NR_ERR_STATE.
 *  - Setup: the first call on each device, with that device current, looks
 *    up the buffer's address (cudaGetSymbolAddress). With CUDA's lazy module
 *    loading this is also when the driver loads the module that holds the
 *    buffer and reserves its NR_STATIC_WAVE_BYTES of device memory, so a
 *    caller that hands its free memory to another allocator, or captures
 *    streams, should make this first call before doing so. A call with
 *    count = 0 does only this set-up (and the argument checks), e.g.
 *    nr_render_samples_static(render, 1, 0). The address is kept per device
 *    ordinal for the rest of the process: it assumes the device's primary
 *    context lives as long as the process (after cudaDeviceReset the library
 *    must not be used on that device again).
 *  - Nothing in the buffer has to start at zero: the first kernel of every
 *    wave resets the queue counters the later kernels read.
 *  - There is one buffer per device per process. Calls that overlap in time
 *    (several host threads, several renders on the same device) race on it
 *    and corrupt each other's paths: serialise them. The call returns when
 *    its work is complete, so calls from one thread never overlap. */
#define NR_STATIC_WAVE_BYTES (32u << 20)
#define NR_STATIC_WAVE_PATHS 270528u
int nr_render_samples_static(nr_render* render, uint32_t first, uint32_t count);
/* Renders one sample index and writes its raw per-sample layers (the
 * reference's sample_aovs before accumulation) to host float CHW buffers;
 * any pointer may be NULL. Used for per-sample parity. */
int nr_render_sample_layers(nr_render* render, uint32_t sample_idx, float* beauty_chw,
                            float* diffuse_chw, float* world_normal_chw, uint32_t* primary_prim);
/* Per-bounce record of one sample index's paths, for diagnosing per-sample
 * differences from the reference (no counterpart in the reference, whose
 * trace_full_kernel, engine/src/trace.cu:47-79, keeps this state in
 * registers). Renders sample_idx like nr_render_sample_layers (raw beauty to
 * `beauty`, 3*H*W floats, may be NULL) and writes, per pixel and bounce b <
 * max_bounces (<= 64), 16 floats at ((y*W + x) * max_bounces + b) * 16: the
 * ray's origin and direction, the hit's registry object id and triangle
 * index as uint32 bits (0xFFFFFFFF: none), its world t, the throughput and
 * the beauty after the bounce, and 1 (as uint32 bits) if the path goes on.
 * Bounces a path never reaches keep all-ones bits. NR_MODE_REFERENCE on the
 * wavefront schedule only (NR_ERR_STATE otherwise). */
int nr_render_trace_log(nr_render* render, uint32_t sample_idx, uint32_t max_bounces,
                        float* host_log, float* beauty);
/* Device pointer of an accumulated layer (DataObject::device_ptr,
 * nectar_render/csrc/data/include/data/data_object.h:163-166). */
int nr_render_layer_device_ptr(nr_render* render, int32_t layer, uint64_t* out_ptr);
/* Copies an accumulated layer to a host float CHW buffer of C*H*W floats. */
int nr_render_read_layer(nr_render* render, int32_t layer, float* host_chw);
/* FP64 sum of beauty (when fp64_accumulate) over every sample rendered since
 * the render was created or reset, divided by the number of those samples:
 * their mean, whatever sample indices they had (a rank's shard of sample
 * indices gives the mean of its shard). */
int nr_render_read_beauty_fp64(nr_render* render, double* host_chw);
/* The same FP64 sum undivided, and the number of samples in it: what a rank
 * rendering a shard of sample indices contributes to a sum over ranks. */
int nr_render_read_beauty_fp64_sum(nr_render* render, double* host_chw, uint64_t* n_samples);
/* Display transform of a layer (process_stream_kernel, stream.cu:146-159):
 * white balance -> tonemap -> sqrt gamma -> clamp -> uint8 CHW, into host memory. */
int nr_render_readback(nr_render* render, int32_t layer, const nr_stream_config* cfg,
                       uint8_t* host_chw);
/* Same transform in float before quantisation (the RMSE domain). */
int nr_render_display_float(nr_render* render, int32_t layer, const nr_stream_config* cfg,
                            float* host_chw);
int nr_render_dims(const nr_render* render, uint32_t* C, uint32_t* H, uint32_t* W);
/* Counters of the last nr_render_samples call when enabled. */
int nr_render_set_counters(nr_render* render, int32_t enabled);
int nr_render_get_counters(const nr_render* render, nr_trace_counters* out);
/* Per-kernel device time of the last nr_render_samples call when enabled. */
int nr_render_set_profiling(nr_render* render, int32_t enabled);
int nr_render_get_profile(const nr_render* render, nr_kernel_profile* out);
/* Wave graphs captured and replayed by this render so far (use_graphs). */
int nr_render_graph_stats(const nr_render* render, uint32_t* captured, uint64_t* replays);
/* Device time in milliseconds of the last nr_render_samples call (CUDA events
 * on the render stream). */
int nr_render_last_ms(const nr_render* render, double* out_ms);
/* Opaque cudaStream_t of the render (for callers that time or order work). */
int nr_render_stream(const nr_render* render, uint64_t* out_stream);

/* viewport ----------------------------------------------------------------- */
/* Shaded preview into the beauty / diffuse / world-normal layers (overwrites
 * them): headlight + directional shading of the material's viewport colour,
 * sky (optionally under the axis grid) on a miss; one centre ray per pixel
 * (RenderEngine::viewport -> trace_viewport_kernel,
 * nectar_render/csrc/engine/src/engine.cpp:77-95, trace.cu:100-162). */
int nr_render_viewport(nr_render* render, int32_t show_axis_grid);
/* Closest hit of the screen-space ray through (u, v) in [0,1]^2
 * (hit_test_ray_kernel, trace.cu:168-188; SceneInterface::query_scene). */
typedef struct nr_pick_result {
  int32_t hit;
  uint32_t object_id;    /* HitRecord::object_id                            */
  uint32_t material_id;  /* HitRecord::material_id                          */
  float t;
  float p[3];
  float n[3];
  float uv[2];
  int32_t front_face;
} nr_pick_result;
int nr_render_pick(nr_render* render, float u, float v, nr_pick_result* out);
/* Outline mask (H x W uint8, 255 on the outline) of the pixels whose centre
 * ray hits `object_id` (selection_mask, nectar_render/csrc/scene/src/
 * scene_interface.cu:54-81). */
int nr_render_selection_mask(nr_render* render, uint32_t object_id, int32_t outline_radius,
                             uint8_t* host_hw);

/* learned denoiser building blocks (no reference counterpart: they replace
 * the OIDN stage, nectar_render/csrc/data/include/data/denoise.h:21-104) -- */
/* 3x3 convolution, stride 1, zero padding 1, over NHWC BF16 tensors of B
 * images of H x W pixels (B*H*W a multiple of 128): y[p, y_off + co] =
 * act(bias[co] + sum_{tap, ci} x[p + off(tap), x_off + ci] * w[tap][co][ci]),
 * FP32 accumulation on the tcgen05 tensor cores; act = ReLU when relu != 0.
 * cin, cout: multiples of 16 up to 256; strides and offsets in channels,
 * multiples of 8. Device pointers; runs on `stream`. */
int nr_conv3x3_forward_device(const void* x, int32_t x_stride, int32_t x_off, const void* w,
                              const float* bias, void* y, int32_t y_stride, int32_t y_off,
                              int32_t cin, int32_t cout, int32_t B, int32_t H, int32_t W,
                              int32_t relu, uint64_t stream);
/* Weight gradient of the same convolution, accumulated into FP32
 * dw[tap][co][ci] += sum_p dy[p, dy_off + co] * x[p + off(tap), x_off + ci]
 * (cout <= 128). */
int nr_conv3x3_wgrad_device(const void* dy, int32_t dy_stride, int32_t dy_off, const void* x,
                            int32_t x_stride, int32_t x_off, float* dw, int32_t cin,
                            int32_t cout, int32_t B, int32_t H, int32_t W, uint64_t stream);

/* Learned denoiser: a five-level U-Net (32 -> 128 channels) on the beauty,
 * diffuse and world-normal layers (the inputs the reference hands to OIDN,
 * nectar_render/csrc/data/include/data/stream.h:160-170) plus the depth
 * layer, convolutions on the tcgen05 tensor cores, trained on the GPU.
 * Images are device float planar CHW, B images of H x W stacked
 * ([B][3][H][W]; depth [B][1][H][W], may be NULL); H and W multiples of 16;
 * B*H*W at most the max_pixels given at creation. */
typedef struct nr_denoiser nr_denoiser;
int nr_denoiser_create(uint32_t max_pixels, uint32_t seed, nr_denoiser** out);
int nr_denoiser_destroy(nr_denoiser* d);
/* Training loss in log space, per channel d = log(1+out) - log(1+target):
 * 1 = absolute error |d| (the default), 0 = squared error 0.5 d^2. */
int nr_denoiser_set_loss(nr_denoiser* d, int32_t kind);
/* One training step toward `target`: forward, loss, backward and (lr > 0)
 * an Adam update; lr <= 0 only computes gradients. *loss = the mean loss
 * before the update. */
int nr_denoiser_train_step(nr_denoiser* d, const float* beauty, const float* diffuse,
                           const float* normal, const float* depth, const float* target,
                           int32_t B, int32_t H, int32_t W, float lr, double* loss,
                           uint64_t stream);
int nr_denoiser_infer(nr_denoiser* d, const float* beauty, const float* diffuse,
                      const float* normal, const float* depth, float* out, int32_t B, int32_t H,
                      int32_t W, uint64_t stream);
/* Parameters (what = 0) or the last step's gradients (what = 1) as host
 * float arrays, layer by layer: weights [9][cout][cin] then bias [cout]. */
int nr_denoiser_param_count(const nr_denoiser* d, uint64_t* out);
int nr_denoiser_get_params(const nr_denoiser* d, int32_t what, float* host);
int nr_denoiser_set_params(nr_denoiser* d, const float* host);
/* Layer count and (cin, cout) pairs in parameter order. */
int nr_denoiser_layers(const nr_denoiser* d, int32_t* count, int32_t* cin_cout);

/* Neural radiance cache (no reference counterpart): a multiresolution
 * hash-grid encoding of position (16 levels x 2 features, 2^19 entries per
 * level, resolutions 16..2048 inside [lo, hi]) plus direction, normal,
 * roughness and albedo, into an MLP of four hidden layers of width 64 (its
 * GEMMs run on the tcgen05 tensor cores), trained online with a relative
 * squared error.
 * Queries are device float [count][16]: position, roughness, outgoing
 * direction (unit, away from the surface), -, normal, -, diffuse albedo, -.
 * Radiance in and out: device float [count][3]. */
typedef struct nr_nrc nr_nrc;
int nr_nrc_create(uint32_t max_queries, const float lo[3], const float hi[3], uint32_t seed,
                  nr_nrc** out);
int nr_nrc_destroy(nr_nrc* n);
int nr_nrc_infer(nr_nrc* n, const float* queries, uint32_t count, float* radiance,
                 uint64_t stream);
/* One Adam step (lr <= 0: gradients only; on the hash grid only the entries
 * the queries touched move); *loss (if not null) = mean relative squared
 * error before the step. */
int nr_nrc_train(nr_nrc* n, const float* queries, const float* target, uint32_t count,
                 float lr, double* loss, uint64_t stream);
/* Host copies: what = 0 MLP weights ([64][64] x 4 then [16][64], out x in),
 * 1 their gradients, 2 grid values, 3 grid gradients, 4 the encoded inputs
 * of the last train call ([count][64]). */
int nr_nrc_count(const nr_nrc* n, int32_t what, uint64_t* out);
int nr_nrc_get(const nr_nrc* n, int32_t what, float* host);
int nr_nrc_set(nr_nrc* n, const float* mlp, const float* grid);

/* Attaches a radiance cache to a render in NR_MODE_PERF (cache = NULL
 * detaches it). Paths stop at hit index terminate_bounce and add the
 * cache's radiance times their throughput; one path in train_one_in runs to
 * full depth and leaves a training record at every hit after the first (the
 * radiance measured behind the hit). When lr > 0, after every wave the cache
 * takes max(min_steps, records / batch) Adam steps (batch 0: 16384, capped
 * at the cache's max_queries; min_steps 0: 4), each on an interleaved subset
 * of the wave's records, every record used once. */
int nr_render_set_nrc(nr_render* render, nr_nrc* cache, uint32_t terminate_bounce,
                      uint32_t train_one_in, float lr, uint32_t batch, uint32_t min_steps);
/* Cache queries answered and training records used since attached. */
int nr_render_nrc_stats(const nr_render* render, uint64_t* queries, uint64_t* records);

/* device-pointer level (callers that own their buffers) -------------------- */
/* Fused running-mean accumulate of one sample layer into an average layer on
 * the given stream: avg = avg*(n-1)/n + s/n (accumulate_samples_kernel,
 * nectar_render/csrc/data/src/data.cu:28-50). Pointers are device float CHW. */
int nr_accumulate_device(float* avg, const float* sample, uint32_t C, uint32_t H, uint32_t W,
                         uint32_t sample_idx, uint64_t stream);
/* Display transform of a device float CHW buffer into device uint8 CHW
 * (process_stream_kernel, nectar_render/csrc/data/src/stream.cu:146-159). */
int nr_display_device(const float* src, uint8_t* dst, uint32_t C, uint32_t H, uint32_t W,
                      const nr_stream_config* cfg, uint64_t stream);

#ifdef __cplusplus
}
#endif
#endif /* NECTAR_B200_H */
