/*
 * oracle.h — C interface shared by the CPU oracle (oracle.cpp, a restatement
 * of the reference integrator) and the reference builds made by
 * oracle/Makefile (ref_cpu_harness.cpp: the reference's own headers compiled
 * for the host; ref_cuda_harness.cu: the reference's CUDA sources).
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the nectarrender_b200 product path
 * links, loads or calls these libraries; tests, the smoke check and the
 * bench's CPU baseline use them as the checker.
 */
#ifndef NR_ORACLE_H
#define NR_ORACLE_H
#include <stdint.h>
#include "../include/nectar_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_mesh {
  const char* obj_path;  /* OBJ file the mesh was read from (reference harnesses parse it) */
  const float* positions; /* 3 per vertex */
  const float* normals;
  const float* tangents;
  const float* uvs;       /* 2 per vertex */
  uint32_t n_vertices;
  const uint32_t* triangles;
  uint32_t n_triangles;
} or_mesh;

/* uint8 planar CHW image of an IMAGE texture (texture.h:8-26), C >= 3. */
typedef struct or_image {
  const uint8_t* chw;
  uint32_t C, H, W;
} or_image;

typedef struct or_scene {
  const nr_material_desc* materials; /* [0] is the default purple Lambertian */
  uint32_t n_materials;
  const nr_object_desc* objects; /* hittables then lights */
  uint32_t n_objects;
  const or_mesh* meshes;
  uint32_t n_meshes;
  int32_t sky_type;
  float sky_start[3], sky_end[3];
  const float* hdri; /* planar CHW float, C >= 3 */
  uint32_t hdri_C, hdri_H, hdri_W;
  float hdri_rotation, hdri_intensity;
  const char* hdri_path; /* Radiance file the HDRI was read from (reference harnesses load it) */
  const or_image* images; /* indexed by nr_texture_desc.image */
  uint32_t n_images;
} or_scene;

/* Output buffers: planar CHW float (3 x H x W) or NULL. primary: one uint32
 * per pixel, (object_id << 22) | (triangle_index + 1) or 0xffffffff.
 * mode 0: rows [row_begin, row_end) of sample `first` only, raw sample values.
 * mode 1: samples [first, first+count) folded into the running mean
 *         avg*(n-1)/n + s/n (data.cu:28-50); beauty64 (if not NULL) gets the
 *         FP64 sum of beauty.
 * draw_rtl: 1 if constructor arguments that each draw a random number are
 * evaluated right to left (g++), 0 for left to right. */
typedef struct or_request {
  uint32_t first, count;
  int32_t mode;
  int32_t draw_rtl;
  uint32_t row_begin, row_end;
  int32_t threads;
  float* beauty;
  float* diffuse;
  float* normal;
  uint32_t* primary;
  double* beauty64;
} or_request;

int oracle_render(const or_scene* s, const nr_camera_desc* cam, const nr_render_config* cfg,
                  const or_request* req);
/* the same with the scene built once: create, render any number of times, destroy */
void* oracle_scene_create(const or_scene* s, int32_t draw_rtl);
int oracle_scene_render(void* scene, const nr_camera_desc* cam, const nr_render_config* cfg,
                        const or_request* req);
void oracle_scene_destroy(void* scene);
/* viewport preview, picking ray and selection outline on a scene handle */
int oracle_scene_viewport(void* scene, const nr_camera_desc* cam, uint32_t seed,
                          int32_t show_axis_grid, float* beauty, float* diffuse, float* normal);
int oracle_scene_pick(void* scene, const nr_camera_desc* cam, uint32_t seed, float u, float v,
                      nr_pick_result* out);
int oracle_scene_selection_mask(void* scene, const nr_camera_desc* cam, uint32_t seed,
                                uint32_t object_id, int32_t radius, uint8_t* out);
int refcpu_scene_viewport(void* scene, const nr_camera_desc* cam, uint32_t seed,
                          int32_t show_axis_grid, float* beauty, float* diffuse, float* normal);
int refcpu_scene_pick(void* scene, const nr_camera_desc* cam, uint32_t seed, float u, float v,
                      nr_pick_result* out);
int refcpu_scene_selection_mask(void* scene, const nr_camera_desc* cam, uint32_t seed,
                                uint32_t object_id, int32_t radius, uint8_t* out);
/* Binary-tree SAH cost C = sum_inner A/A_root + sum_leaf A/A_root * N of the
 * reference builder (bvh.h:35-320) over triangle boxes of a mesh. */
double oracle_mesh_sah(const or_mesh* m, uint64_t* n_nodes);
/* n-rooks pattern (camera.h:45-61), 2*n floats. */
int oracle_n_rooks(uint32_t n, uint32_t seed, int32_t draw_rtl, float* out);
/* Generator draws: count uniform floats of (seed, subsequence) from draw 0. */
int oracle_uniforms(uint32_t seed, uint32_t subsequence, uint32_t count, float* out);

/* file readers restating the reference's loaders (OBJ: parse_obj_file,
 * mesh.h:39-141; HDR: load_image_float, texture.h:28-47) */
int oracle_load_obj(const char* path, float* positions, float* normals, float* tangents,
                    float* uvs, uint32_t* triangles, uint32_t* n_vertices, uint32_t* n_triangles,
                    uint32_t capacity_vertices, uint32_t capacity_triangles);
int oracle_load_hdr(const char* path, float* chw, uint32_t* C, uint32_t* H, uint32_t* W,
                    uint64_t capacity);

/* display transform of process_stream_kernel (data/src/stream.cu:146-159)
 * over hw pixels of a planar 3-channel float image */
int oracle_display(const float* chw, uint32_t hw, const nr_stream_config* cfg, uint8_t* out8,
                   float* outf);

/* same signatures in the reference builds */
int refcpu_render(const or_scene* s, const nr_camera_desc* cam, const nr_render_config* cfg,
                  const or_request* req);
void* refcpu_scene_create(const or_scene* s, int32_t draw_rtl);
int refcpu_scene_render(void* scene, const nr_camera_desc* cam, const nr_render_config* cfg,
                        const or_request* req);
void refcpu_scene_destroy(void* scene);
double refcpu_mesh_sah(const or_mesh* m, uint64_t* n_nodes);
int refcpu_n_rooks(uint32_t n, uint32_t seed, float* out);
int refcpu_uniforms(uint32_t seed, uint32_t subsequence, uint32_t count, float* out);
int refcpu_load_obj(const char* path, float* positions, float* normals, float* tangents,
                    float* uvs, uint32_t* triangles, uint32_t* n_vertices, uint32_t* n_triangles,
                    uint32_t capacity_vertices, uint32_t capacity_triangles);
int refcpu_load_hdr(const char* path, float* chw, uint32_t* C, uint32_t* H, uint32_t* W,
                    uint64_t capacity);

#ifdef __cplusplus
}
#endif
#endif
