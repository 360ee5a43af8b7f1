// scene_device.cuh — flat device scene layout.
//
// The reference builds each object, material and texture on the device with a
// <<<1,1>>> placement-new kernel and links them by pointers
// (nectar_render/csrc/core/src/cuda.cu:11-23, hittable.h:42-131,
// material.h:385-449); a hit costs pointer chases objects[i] -> Hittable ->
// d_mesh -> arrays. Here every record lives in one array per kind, uploaded
// once, and addressed by index:
//   objects[]   one 128-byte DevObject per hittable (transform + type + ids)
//   materials[] one DevMaterial per registry entry (id 0 = default purple)
//   meshes[]    one DevMesh per mesh: leaf-ordered triangle records, BVH
//               nodes, and indexed per-vertex shading attributes
//   tlas        the top-level BVH over object bounds
// BVH nodes are 16-byte aligned and read with 128-bit loads.
#pragma once
#include "vecmath.cuh"

namespace nr {

// Binary node with both child boxes (64 B, 4 x 16 B):
//   a = {c0.lo.x, c0.hi.x, c0.lo.y, c0.hi.y}
//   b = {c1.lo.x, c1.hi.x, c1.lo.y, c1.hi.y}
//   c = {c0.lo.z, c0.hi.z, c1.lo.z, c1.hi.z}
//   d = {c0 link, c1 link, c0 count, c1 count}
// link >= 0: inner node index; link < 0: leaf whose first primitive slot is ~link
// and whose primitive count is the count field.
struct alignas(16) Bvh2Node {
  float4 a, b, c;
  int4 d;
};

// Compressed 8-wide node (80 B, 5 x 16 B), the layout of Ylitie, Karras and
// Laine, "Efficient Incoherent Ray Traversal on GPUs Through Compressed Wide
// BVHs" (HPG 2017):
//   n0 = {origin.x, origin.y, origin.z, (ex | ey<<8 | ez<<16 | imask<<24)}
//   n1 = {child_base, prim_base, meta[0..3], meta[4..7]}
//   n2 = {qlo.x[0..3], qlo.x[4..7], qlo.y[0..3], qlo.y[4..7]}
//   n3 = {qlo.z[0..3], qlo.z[4..7], qhi.x[0..3], qhi.x[4..7]}
//   n4 = {qhi.y[0..3], qhi.y[4..7], qhi.z[0..3], qhi.z[4..7]}
// Child slot i covers origin + 2^(e-127) * [qlo, qhi]. meta: empty slot 0;
// inner child 0b00111000 | (24 + i) ... see bvh_build.cu for the encoding.
struct alignas(16) Bvh8Node {
  float4 n0;
  uint4 n1, n2, n3, n4;
};

// Triangle record in BVH leaf order (48 B): v0 and the two edges exactly as
// the reference's Moller-Trumbore forms them (mesh.h:344-345), plus the
// original triangle index for shading.
struct alignas(16) TriRecord {
  float4 v0;  // .w = original triangle index (bits)
  float4 e1;  // v1 - v0
  float4 e2;  // v2 - v0
};

// One face of the reference's Cube (shapes.h:192-223): rotation, its
// transpose and position; the scale is 1.
struct CubeFace {
  M3 R, invR;
  V3 pos;
};

struct DevTexture {
  int32_t type;  // 0 constant, 1 image
  float r, g, b;
  const uint8_t* data;  // planar CHW uint8
  uint32_t C, H, W;
  float scale;
};

struct DevMaterial {
  int32_t type;
  float ior;
  float brightness;
  float tint[3];
  DevTexture tex[5];
};

struct alignas(16) DevObject {
  M3 R;          // world <- object rotation
  M3 invR;       // transpose
  V3 pos;
  V3 scale;
  V3 inv_s;      // 1 / (scale + FMIN) computed as the reference does
  int32_t type;  // NR_HITTABLE_*
  int32_t wrapped_type;
  uint32_t material;
  uint32_t mesh;
  float radius;           // sphere radius + FMIN (shapes.h:9)
  float neg_inv_density;  // -1 / (density + FMIN) (volumes.h:7-8)
  uint32_t object_id;     // registry id (insertion order)
  uint32_t pad;
};

struct DevMesh {
  const TriRecord* tris2;   // leaf order of the 2-wide tree
  const TriRecord* tris8;   // leaf order of the 8-wide tree
  const Bvh2Node* bvh2;     // binary tree (inner nodes)
  const Bvh8Node* bvh8;     // compressed wide tree
  const uint32_t* tri_vidx; // 3 vertex indices per original triangle
  const float* vnormal;     // 3 floats per vertex
  const float* vtangent;    // 3 floats per vertex
  const float* vuv;         // 2 floats per vertex
  uint32_t n_tris;
  uint32_t n_bvh2;
  uint32_t n_bvh8;
  uint32_t pad;
};

struct DevSky {
  int32_t type;  // NR_SKY_*
  float start[3];
  float end[3];
  float rotation;
  float intensity;
  M3 rot;             // rotation_y(deg2rad(rotation)) built as the reference does
  const float* data;  // planar CHW float
  int32_t C, H, W;
  // importance sampling (perf mode): alias tables over rows and, per row,
  // over its columns; the probability of each texel
  const float* row_prob;       // H acceptance probabilities
  const uint32_t* row_alias;   // H alias rows
  const float* col_prob;       // H*W acceptance probabilities
  const uint32_t* col_alias;   // H*W alias columns
  const float* texel_pdf;      // H*W probability of each texel
  float total_weight;
};

struct DevScene {
  const DevObject* objects;  // in top-level leaf order
  uint32_t n_objects;
  const DevMaterial* materials;
  uint32_t n_materials;
  const DevMesh* meshes;
  uint32_t n_meshes;
  const Bvh2Node* tlas2;
  const Bvh8Node* tlas8;
  const uint32_t* tlas_prims;  // 2-wide top-level leaf slot -> object slot
  const uint32_t* tlas_prims8; // 8-wide top-level leaf slot -> object slot
  uint32_t n_tlas2;
  uint32_t n_tlas8;
  int32_t light;  // object slot of lights[0], -1 if the scene has no lights
  int32_t use_bvh8;
  const CubeFace* cube_faces;  // 6 faces
  DevSky sky;
  // Bounds of one traversal: steps per query and entries per traversal stack
  // (the smaller of this and the kernel's own stack). Exceeding either sets an
  // error bit (8: steps, 1: stack) that the host reports as NR_ERR_DEVICE.
  uint32_t max_steps;
  uint32_t stack_limit;
};

}  // namespace nr
