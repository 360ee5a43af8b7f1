// host_io.h — OBJ and Radiance .hdr readers.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace nr {

struct HostMesh {
  std::vector<float> positions;  // 3 per vertex
  std::vector<float> normals;    // 3 per vertex
  std::vector<float> tangents;   // 3 per vertex
  std::vector<float> uvs;        // 2 per vertex
  std::vector<uint32_t> triangles;  // 3 per triangle
};

struct HostImageF {
  uint32_t C = 0, H = 0, W = 0;
  std::vector<float> chw;
};

// An OBJ file as parsed, before its vertices are assembled: the v / vn / vt
// arrays (3, 3 and 2 floats per entry) and every triangle corner as the
// index triple (v, vt, vn), 0-based, -1 when absent (polygons already
// triangulated).
struct ObjRaw {
  std::vector<float> vpos, vnor, vtex;
  std::vector<int32_t> corners;
};

bool parse_obj(const std::string& path, ObjRaw& raw, std::string& err);
// Deduplicates the corners into vertices, generates missing normals and the
// tangents (host; mesh_ingest.cu does the same on the GPU).
void assemble_obj(const ObjRaw& raw, HostMesh& out);
bool load_obj(const std::string& path, HostMesh& out, std::string& err);
bool load_hdr(const std::string& path, HostImageF& out, std::string& err);

}  // namespace nr
