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

bool load_obj(const std::string& path, HostMesh& out, std::string& err);
bool load_hdr(const std::string& path, HostImageF& out, std::string& err);

}  // namespace nr
