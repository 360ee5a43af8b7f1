// mesh_ingest.cuh — OBJ vertex assembly on the GPU: deduplication of the
// corners' (v, vt, vn) triples in order of first use, missing normals and
// per-vertex tangents, with the same result as the host assemble_obj.
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "host_io.h"

namespace nr {

// Assembles `raw` on the current device (temporary device buffers, freed
// before returning) and copies the mesh to `out`. Empty string on success.
std::string assemble_obj_device(const ObjRaw& raw, HostMesh& out, cudaStream_t st);

}  // namespace nr
