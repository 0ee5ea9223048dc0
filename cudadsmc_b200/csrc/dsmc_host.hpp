// Host-side helpers of the C ABI (no GPU needed).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "dsmc_b200.h"

namespace dsmcb {

// Uniform geometry grid over a mesh (reg_grid_t, include/reggrid.h:32-56).
struct GeomGrid {
  float bbox[6];
  float cell[3];
  uint32_t dim[3];
  std::vector<uint32_t> count;    // triangles per cell
  std::vector<uint32_t> tri_ids;  // triangle ids, cell-major, triangle order within a cell
  std::vector<uint8_t> flags;     // has geometry (after the enclose fill)
};

extern std::string g_config_error;

int config_default(dsmc_config* c);
int config_read_xml(const char* path, dsmc_config* c);
int config_from_args(int argc, const char* const* argv, dsmc_config* c, float* run_for);

int read_raw_mesh(const char* path, std::vector<float>& verts, std::vector<uint32_t>& tris,
                  std::vector<float>& fnorm);
void face_normals(const std::vector<float>& v, const std::vector<uint32_t>& t, std::vector<float>& n);
void mesh_icosphere(int level, float radius, const float* center, std::vector<float>& verts,
                    std::vector<uint32_t>& tris);
void mesh_capsule(float rn, float theta_deg, float length, const float* c, uint32_t ntarget,
                  uint64_t seed, std::vector<float>& verts, std::vector<uint32_t>& tris);
bool tri_box_overlap(const float center[3], const float half[3], const float tri[9]);
// The grid's frame: dim, the mesh's bounding box and the cell size.
void geometry_grid_frame(const float* verts, uint32_t nverts, const int dim[3], GeomGrid& out);
void build_geometry_grid(const float* verts, uint32_t nverts, const uint32_t* tris, uint32_t ntris,
                         const int dim[3], GeomGrid& out);

}  // namespace dsmcb
