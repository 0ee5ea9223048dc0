// Device build of the geometry grid (dsmc_geomgrid.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "dsmc_host.hpp"

namespace dsmcb {

// The device arrays the traversal kernels read (cudaMalloc'd; the caller
// frees them): per cell the has-geometry flag and the entry range, per entry
// the triangle record (3 float4) and the plane.
struct GeomDevice {
  uint32_t* flags = nullptr;
  uint2* se = nullptr;
  float4* tri = nullptr;
  float4* plane = nullptr;
};

// Bins the mesh (host arrays) into g's frame (bbox, cell and dim set, e.g. by
// geometry_grid_frame) on the device, fills `out`, and leaves the host copy
// of the grid (count, tri_ids, flags) in g.  Synchronous.
cudaError_t build_geometry_device(GeomGrid& g, const float* verts, uint32_t nverts, const uint32_t* tris,
                                  uint32_t ntris, const float* normals, GeomDevice& out);

// The entry ranges, triangle records and planes of a given binning (device
// arrays: start has cells + 1 exclusive offsets, ids the triangle of each
// entry; verts, tris and normals on the device); allocates out.se, out.tri
// and out.plane.
cudaError_t geometry_entries_device(const uint32_t* start, const uint32_t* ids, uint32_t cells,
                                    uint32_t entries, const float* verts, const uint32_t* tris,
                                    const float* normals, GeomDevice& out);

}  // namespace dsmcb
