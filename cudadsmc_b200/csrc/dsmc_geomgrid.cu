// Geometry grid of a mesh, built on the device: the binning of
// Model::CreateGrid and reg_grid_t::encloseGrid (src/model.cpp:733-769,
// src/reggrid.cpp:27-93), then the per-entry records the traversal kernels
// read.
//
// k_bin_tris: a warp per triangle walks the cells its bounding box touches
// (plus one cell of margin, as the reference does) and runs the
// separating-axis overlap test (Akenine-Moller 2001) on each.  The count pass
// adds to the per-cell counts (and the per scan tile totals the scan kernel
// needs); the fill pass writes the triangle id at a ticket of the cell's
// range.  k_bin_order then restores triangle order inside each cell, the
// order the reference's cell-major loop produces, and k_enclose flags the
// cells between flagged cells along z (src/reggrid.cpp:49-79).  k_entries
// writes per entry the triangle's vertices with its face normal packed into
// .w, and its plane (unit normal and offset, evaluated in FP64).
//
// The arithmetic is that of the host build (dsmc_host.cpp:
// build_geometry_grid, tri_box_overlap, compiled without contraction) with
// each rounding step explicit, so that both builds bin every triangle into
// the same cells.
#include <vector>

#include "dsmc_device.cuh"
#include "dsmc_geomgrid.hpp"
#include "dsmc_kernels.cuh"

namespace dsmcb {
namespace {

struct BinFrame {
  float mn[3], cell[3];
  uint32_t dim[3];
};

__device__ __forceinline__ float dot3_rn(const float a[3], const float v[3]) {
  return __fadd_rn(__fadd_rn(__fmul_rn(a[0], v[0]), __fmul_rn(a[1], v[1])), __fmul_rn(a[2], v[2]));
}
// std::min(std::min(a, b), c) and std::max(std::max(a, b), c)
__device__ __forceinline__ float min3f(float a, float b, float c) {
  const float m = b < a ? b : a;
  return c < m ? c : m;
}
__device__ __forceinline__ float max3f(float a, float b, float c) {
  const float m = a < b ? b : a;
  return m < c ? c : m;
}

// Separating-axis triangle/box test: disjoint iff the projections are
// disjoint on one of 13 axes (3 box normals, the triangle normal, 9 edge x
// box-normal crosses).  The host build's steps, each rounding explicit.
__device__ bool tri_box_overlap_dev(const float center[3], const float half[3], const float tri[9]) {
  float v[3][3];
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int k = 0; k < 3; k++) v[i][k] = __fsub_rn(tri[3 * i + k], center[k]);
  float e[3][3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    e[0][k] = __fsub_rn(v[1][k], v[0][k]);
    e[1][k] = __fsub_rn(v[2][k], v[1][k]);
    e[2][k] = __fsub_rn(v[0][k], v[2][k]);
  }
#pragma unroll
  for (int i = 0; i < 3; i++) {
#pragma unroll
    for (int j = 0; j < 3; j++) {
      float a[3] = {0.f, 0.f, 0.f};
      if (j == 0) { a[1] = -e[i][2]; a[2] = e[i][1]; }
      if (j == 1) { a[0] = e[i][2]; a[2] = -e[i][0]; }
      if (j == 2) { a[0] = -e[i][1]; a[1] = e[i][0]; }
      const float p0 = dot3_rn(a, v[0]), p1 = dot3_rn(a, v[1]), p2 = dot3_rn(a, v[2]);
      const float mn = min3f(p0, p1, p2), mx = max3f(p0, p1, p2);
      const float aa[3] = {fabsf(a[0]), fabsf(a[1]), fabsf(a[2])};
      const float r = dot3_rn(half, aa);
      if (mn > r || mx < -r) return false;
    }
  }
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const float mn = min3f(v[0][k], v[1][k], v[2][k]), mx = max3f(v[0][k], v[1][k], v[2][k]);
    if (mn > half[k] || mx < -half[k]) return false;
  }
  const float n[3] = {__fsub_rn(__fmul_rn(e[0][1], e[1][2]), __fmul_rn(e[0][2], e[1][1])),
                      __fsub_rn(__fmul_rn(e[0][2], e[1][0]), __fmul_rn(e[0][0], e[1][2])),
                      __fsub_rn(__fmul_rn(e[0][0], e[1][1]), __fmul_rn(e[0][1], e[1][0]))};
  const float d = dot3_rn(n, v[0]);
  const float an[3] = {fabsf(n[0]), fabsf(n[1]), fabsf(n[2])};
  const float r = dot3_rn(half, an);
  return !(d > r || d < -r);
}

// A warp per triangle over the cells [lo, hi] its bounding box touches (one
// cell of margin).  FILL false: counts, tile totals and flags; FILL true: the
// triangle's id at a ticket of each overlapped cell's range.
template <bool FILL>
__global__ void __launch_bounds__(256) k_bin_tris(BinFrame F, const float* verts, const uint32_t* tris,
                                                  uint32_t ntris, uint32_t* count, uint32_t* tile_sum,
                                                  uint32_t* flags, const uint32_t* start,
                                                  uint32_t* cursor, uint32_t* ids) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (t >= ntris) return;
  float tri[9];
#pragma unroll
  for (int q = 0; q < 3; q++)
#pragma unroll
    for (int k = 0; k < 3; k++) tri[3 * q + k] = verts[3 * (size_t)tris[3 * (size_t)t + q] + k];
  int lo[3], hi[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const float tmn = min3f(tri[k], tri[3 + k], tri[6 + k]);
    const float tmx = max3f(tri[k], tri[3 + k], tri[6 + k]);
    const float qa = floorf(__fdiv_rn(__fsub_rn(tmn, F.mn[k]), F.cell[k])) - 1.f;
    const float qb = floorf(__fdiv_rn(__fsub_rn(tmx, F.mn[k]), F.cell[k])) + 1.f;
    lo[k] = (int)fmax(0.0, (double)qa);
    hi[k] = (int)fmin((double)F.dim[k] - 1.0, (double)qb);
  }
  if (hi[0] < lo[0] || hi[1] < lo[1] || hi[2] < lo[2]) return;
  const uint32_t nx = (uint32_t)(hi[0] - lo[0] + 1), ny = (uint32_t)(hi[1] - lo[1] + 1);
  const uint64_t ncand = (uint64_t)nx * ny * (uint32_t)(hi[2] - lo[2] + 1);
  for (uint64_t k = lane; k < ncand; k += 32) {
    const uint32_t x = (uint32_t)lo[0] + (uint32_t)(k % nx);
    const uint32_t y = (uint32_t)lo[1] + (uint32_t)((k / nx) % ny);
    const uint32_t z = (uint32_t)lo[2] + (uint32_t)(k / ((uint64_t)nx * ny));
    const uint32_t xyz[3] = {x, y, z};
    float center[3], half[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const float bmin = __fadd_rn(F.mn[a], __fmul_rn((float)xyz[a], F.cell[a]));
      const float bmax = __fadd_rn(bmin, F.cell[a]);
      half[a] = __fdiv_rn(__fsub_rn(bmax, bmin), 2.f);
      center[a] = __fadd_rn(bmin, half[a]);
    }
    if (!tri_box_overlap_dev(center, half, tri)) continue;
    const uint32_t c = F.dim[0] * F.dim[1] * z + F.dim[0] * y + x;
    if (!FILL) {
      atomicAdd(&count[c], 1u);
      atomicAdd(&tile_sum[c >> kScanShift], 1u);
      flags[c] = 1u;
    } else {
      ids[start[c] + atomicAdd(&cursor[c], 1u)] = t;
    }
  }
}

// Triangle order inside each cell (the fill's tickets come in any order);
// cells hold few entries, so an insertion sort per thread.
__global__ void __launch_bounds__(256) k_bin_order(const uint32_t* start, uint32_t* ids, uint32_t cells) {
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < cells; c += gridDim.x * blockDim.x) {
    const uint32_t s = start[c], e = start[c + 1];
    for (uint32_t i = s + 1; i < e; i++) {
      const uint32_t v = ids[i];
      uint32_t j = i;
      while (j > s && ids[j - 1] > v) {
        ids[j] = ids[j - 1];
        j--;
      }
      ids[j] = v;
    }
  }
}

// Along z, the cells between a flagged cell and the next flagged cell become
// flagged, pairwise from the bottom (src/reggrid.cpp:49-79); a thread per
// (x, y) column.
__global__ void __launch_bounds__(256) k_enclose(uint32_t* flags, uint32_t dx, uint32_t dy, uint32_t dz) {
  for (uint32_t col = blockIdx.x * blockDim.x + threadIdx.x; col < dx * dy; col += gridDim.x * blockDim.x) {
    const uint32_t x = col % dx, y = col / dx;
    bool last_full = false;
    uint32_t last_z = 0;
    for (uint32_t z = 0; z < dz; z++) {
      if (flags[dx * dy * z + dx * y + x]) {
        if (!last_full) {
          last_z = z;
          last_full = true;
        } else {
          for (; last_z != z; last_z++) flags[dx * dy * last_z + dx * y + x] = 1u;
          last_full = false;
        }
      }
    }
  }
}

// Per cell its entry range, (kNone, kNone) when empty.
__global__ void __launch_bounds__(256) k_cell_ranges(const uint32_t* start, uint2* se, uint32_t cells) {
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < cells; c += gridDim.x * blockDim.x) {
    const uint32_t s = start[c], e = start[c + 1];
    se[c] = e > s ? make_uint2(s, e) : make_uint2(kNone, kNone);
  }
}

// Per entry: the triangle's vertices with its face normal in .w, and its
// plane from the vertices in FP64 (unit normal n, offset n . a), rounded to
// FP32 at the end.
__global__ void __launch_bounds__(256) k_entries(const uint32_t* ids, uint32_t n, const float* verts,
                                                 const uint32_t* tris, const float* normals, float4* tri,
                                                 float4* plane) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t t = ids[i];
    const float* a = verts + 3 * (size_t)tris[3 * (size_t)t];
    const float* b = verts + 3 * (size_t)tris[3 * (size_t)t + 1];
    const float* c = verts + 3 * (size_t)tris[3 * (size_t)t + 2];
    const float* nn = normals + 3 * (size_t)t;
    tri[kTriStride * (size_t)i] = make_float4(a[0], a[1], a[2], nn[0]);
    tri[kTriStride * (size_t)i + 1] = make_float4(b[0], b[1], b[2], nn[1]);
    tri[kTriStride * (size_t)i + 2] = make_float4(c[0], c[1], c[2], nn[2]);
    const double e1[3] = {__dsub_rn(b[0], a[0]), __dsub_rn(b[1], a[1]), __dsub_rn(b[2], a[2])};
    const double e2[3] = {__dsub_rn(c[0], a[0]), __dsub_rn(c[1], a[1]), __dsub_rn(c[2], a[2])};
    double pn[3] = {__dsub_rn(__dmul_rn(e1[1], e2[2]), __dmul_rn(e1[2], e2[1])),
                    __dsub_rn(__dmul_rn(e1[2], e2[0]), __dmul_rn(e1[0], e2[2])),
                    __dsub_rn(__dmul_rn(e1[0], e2[1]), __dmul_rn(e1[1], e2[0]))};
    const double l = __dsqrt_rn(
        __dadd_rn(__dadd_rn(__dmul_rn(pn[0], pn[0]), __dmul_rn(pn[1], pn[1])), __dmul_rn(pn[2], pn[2])));
    if (l > 0) {
      pn[0] = __ddiv_rn(pn[0], l);
      pn[1] = __ddiv_rn(pn[1], l);
      pn[2] = __ddiv_rn(pn[2], l);
    }
    const double w =
        __dadd_rn(__dadd_rn(__dmul_rn(pn[0], a[0]), __dmul_rn(pn[1], a[1])), __dmul_rn(pn[2], a[2]));
    plane[i] = make_float4(__double2float_rn(pn[0]), __double2float_rn(pn[1]), __double2float_rn(pn[2]),
                           __double2float_rn(w));
  }
}

uint32_t blocks_for(uint64_t threads) {
  const uint64_t b = (threads + 255) / 256;
  const uint64_t cap = (uint64_t)num_sms() * 32;
  return (uint32_t)(b == 0 ? 1 : (b < cap ? b : cap));
}

template <class T>
cudaError_t alloc_n(T** p, size_t n) {
  return cudaMalloc(reinterpret_cast<void**>(p), (n ? n : 1) * sizeof(T));
}

// Device copies that free themselves.
struct DevBufs {
  std::vector<void*> ptrs;
  template <class T>
  cudaError_t get(T** p, size_t n) {
    const cudaError_t e = alloc_n(p, n);
    if (e == cudaSuccess) ptrs.push_back(*p);
    return e;
  }
  template <class T>
  cudaError_t put(T** p, const T* host, size_t n) {
    cudaError_t e = get(p, n);
    if (e == cudaSuccess && n) e = cudaMemcpy(*p, host, n * sizeof(T), cudaMemcpyHostToDevice);
    return e;
  }
  ~DevBufs() {
    for (void* p : ptrs) cudaFree(p);
  }
};

}  // namespace

cudaError_t geometry_entries_device(const uint32_t* start, const uint32_t* ids, uint32_t cells,
                                    uint32_t entries, const float* verts, const uint32_t* tris,
                                    const float* normals, GeomDevice& out) {
  cudaError_t e = alloc_n(&out.se, cells);
  if (!e) e = alloc_n(&out.tri, kTriStride * ((size_t)entries + 1));
  if (!e) e = alloc_n(&out.plane, (size_t)entries + 1);
  if (e) return e;
  k_cell_ranges<<<blocks_for(cells), 256>>>(start, out.se, cells);
  if (entries) k_entries<<<blocks_for(entries), 256>>>(ids, entries, verts, tris, normals, out.tri, out.plane);
  return cudaGetLastError();
}

cudaError_t build_geometry_device(GeomGrid& g, const float* verts, uint32_t nverts, const uint32_t* tris,
                                  uint32_t ntris, const float* normals, GeomDevice& out) {
  const uint32_t dx = g.dim[0], dy = g.dim[1], dz = g.dim[2];
  const uint32_t cells = dx * dy * dz;
  const uint32_t n_tiles = (cells + kScanTile - 1) / kScanTile;
  BinFrame F;
  for (int k = 0; k < 3; k++) {
    F.mn[k] = g.bbox[k];
    F.cell[k] = g.cell[k];
    F.dim[k] = g.dim[k];
  }
  DevBufs tmp;
  float *d_verts = nullptr, *d_normals = nullptr;
  uint32_t *d_tris = nullptr, *count = nullptr, *cursor = nullptr, *start = nullptr, *tile_sum = nullptr;
  uint32_t* ids = nullptr;
  Meta* meta = nullptr;
  cudaError_t e = tmp.put(&d_verts, verts, 3 * (size_t)nverts);
  if (!e) e = tmp.put(&d_tris, tris, 3 * (size_t)ntris);
  if (!e) e = tmp.put(&d_normals, normals, 3 * (size_t)ntris);
  if (!e) e = tmp.get(&count, cells);
  if (!e) e = tmp.get(&cursor, cells);
  if (!e) e = tmp.get(&start, (size_t)cells + 1);
  if (!e) e = tmp.get(&tile_sum, n_tiles);
  if (!e) e = tmp.get(&meta, 1);
  if (!e) e = alloc_n(&out.flags, cells);
  if (e) return e;
  if (!e) e = cudaMemset(count, 0, cells * sizeof(uint32_t));
  if (!e) e = cudaMemset(tile_sum, 0, n_tiles * sizeof(uint32_t));
  if (!e) e = cudaMemset(out.flags, 0, cells * sizeof(uint32_t));
  if (!e) e = cudaMemset(meta, 0, sizeof(Meta));
  if (e) return e;
  const uint32_t bin_blocks = (uint32_t)(((uint64_t)ntris * 32 + 255) / 256);
  if (ntris) {
    k_bin_tris<false><<<bin_blocks, 256>>>(F, d_verts, d_tris, ntris, count, tile_sum, out.flags, nullptr,
                                           nullptr, nullptr);
  }
  // exclusive scan of the counts (the scan kernel resets counts and cursors)
  e = launch_scan(count, cursor, start, cells, tile_sum, n_tiles, meta, 0, nullptr);
  uint32_t entries = 0;
  if (!e) e = cudaMemcpy(&entries, start + cells, 4, cudaMemcpyDeviceToHost);
  if (!e) e = tmp.get(&ids, (size_t)entries);
  if (e) return e;
  if (ntris && entries) {
    k_bin_tris<true><<<bin_blocks, 256>>>(F, d_verts, d_tris, ntris, nullptr, nullptr, nullptr, start, cursor,
                                          ids);
    k_bin_order<<<blocks_for(cells), 256>>>(start, ids, cells);
  }
  k_enclose<<<blocks_for((uint64_t)dx * dy), 256>>>(out.flags, dx, dy, dz);
  e = cudaGetLastError();
  if (!e) e = geometry_entries_device(start, ids, cells, entries, d_verts, d_tris, d_normals, out);
  // the host copy (the fill's cell test and the clearance's distances read it)
  std::vector<uint32_t> st((size_t)cells + 1), fl(cells);
  g.tri_ids.resize(entries);
  if (!e) e = cudaMemcpy(st.data(), start, st.size() * 4, cudaMemcpyDeviceToHost);
  if (!e && entries) e = cudaMemcpy(g.tri_ids.data(), ids, (size_t)entries * 4, cudaMemcpyDeviceToHost);
  if (!e) e = cudaMemcpy(fl.data(), out.flags, (size_t)cells * 4, cudaMemcpyDeviceToHost);
  if (e) return e;
  g.count.resize(cells);
  g.flags.resize(cells);
  for (uint32_t c = 0; c < cells; c++) {
    g.count[c] = st[c + 1] - st[c];
    g.flags[c] = (uint8_t)(fl[c] != 0);
  }
  return cudaSuccess;
}

}  // namespace dsmcb
