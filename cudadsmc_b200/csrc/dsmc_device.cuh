// Device arithmetic for the DSMC timestep.
//
// Every function that has a counterpart in the reference evaluates the same
// FP32 expressions in the same order (with the same promotions to double), so
// nvcc makes the same contraction choices and the results agree with the
// reference's own kernels.  Counterparts are cited as file:line of
// denglide/CudaDsmc.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace dsmcb {

constexpr float kPiF = 3.14159265358979f;      // DSMC_PI, include/dsmc.h:26
constexpr double kBounceDelta = 0.001;         // BOUNCE_DELTA, kernels/dsmc_kernel.cu:53
constexpr uint32_t kCollisionLimit = 10u;      // COLLISION_LIMIT, kernels/dsmc_kernel.cu:1250
constexpr float kPathEps = 0.0001f;            // EPS, kernels/dsmc_kernel.cu:1251
constexpr float kModelWidth = 0.0001f;         // MODEL_WIDTH, kernels/dsmc_kernel.cu:1253
constexpr double kTriEpsilon = 0.000001;       // EPSILON, kernels/tri_intersect.cu:1
constexpr uint32_t kNone = 0xffffffffu;
constexpr uint32_t kDeadKey = 0xffffffffu;     // key of a particle that left the domain
constexpr float kBoltzmann = 1.3806e-23f;      // DSMC_BOLZ, include/dsmc.h:33

// ------------------------------------------------------------------ RNG ----

// TausStep / LCGStep / HybridTausRng(Int), kernels/mtwister.cu:118-153.
__device__ __forceinline__ uint32_t taus_step(uint32_t& z, int s1, int s2, int s3, uint32_t m) {
  uint32_t b = ((z << s1) ^ z) >> s2;
  z = ((z & m) << s3) ^ b;
  return z;
}

__device__ __forceinline__ uint32_t hybrid_taus_int(uint4& s) {
  uint32_t a = taus_step(s.x, 13, 19, 12, 4294967294u);
  uint32_t b = taus_step(s.y, 2, 25, 4, 4294967288u);
  uint32_t c = taus_step(s.z, 3, 11, 17, 4294967280u);
  s.w = s.w * 1664525u + 1013904223u;
  return a ^ b ^ c ^ s.w;
}

__device__ __forceinline__ float hybrid_taus_float(uint4& s) {
  return (float)(2.3283064365387e-10 * (double)hybrid_taus_int(s));
}

// Philox-4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw, SC'11):
// ten rounds of two 32x32->64 multiplies mixed with the key, the key bumped by
// the Weyl increments between rounds.
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
    uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    k.x += 0x9E3779B9u;
    k.y += 0xBB67AE85u;
  }
  return c;
}

// One Philox block, out of line: the streams below refill from one copy of
// the ten rounds instead of an inlined copy at every draw site.
static __device__ __noinline__ uint4 philox_block(uint32_t b, uint32_t c1, uint32_t c2, uint32_t c3,
                                                  uint2 k) {
  return philox4x32_10(make_uint4(b, c1, c2, c3), k);
}

// A Philox stream: (key, counter words 1..3 fixed) and a running block index
// in word 0; hands out 32-bit words four at a time.  INLINE_REFILL expands
// the ten rounds at the draw site (the collision loops, where a call per
// refill costs more than the code size); elsewhere the refill is the
// out-of-line philox_block.  Both give the same words.
template <bool INLINE_REFILL>
struct PhiloxStreamT {
  uint2 key;
  uint32_t c1, c2, c3;
  uint32_t block;
  uint4 buf;
  int used;
  __device__ __forceinline__ void init(uint2 k, uint32_t a, uint32_t b, uint32_t c) {
    key = k; c1 = a; c2 = b; c3 = c; block = 0; used = 4;
  }
  __device__ __forceinline__ uint32_t next() {
    if (used == 4) {
      buf = INLINE_REFILL ? philox4x32_10(make_uint4(block, c1, c2, c3), key)
                          : philox_block(block, c1, c2, c3, key);
      block++;
      used = 0;
    }
    uint32_t r = used == 0 ? buf.x : used == 1 ? buf.y : used == 2 ? buf.z : buf.w;
    used++;
    return r;
  }
  // uniform in (0, 1): 24 random bits, offset by half an ulp of 2^-24
  __device__ __forceinline__ float uniform() {
    return ((float)(next() >> 8) + 0.5f) * (1.0f / 16777216.0f);
  }
};
using PhiloxStream = PhiloxStreamT<false>;
using PhiloxStreamInline = PhiloxStreamT<true>;

// ------------------------------------------------------------ geometry ----

// float -> uint as the reference's implicit conversions compile
// (cvt.rzi.u32.f32: truncation, saturation, NaN -> 0).
__device__ __forceinline__ uint32_t f2u(float f) { return (uint32_t)f; }

// Loads of the body's geometry (triangle grid, planes, vertices, clearance
// table) with the L2 eviction priority evict_last: these 10-20 MB are read
// by a few percent of the particles every step, after streaming kernels have
// passed several hundred MB through L2; with normal priority they were
// evicted every step and each dependent step of a traversal paid a DRAM
// round trip.
__device__ __forceinline__ uint64_t l2_keep() {
  uint64_t pol;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ float4 geo_ld(const float4* a) {
  float4 r;
  asm("ld.global.nc.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
      : "=f"(r.x), "=f"(r.y), "=f"(r.z), "=f"(r.w)
      : "l"(a), "l"(l2_keep()));
  return r;
}
__device__ __forceinline__ uint2 geo_ld(const uint2* a) {
  uint2 r;
  asm("ld.global.nc.L2::cache_hint.v2.u32 {%0, %1}, [%2], %3;" : "=r"(r.x), "=r"(r.y) : "l"(a), "l"(l2_keep()));
  return r;
}
__device__ __forceinline__ float2 geo_ld(const float2* a) {
  float2 r;
  asm("ld.global.nc.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;" : "=f"(r.x), "=f"(r.y) : "l"(a), "l"(l2_keep()));
  return r;
}
__device__ __forceinline__ float geo_ld(const float* a) {
  float r;
  asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(r) : "l"(a), "l"(l2_keep()));
  return r;
}
__device__ __forceinline__ uint32_t geo_ld(const uint32_t* a) {
  uint32_t r;
  asm("ld.global.nc.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(r) : "l"(a), "l"(l2_keep()));
  return r;
}
__device__ __forceinline__ void geo_prefetch(const void* a) {
  asm volatile("prefetch.global.L2::evict_last [%0];" ::"l"(a));
}

struct GridGeom {
  float3 gmin, gmax, cell;
  uint3 dim;
};

// GetCellID3D, kernels/dsmc_kernel.cu:1701-1710.
__device__ __forceinline__ uint32_t cell_id3d(const GridGeom& g, float px, float py, float pz) {
  uint32_t x = (px - g.gmin.x) / g.cell.x;
  uint32_t y = (py - g.gmin.y) / g.cell.y;
  uint32_t z = (pz - g.gmin.z) / g.cell.z;
  return min(z, g.dim.z - 1) * g.dim.x * g.dim.y + min(y, g.dim.y - 1) * g.dim.x +
         min(x, g.dim.x - 1);
}

// GetCollisionCellID(float4), kernels/dsmc_kernel.cu:180-204.
__device__ __forceinline__ uint32_t coll_cell_id(const GridGeom& g, float3 p) {
  if (p.x < g.gmin.x || p.y < g.gmin.y || p.z < g.gmin.z || p.x > g.gmax.x || p.y > g.gmax.y ||
      p.z > g.gmax.z)
    return kNone;
  uint32_t x = (p.x - g.gmin.x) / g.cell.x;
  uint32_t y = (p.y - g.gmin.y) / g.cell.y;
  uint32_t z = (p.z - g.gmin.z) / g.cell.z;
  x = min(x, g.dim.x - 1);
  y = min(y, g.dim.y - 1);
  z = min(z, g.dim.z - 1);
  return z * g.dim.x * g.dim.y + y * g.dim.x + x;
}

// normalize / length / distance4 / reflect4, kernels/vectors.cu:24-106.
__device__ __forceinline__ float3 normalize3(float3 v) {
  float l = sqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
  if (l > 0) return make_float3(v.x / l, v.y / l, v.z / l);
  return v;
}

__device__ __forceinline__ float length3(float3 vec) {
  return sqrtf(vec.x * vec.x + vec.y * vec.y + vec.z * vec.z);
}

__device__ __forceinline__ float distance3(float3 v1, float3 v2) {
  return sqrtf((v2.x - v1.x) * (v2.x - v1.x) + (v2.y - v1.y) * (v2.y - v1.y) +
               (v2.z - v1.z) * (v2.z - v1.z));
}

__device__ __forceinline__ float3 reflect3(float3 v, float3 n) {
  float dt = v.x * n.x + v.y * n.y + v.z * n.z;
  return make_float3(v.x - 2 * dt * n.x, v.y - 2 * dt * n.y, v.z - 2 * dt * n.z);
}

// Moller-Trumbore ray/triangle test, kernels/tri_intersect.cu:14-56.
__device__ __forceinline__ bool intersect_triangle(float3 orig, float3 dir, float3 vert0,
                                                   float3 vert1, float3 vert2, float* t, float* u,
                                                   float* v) {
  float3 edge1, edge2, tvec, pvec, qvec;
  edge1.x = vert1.x - vert0.x; edge1.y = vert1.y - vert0.y; edge1.z = vert1.z - vert0.z;
  edge2.x = vert2.x - vert0.x; edge2.y = vert2.y - vert0.y; edge2.z = vert2.z - vert0.z;
  pvec.x = dir.y * edge2.z - dir.z * edge2.y;
  pvec.y = dir.z * edge2.x - dir.x * edge2.z;
  pvec.z = dir.x * edge2.y - dir.y * edge2.x;
  float det = edge1.x * pvec.x + edge1.y * pvec.y + edge1.z * pvec.z;
  if (det > -kTriEpsilon && det < kTriEpsilon) return false;
  float inv_det = __frcp_rn(det);  // == (float)(1.0 / (double)det), correctly rounded
  tvec.x = orig.x - vert0.x; tvec.y = orig.y - vert0.y; tvec.z = orig.z - vert0.z;
  *u = (tvec.x * pvec.x + tvec.y * pvec.y + tvec.z * pvec.z) * inv_det;
  if (*u < 0.0f || *u > 1.0f) return false;
  qvec.x = tvec.y * edge1.z - tvec.z * edge1.y;
  qvec.y = tvec.z * edge1.x - tvec.x * edge1.z;
  qvec.z = tvec.x * edge1.y - tvec.y * edge1.x;
  *v = (dir.x * qvec.x + dir.y * qvec.y + dir.z * qvec.z) * inv_det;
  if (*v < 0.0f || *u + *v > 1.0f) return false;
  *t = (edge2.x * qvec.x + edge2.y * qvec.y + edge2.z * qvec.z) * inv_det;
  return true;
}

// Programmatic dependent launch.  The step's kernels are launched with
// programmatic stream serialization (launch_chained): a kernel's CTAs may be
// dispatched while the kernel before it in the stream drains, and each waits
// here, before its first access to memory, until that kernel has completed
// and its writes are visible (griddepcontrol.wait is a no-op for a kernel
// launched without the attribute).  It then allows the next kernel's launch
// to begin, which dispatches once every CTA of this one has started.  Every
// CTA of a chained kernel calls this first, whatever work it has: a kernel
// waits only for its direct predecessor, so the chain orders the whole step
// only if no kernel can complete before the one it follows.
__device__ __forceinline__ void chained_entry() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Geometry on the device: the uniform grid over the body, a per-cell flag,
// per-cell [start,end) into the bin entries, and per bin entry the three
// vertices with the face normal packed into the .w lanes.
struct GeomView {
  GridGeom grid;
  const uint32_t* flags;
  const uint2* start_end;  // bin entries of each cell; (kNone, kNone) when empty
  // kTriStride float4 per bin entry: (v0, n.x), (v1, n.y), (v2, n.z)
  const float4* tri;
  // per bin entry, the triangle's plane (unit normal, offset), packed apart
  // from the vertices so that a cell's planes share cache lines
  const float4* plane;
  // per bin entry, (r, k): a particle leaving the entry's triangle outward
  // (re-emitted or reflected from it) along a path shorter than r whose
  // direction makes more than k with the normal (the sine of its elevation)
  // crosses no listed triangle; r = 0 where that holds for no path; null:
  // no table
  const float2* reach;
  // per grid cell, a slab that holds every vertex of the cell's listed
  // triangles: (m, e) with |m . x - e| <= 1 on all of them (m the slab's
  // normal over its half thickness); a path that stays outside the slab
  // crosses none of the cell's triangles.  (0, 0, 0, 0) passes every path;
  // null: no slabs
  const float4* slab;
  // clearance table: per cell of cgrid (the triangle grid refined by a small
  // factor, same bounds), a lower bound of the distance from any point of the
  // cell to the surface
  GridGeom cgrid;
  const float* clear;
  int diffuse;        // 0: specular (reference); 1: diffuse at wall_temp
  float wall_vstd;    // sqrt(k T_wall / m)
  int nearest;        // 0: reference first-hit in start/end cells; 1: nearest hit along the path
};

constexpr int kTriStride = 3;

// Ray/triangle test with a determinant threshold relative to the triangle's
// size (the reference's absolute 1e-6 rejects near-grazing rays on small
// triangles).
// Rounding steps explicit (no contraction), the forms of dot_x/cross_x below.
__device__ __forceinline__ float dot_x(float3 a, float3 b) {
  return fmaf(a.z, b.z, fmaf(a.x, b.x, __fmul_rn(a.y, b.y)));
}
__device__ __forceinline__ float3 cross_x(float3 a, float3 b) {
  return make_float3(fmaf(a.y, b.z, -__fmul_rn(a.z, b.y)), fmaf(a.z, b.x, -__fmul_rn(a.x, b.z)),
                     fmaf(a.x, b.y, -__fmul_rn(a.y, b.x)));
}
__device__ __forceinline__ bool intersect_triangle_rel(float3 o, float3 d, float3 a, float3 b,
                                                       float3 c, float* t) {
  const float3 e1 = make_float3(b.x - a.x, b.y - a.y, b.z - a.z);
  const float3 e2 = make_float3(c.x - a.x, c.y - a.y, c.z - a.z);
  const float3 pv = cross_x(d, e2);
  const float det = dot_x(e1, pv);
  const float scale = dot_x(e1, e1) + dot_x(e2, e2);
  if (fabsf(det) <= __fmul_rn(1e-9f, scale)) return false;
  const float inv = 1.0f / det;
  const float3 tv = make_float3(o.x - a.x, o.y - a.y, o.z - a.z);
  const float u = __fmul_rn(dot_x(tv, pv), inv);
  if (u < 0.f || u > 1.f) return false;
  const float3 qv = cross_x(tv, e1);
  const float v = __fmul_rn(dot_x(d, qv), inv);
  if (v < 0.f || u + v > 1.f) return false;
  *t = __fmul_rn(dot_x(e2, qv), inv);
  return true;
}

// Nearest triangle crossed by the segment o + s d, s in [0, dist] (d unit),
// among the triangles of every geometry cell the segment passes through
// (Amanatides-Woo traversal of the uniform grid).  The walk keeps its state
// per axis in scalars (no arrays indexed at run time, which would live in
// local memory), and the next cell's triangle range is loaded while the
// current cell's triangles are tested, so each cell costs one round trip to
// memory for its planes (and one more for the vertices of the few triangles
// whose plane the segment crosses).
struct DdaAxis {
  int i, step, dim;
  float tmax, tdel;
};

__device__ __forceinline__ bool dda_axis_init(float o, float d, float lo, float hi, float cs, int dim,
                                              float& t0, float& t1, DdaAxis& a) {
  a.dim = dim;
  if (fabsf(d) < 1e-30f) {
    if (o < lo || o > hi) return false;
    a.step = 0;
    a.tmax = 3.0e38f;
    a.tdel = 3.0e38f;
    return true;
  }
  const float id = 1.f / d;
  float ta = (lo - o) * id, tb = (hi - o) * id;
  if (ta > tb) { const float s = ta; ta = tb; tb = s; }
  t0 = fmaxf(t0, ta);
  t1 = fminf(t1, tb);
  a.step = d > 0.f ? 1 : -1;
  a.tdel = fabsf(cs * id);
  return true;
}

__device__ __forceinline__ void dda_axis_start(float o, float d, float lo, float cs, float tstart, DdaAxis& a) {
  const float pp = o + d * tstart;
  const int i = (int)floorf((pp - lo) / cs);
  a.i = min(max(i, 0), a.dim - 1);
  if (a.step > 0) a.tmax = (lo + (a.i + 1) * cs - o) / d;
  else if (a.step < 0) a.tmax = (lo + a.i * cs - o) / d;
}

// The axis whose boundary the walk crosses next (0, 1, 2).
__device__ __forceinline__ int dda_next_axis(const DdaAxis& x, const DdaAxis& y, const DdaAxis& z) {
  return (x.tmax <= y.tmax && x.tmax <= z.tmax) ? 0 : (y.tmax <= z.tmax ? 1 : 2);
}

// The walk over the grid's cells along o + s d, s in [t0, t1] (the segment
// clipped to the grid's box): one axis state per dimension.
struct DdaWalk {
  DdaAxis X, Y, Z;
  float t1;
};

// Sets the walk up for the segment of length dist; false if it misses the grid.
__device__ __forceinline__ bool dda_begin(const GridGeom& g, float3 o, float3 d, float dist, DdaWalk& w) {
  float t0 = 0.f;
  w.t1 = dist;
  if (!dda_axis_init(o.x, d.x, g.gmin.x, g.gmax.x, g.cell.x, (int)g.dim.x, t0, w.t1, w.X)) return false;
  if (!dda_axis_init(o.y, d.y, g.gmin.y, g.gmax.y, g.cell.y, (int)g.dim.y, t0, w.t1, w.Y)) return false;
  if (!dda_axis_init(o.z, d.z, g.gmin.z, g.gmax.z, g.cell.z, (int)g.dim.z, t0, w.t1, w.Z)) return false;
  if (t0 > w.t1) return false;
  dda_axis_start(o.x, d.x, g.gmin.x, g.cell.x, t0, w.X);
  dda_axis_start(o.y, d.y, g.gmin.y, g.cell.y, t0, w.Y);
  dda_axis_start(o.z, d.z, g.gmin.z, g.cell.z, t0, w.Z);
  return true;
}

__device__ __forceinline__ uint32_t dda_cell(const GridGeom& g, int ix, int iy, int iz) {
  return ((uint32_t)iz * g.dim.y + (uint32_t)iy) * g.dim.x + (uint32_t)ix;
}

// The walk's next step: the current cell's exit distance, the axis crossed
// and the next cell; true if the walk goes on to it (still inside the path
// and the grid).
struct DdaNext {
  float texit;
  int ax, nx, ny, nz;
};
__device__ __forceinline__ bool dda_peek(const DdaWalk& w, DdaNext& n) {
  n.texit = fminf(w.X.tmax, fminf(w.Y.tmax, w.Z.tmax));
  n.ax = dda_next_axis(w.X, w.Y, w.Z);
  n.nx = w.X.i;
  n.ny = w.Y.i;
  n.nz = w.Z.i;
  if (n.ax == 0) n.nx += w.X.step; else if (n.ax == 1) n.ny += w.Y.step; else n.nz += w.Z.step;
  return n.texit <= w.t1 && n.nx >= 0 && n.nx < w.X.dim && n.ny >= 0 && n.ny < w.Y.dim && n.nz >= 0 &&
         n.nz < w.Z.dim;
}
__device__ __forceinline__ void dda_take(DdaWalk& w, const DdaNext& n) {
  if (n.ax == 0) { w.X.i = n.nx; w.X.tmax += w.X.tdel; }
  else if (n.ax == 1) { w.Y.i = n.ny; w.Y.tmax += w.Y.tdel; }
  else { w.Z.i = n.nz; w.Z.tmax += w.Z.tdel; }
}

// The walk's iteration limit for a grid.
__device__ __forceinline__ int dda_max_iter(const GridGeom& g) { return (int)(g.dim.x + g.dim.y + g.dim.z) + 3; }

// Slab pre-test of a grid cell (GeomView::slab) for the segment o + s d,
// s in [0, dist]: false when both ends lie beyond the same face of the slab.
// The margin covers the rounding of the two products, whose terms grow with
// the slab's inverse thickness.
__device__ __forceinline__ bool slab_may_cross(float4 S, float3 o, float3 d, float dist) {
  const float s0 = fmaf(S.z, o.z, fmaf(S.x, o.x, __fmul_rn(S.y, o.y))) - S.w;
  const float s1 = fmaf(dist, fmaf(S.z, d.z, fmaf(S.x, d.x, __fmul_rn(S.y, d.y))), s0);
  const float big = fabsf(S.x) + fabsf(S.y) + fabsf(S.z);
  const float tol = 1.f + fmaf(4e-7f * big, fabsf(o.x) + fabsf(o.y) + fabsf(o.z) + dist, 4e-7f * fabsf(S.w));
  return !((s0 > tol && s1 > tol) || (s0 < -tol && s1 < -tol));
}

// Plane pre-test of a triangle for the segment o + s d, s in [0, dist]: false
// when both ends lie on one side of its plane (beyond a rounding margin).
__device__ __forceinline__ bool plane_may_cross(float4 P, float3 o, float3 d, float dist) {
  const float3 pn = make_float3(P.x, P.y, P.z);
  const float s0 = dot_x(pn, o) - P.w;
  const float s1 = fmaf(dist, dot_x(pn, d), s0);
  const float tol = __fmul_rn(1e-7f, fabsf(P.w) + 1.f);
  return !((s0 > tol && s1 > tol) || (s0 < -tol && s1 < -tol));
}

// Whether the segment crosses bin entry i's triangle, at *t in [0, dist].
__device__ __forceinline__ bool entry_crossing(const GeomView& G, uint32_t i, float3 o, float3 d, float dist,
                                               float* t) {
  const float4 A = geo_ld(&G.tri[kTriStride * (size_t)i]);
  const float4 B = geo_ld(&G.tri[kTriStride * (size_t)i + 1]);
  const float4 C = geo_ld(&G.tri[kTriStride * (size_t)i + 2]);
  return intersect_triangle_rel(o, d, make_float3(A.x, A.y, A.z), make_float3(B.x, B.y, B.z),
                                make_float3(C.x, C.y, C.z), t) &&
         *t >= 0.f && *t <= dist;
}

__device__ __forceinline__ bool nearest_wall_hit(const GeomView& G, float3 o, float3 d, float dist,
                                                 float* t_out, uint32_t* entry_out) {
  DdaWalk w;
  if (!dda_begin(G.grid, o, d, dist, w)) return false;
  float best = 3.0e38f;
  uint32_t best_i = kNone;
  uint2 se = geo_ld(&G.start_end[dda_cell(G.grid, w.X.i, w.Y.i, w.Z.i)]);
  const int max_iter = dda_max_iter(G.grid);
  for (int it = 0; it < max_iter; it++) {
    // the walk's next cell, and its triangle range on the way
    DdaNext nx;
    const bool more = dda_peek(w, nx);
    uint2 se_next = make_uint2(0u, 0u);
    if (more) se_next = geo_ld(&G.start_end[dda_cell(G.grid, nx.nx, nx.ny, nx.nz)]);
    for (uint32_t i0 = se.x; i0 < se.y; i0 += 8) {
      // the planes of up to 8 of the cell's triangles in one round of loads
      float4 P[8];
#pragma unroll
      for (int k = 0; k < 8; k++)
        P[k] = i0 + k < se.y ? geo_ld(&G.plane[i0 + k]) : make_float4(0.f, 0.f, 0.f, 1.f);
      // the triangles whose plane the segment may cross are the candidates,
      // one bit each
      uint32_t cand = 0u;
#pragma unroll
      for (int k = 0; k < 8; k++) {
        if (i0 + k >= se.y) break;
        if (plane_may_cross(P[k], o, d, dist)) cand |= 1u << k;
      }
      // the candidates' vertices, in triangle order: the j-th round of the
      // loop loads every lane's j-th candidate at once, whatever its slot
      while (cand) {
        const uint32_t i = i0 + (uint32_t)(__ffs(cand) - 1);
        cand &= cand - 1u;
        float t;
        if (entry_crossing(G, i, o, d, dist, &t) && t < best) {
          best = t;
          best_i = i;
        }
      }
    }
    if (best <= nx.texit || !more) break;
    dda_take(w, nx);
    se = se_next;
  }
  if (best_i == kNone) return false;
  *t_out = best;
  *entry_out = best_i;
  return true;
}

// Whether o lies inside the closed mesh: parity of the triangles crossed by
// the ray from o along a fixed direction off every axis, up to the grid's
// boundary.  A crossing counts in the geometry cell whose stretch of the ray
// holds it, so a triangle binned in several cells counts once.
__device__ __forceinline__ bool inside_mesh(const GeomView& G, float3 o) {
  const GridGeom& g = G.grid;
  if (coll_cell_id(g, o) == kNone) return false;
  const float da[3] = {0.80178373f, 0.53452248f, 0.26726124f};  // (3, 2, 1) / sqrt(14)
  const float3 d = make_float3(da[0], da[1], da[2]);
  const float oa[3] = {o.x, o.y, o.z};
  const float lo[3] = {g.gmin.x, g.gmin.y, g.gmin.z};
  const float cs[3] = {g.cell.x, g.cell.y, g.cell.z};
  const int dm[3] = {(int)g.dim.x, (int)g.dim.y, (int)g.dim.z};
  int idx[3];
  float tmax[3], tdel[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const int i = (int)floorf((oa[a] - lo[a]) / cs[a]);
    idx[a] = min(max(i, 0), dm[a] - 1);
    tmax[a] = (lo[a] + (idx[a] + 1) * cs[a] - oa[a]) / da[a];
    tdel[a] = cs[a] / da[a];
  }
  float tcur = 0.f;
  uint32_t crossings = 0;
  const int max_iter = dm[0] + dm[1] + dm[2] + 3;
  for (int it = 0; it < max_iter; it++) {
    const uint32_t c = ((uint32_t)idx[2] * g.dim.y + (uint32_t)idx[1]) * g.dim.x + (uint32_t)idx[0];
    const float texit = fminf(tmax[0], fminf(tmax[1], tmax[2]));
    if (geo_ld(&G.flags[c]) != 0) {
      const uint2 se = geo_ld(&G.start_end[c]);
      for (uint32_t i = se.x; i < se.y; i++) {
        const float4 A = geo_ld(&G.tri[kTriStride * (size_t)i]);
        const float4 B = geo_ld(&G.tri[kTriStride * (size_t)i + 1]);
        const float4 C = geo_ld(&G.tri[kTriStride * (size_t)i + 2]);
        float t;
        if (intersect_triangle_rel(o, d, make_float3(A.x, A.y, A.z), make_float3(B.x, B.y, B.z),
                                   make_float3(C.x, C.y, C.z), &t) &&
            t > 0.f && t >= tcur && t < texit)
          crossings++;
      }
    }
    const int a = (tmax[0] <= tmax[1] && tmax[0] <= tmax[2]) ? 0 : (tmax[1] <= tmax[2] ? 1 : 2);
    idx[a] += 1;
    if (idx[a] >= dm[a]) break;
    tcur = texit;
    tmax[a] += tdel[a];
  }
  return (crossings & 1u) != 0;
}

// Diffuse re-emission about the unit normal n on the side the particle came
// from (full accommodation at the wall temperature): normal speed from the
// flux-weighted half-range Maxwellian, tangential components Gaussian.
// r1, r2, r3: uniforms in (0, 1).  Out of line (walls are the cold path).
// Rounding steps explicit (no contraction), so that a CPU restatement
// evaluates the same steps (only logf and sincosf may differ in the last bit).
static __device__ __noinline__ float3 diffuse_emit_r(float3 n_out, float vstd, float r1, float r2,
                                                     float r3) {
  const float vn = __fmul_rn(vstd, sqrtf(__fmul_rn(-2.0f, logf(r1))));
  const float rad = __fmul_rn(vstd, sqrtf(__fmul_rn(-2.0f, logf(r2))));
  float s, c;
  sincosf(__fmul_rn(6.2831853f, r3), &s, &c);
  const float t1 = __fmul_rn(rad, c), t2 = __fmul_rn(rad, s);
  // orthonormal tangent basis of n_out
  const float3 a = fabsf(n_out.x) < 0.9f ? make_float3(1.f, 0.f, 0.f) : make_float3(0.f, 1.f, 0.f);
  const float3 q = cross_x(a, n_out);
  const float ql = sqrtf(dot_x(q, q));
  const float3 e1 = ql > 0.f ? make_float3(q.x / ql, q.y / ql, q.z / ql) : q;
  const float3 e2 = cross_x(n_out, e1);
  return make_float3(fmaf(t2, e2.x, fmaf(t1, e1.x, __fmul_rn(vn, n_out.x))),
                     fmaf(t2, e2.y, fmaf(t1, e1.y, __fmul_rn(vn, n_out.y))),
                     fmaf(t2, e2.z, fmaf(t1, e1.z, __fmul_rn(vn, n_out.z))));
}
__device__ __forceinline__ float3 diffuse_emit(float3 n_out, float vstd, PhiloxStream& rng) {
  const float r1 = rng.uniform(), r2 = rng.uniform(), r3 = rng.uniform();
  return diffuse_emit_r(n_out, vstd, r1, r2, r3);
}

// CollideWithGeometry, kernels/dsmc_kernel.cu:1256-1314: the first triangle
// of the cell's list (in list order) that the path crosses reflects the
// particle; the remaining path continues from the hit point.
__device__ __forceinline__ bool collide_with_geometry(const GeomView& G, float3* pos, float3* vel,
                                                      float3* old_pos, uint32_t cellid,
                                                      PhiloxStream* rng) {
  uint2 idx_stend = geo_ld(&G.start_end[cellid]);
  float3 dir = normalize3(*vel);
  float t, u, v;
  float dist = distance3(*old_pos, *pos);
  if (dist < kPathEps) return false;
  for (uint32_t i = idx_stend.x; i < idx_stend.y; i++) {
    float4 a = geo_ld(&G.tri[kTriStride * (size_t)i]);
    float4 b = geo_ld(&G.tri[kTriStride * (size_t)i + 1]);
    float4 c = geo_ld(&G.tri[kTriStride * (size_t)i + 2]);
    float3 v1 = make_float3(a.x, a.y, a.z), v2 = make_float3(b.x, b.y, b.z),
           v3 = make_float3(c.x, c.y, c.z);
    if (intersect_triangle(*old_pos, dir, v1, v2, v3, &t, &u, &v)) {
      if (t >= 0 && t <= dist) {
        float uv = 1 - u - v;
        float3 norm = make_float3(a.w, b.w, c.w);
        float3 width = make_float3(norm.x * kModelWidth, norm.y * kModelWidth, norm.z * kModelWidth);
        float3 p;
        p.x = v1.x * uv + v2.x * u + v3.x * v;
        p.y = v1.y * uv + v2.y * u + v3.y * v;
        p.z = v1.z * uv + v2.z * u + v3.z * v;
        if (G.diffuse) {
          // re-emit on the side the particle arrived from; the rest of the
          // step's flight time continues at the new velocity
          float sp = length3(*vel);
          float side = (dir.x * norm.x + dir.y * norm.y + dir.z * norm.z) > 0.f ? -1.f : 1.f;
          float3 n_out = make_float3(side * norm.x, side * norm.y, side * norm.z);
          *vel = diffuse_emit(n_out, G.wall_vstd, *rng);
          width = make_float3(n_out.x * kModelWidth, n_out.y * kModelWidth, n_out.z * kModelWidth);
          float tau = (dist - t) / sp;
          pos->x = p.x + vel->x * tau;
          pos->y = p.y + vel->y * tau;
          pos->z = p.z + vel->z * tau;
        } else {
          *vel = reflect3(*vel, norm);
          float3 p1p = normalize3(*vel);
          float od = dist - t;
          pos->x = p.x + p1p.x * od;
          pos->y = p.y + p1p.y * od;
          pos->z = p.z + p1p.z * od;
        }
        old_pos->x = p.x + width.x;
        old_pos->y = p.y + width.y;
        old_pos->z = p.z + width.z;
        return true;
      }
    }
  }
  return false;
}

}  // namespace dsmcb
