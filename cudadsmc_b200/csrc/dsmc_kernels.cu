// Kernels of the DSMC timestep (sm_100a).
//
// Memory plan per particle and step (SoA FP32 state, 24 B):
//   scatter: read (key,ticket) 8 B + state 24 B, write state 24 B + orig 4 B
//   cell:    read state 24 B + orig 4 B, write state 24 B + (key,ticket) 8 B
// Per-cell arrays (counts, starts, (sigma*g)max/remainder, RNG state) add a
// few bytes per particle.  All particle traffic is coalesced except the
// scatter's writes, which land near-sorted because most particles stay in or
// next to their cell between steps.
#include "dsmc_kernels.cuh"

namespace dsmcb {

namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

// Ticket from a per-key counter, aggregated over the lanes of `mask` holding
// the same key: one atomic per distinct key per warp.  Also counts the key's
// scan tile in the block's shared histogram.
__device__ __forceinline__ uint32_t warp_ticket(uint32_t* count, uint32_t key, unsigned mask,
                                                uint32_t* s_tile) {
  unsigned peers = __match_any_sync(mask, key);
  int leader = __ffs(peers) - 1;
  unsigned lane = lane_id();
  uint32_t rank = __popc(peers & ((1u << lane) - 1u));
  uint32_t base = 0;
  if ((int)lane == leader) {
    uint32_t cnt = __popc(peers);
    base = atomicAdd(&count[key], cnt);
    atomicAdd(&s_tile[key >> kScanShift], cnt);
  }
  base = __shfl_sync(mask, base, leader);
  return base + rank;
}

__device__ __forceinline__ void flush_tile_hist(uint32_t* s_tile, uint32_t* tile_sum, uint32_t n) {
  for (uint32_t t = threadIdx.x; t < n; t += blockDim.x) {
    uint32_t v = s_tile[t];
    if (v) atomicAdd(&tile_sum[t], v);
  }
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}
__device__ __forceinline__ double warp_sum_f64(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}
__device__ __forceinline__ uint32_t warp_sum_u32(uint32_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

// ------------------------------------------------------------ RNG views ----

struct TausRng {
  uint4 s;
  __device__ __forceinline__ uint32_t u32() { return hybrid_taus_int(s); }
  __device__ __forceinline__ float f32() { return hybrid_taus_float(s); }
};
struct PhiloxRng {
  PhiloxStream s;
  __device__ __forceinline__ uint32_t u32() { return s.next(); }
  __device__ __forceinline__ float f32() { return s.uniform(); }
};

// Stream purposes in Philox counter word 3.
constexpr uint32_t kPurposeCollide = 0x636f6c6cu;
constexpr uint32_t kPurposeWall = 0x77616c6cu;
constexpr uint32_t kPurposeInit = 0x696e6974u;
constexpr uint32_t kPurposeInject = 0x696e6a65u;

// ------------------------------------------------------ velocity access ----

struct SmemVel {
  float* u; float* v; float* w;
  const uint16_t* slot;
  uint32_t off;
  __device__ __forceinline__ float3 get(uint32_t k) const {
    uint32_t j = slot[off + k];
    return make_float3(u[j], v[j], w[j]);
  }
  __device__ __forceinline__ void set(uint32_t k, float3 a) const {
    uint32_t j = slot[off + k];
    u[j] = a.x; v[j] = a.y; w[j] = a.z;
  }
};

struct GlobalVel {
  float* u; float* v; float* w;
  uint32_t off;
  __device__ __forceinline__ float3 get(uint32_t k) const {
    return make_float3(u[off + k], v[off + k], w[off + k]);
  }
  __device__ __forceinline__ void set(uint32_t k, float3 a) const {
    u[off + k] = a.x; v[off + k] = a.y; w[off + k] = a.z;
  }
};

// ------------------------------------------------------------- collide ----

// NTC collisions of one cell: ComputeBirdCollisionsNoMTDev,
// kernels/dsmc_kernel.cu:912-1000.  Particles of the cell are acc.get(0..n-1)
// in sorted order; pair members are start + rand % n as in the reference.
template <class Rng, class Acc>
__device__ __forceinline__ void ntc_cell(const StepParams& p, uint32_t cell, int partCount,
                                         Acc acc, Rng& rng, uint32_t& sel, uint32_t& col,
                                         double& sum_g) {
  float4 stat = make_float4(0.f, 0.f, 0.f, 0.f);
  if (p.stat4) stat = p.stat4[cell];
  float2 vmax = p.maxrem[cell];
  const float avgConc = p.ntc_local ? (float)(partCount - 1) : p.avg_conc;
  float fpc = (0.5 * partCount * avgConc * p.fnum * vmax.x * p.dt) / p.cell_volume + vmax.y;
  uint32_t pairsCount = fpc;
  stat.x += pairsCount;
  vmax.y = fpc - pairsCount;
  sel += pairsCount;
  for (uint32_t i = 0; i < pairsCount; i++) {
    uint32_t px = rng.u32() % (uint32_t)partCount;
    float3 v1 = acc.get(px);
    uint32_t py = rng.u32() % (uint32_t)partCount;
    float3 v2 = acc.get(py);
    float mag = length3(make_float3(v1.x - v2.x, v1.y - v2.y, v1.z - v2.z));
    float v;
    if (p.hard_sphere) {
      v = mag * p.cross_section;
    } else {
      v = mag > 0.f ? mag * (p.cross_section * powf(p.vhs_gref / mag, p.vhs_exp)) : 0.f;
    }
    if (v / vmax.x > rng.f32()) {
      stat.y++;
      stat.z += mag;
      col++;
      sum_g += mag;
      float b = 2.0f * rng.f32() - 1.0f;
      float a = sqrtf(1 - b * b);
      float c = 2 * kPiF * rng.f32();
      float3 angles = make_float3(b * mag / 2.0f, a * mag * __cosf(c) / 2.0f,
                                  a * mag * __sinf(c) / 2.0f);
      float3 v11, v22;
      v11.x = (v1.x + v2.x) / 2.0f + angles.x;
      v11.y = (v1.y + v2.y) / 2.0f + angles.y;
      v11.z = (v1.z + v2.z) / 2.0f + angles.z;
      acc.set(px, v11);
      v22.x = (v1.x + v2.x) / 2.0f - angles.x;
      v22.y = (v1.y + v2.y) / 2.0f - angles.y;
      v22.z = (v1.z + v2.z) / 2.0f - angles.z;
      acc.set(py, v22);
    }
    if (v > vmax.x) vmax.x = v;
  }
  p.maxrem[cell] = vmax;
  if (p.stat4) p.stat4[cell] = stat;
}

template <class Acc>
__device__ __forceinline__ void collide_cell(const StepParams& p, uint32_t cell, int partCount,
                                             Acc acc, uint32_t step, uint32_t& sel, uint32_t& col,
                                             double& sum_g) {
  if (partCount < 2) return;
  if (p.rng_kind == 0) {
    TausRng r;
    r.s = p.seeds[cell];
    ntc_cell(p, cell, partCount, acc, r, sel, col, sum_g);
    p.seeds[cell] = r.s;
  } else {
    PhiloxRng r;
    r.s.init(p.seed, cell, step, kPurposeCollide);
    ntc_cell(p, cell, partCount, acc, r, sel, col, sum_g);
  }
}

// ---------------------------------------------------------------- move ----

// The reference's four boundary functors, kernels/dsmc_kernel.cu:1316-1555,
// with their order of face checks and their double-precision wrap.
__device__ __forceinline__ void ref_bc(int periodic, const GridGeom& g, float3& pos, float3& vel) {
  switch (periodic) {
    case 'z':
      if (pos.z > g.gmax.z) pos.z = g.gmin.z + kBounceDelta + pos.z - g.gmax.z;
      if (pos.y > g.gmax.y) { pos.y = g.gmax.y - kBounceDelta; vel.y *= -1; }
      if (pos.z < g.gmin.z) pos.z = g.gmax.z - kBounceDelta + pos.z - g.gmin.z;
      if (pos.y < g.gmin.y) { pos.y = g.gmin.y + kBounceDelta; vel.y *= -1; }
      if (pos.x < g.gmin.x) { pos.x = g.gmin.x + kBounceDelta; vel.x *= -1; }
      if (pos.x > g.gmax.x) { pos.x = g.gmax.x - kBounceDelta; vel.x *= -1; }
      break;
    case 'x':
      if (pos.x > g.gmax.x) pos.x = g.gmin.x + kBounceDelta + pos.x - g.gmax.x;
      if (pos.y > g.gmax.y) { pos.y = g.gmax.y - kBounceDelta; vel.y *= -1; }
      if (pos.x < g.gmin.x) pos.x = g.gmax.x - kBounceDelta + pos.x - g.gmin.x;
      if (pos.y < g.gmin.y) { pos.y = g.gmin.y + kBounceDelta; vel.y *= -1; }
      if (pos.z < g.gmin.z) { pos.z = g.gmin.z + kBounceDelta; vel.z *= -1; }
      if (pos.z > g.gmax.z) { pos.z = g.gmax.z - kBounceDelta; vel.z *= -1; }
      break;
    case 'y':
      if (pos.y > g.gmax.y) pos.y = g.gmin.y + kBounceDelta + pos.y - g.gmax.y;
      if (pos.x > g.gmax.x) { pos.x = g.gmax.x - kBounceDelta; vel.x *= -1; }
      if (pos.y < g.gmin.y) pos.y = g.gmax.y - kBounceDelta + pos.y - g.gmin.y;
      if (pos.x < g.gmin.x) { pos.x = g.gmin.x + kBounceDelta; vel.x *= -1; }
      if (pos.z < g.gmin.z) { pos.z = g.gmin.z + kBounceDelta; vel.z *= -1; }
      if (pos.z > g.gmax.z) { pos.z = g.gmax.z - kBounceDelta; vel.z *= -1; }
      break;
    default:
      if (pos.y > g.gmax.y) { pos.y = g.gmax.y - kBounceDelta; vel.y *= -1; }
      if (pos.x > g.gmax.x) { pos.x = g.gmax.x - kBounceDelta; vel.x *= -1; }
      if (pos.y < g.gmin.y) { pos.y = g.gmin.y + kBounceDelta; vel.y *= -1; }
      if (pos.x < g.gmin.x) { pos.x = g.gmin.x + kBounceDelta; vel.x *= -1; }
      if (pos.z < g.gmin.z) { pos.z = g.gmin.z + kBounceDelta; vel.z *= -1; }
      if (pos.z > g.gmax.z) { pos.z = g.gmax.z - kBounceDelta; vel.z *= -1; }
      break;
  }
}

__device__ __forceinline__ float& comp(float3& a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }
__device__ __forceinline__ float compc(const float3& a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }

// Per-face domain boundaries (extension): specular and diffuse walls with the
// exact crossing point, outflow (particle removed), periodic wrap.  Returns
// false when the particle left the domain.
__device__ __forceinline__ bool face_bc(const StepParams& p, float3& pos, float3& vel,
                                        PhiloxStream& rng) {
  const GridGeom& g = p.grid;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    float lo = compc(g.gmin, a), hi = compc(g.gmax, a);
    float x = comp(pos, a);
    int face = -1;
    float bound = 0.f;
    if (x < lo) { face = 2 * a; bound = lo; }
    else if (x > hi) { face = 2 * a + 1; bound = hi; }
    if (face < 0) continue;
    int kind = p.face_kind[face];
    if (kind == 2 || kind == 4) return false;  // outflow / inflow face: leaves
    if (kind == 3) {
      comp(pos, a) = face & 1 ? x - (hi - lo) : x + (hi - lo);
      continue;
    }
    if (kind == 0) {
      comp(pos, a) = 2.f * bound - x;
      comp(vel, a) = -comp(vel, a);
      continue;
    }
    // diffuse wall: back to the crossing point, re-emit, fly the rest
    float va = comp(vel, a);
    float tau = va != 0.f ? (x - bound) / va : 0.f;
    pos.x -= vel.x * tau; pos.y -= vel.y * tau; pos.z -= vel.z * tau;
    comp(pos, a) = bound;
    float3 n_in = make_float3(0.f, 0.f, 0.f);
    comp(n_in, a) = face & 1 ? -1.f : 1.f;
    vel = diffuse_emit(n_in, p.face_vstd[face], rng);
    pos.x += vel.x * tau; pos.y += vel.y * tau; pos.z += vel.z * tau;
  }
  // a re-emitted particle that crossed another face in the rest of its flight
  // is clamped inside
  pos.x = fminf(fmaxf(pos.x, g.gmin.x), g.gmax.x);
  pos.y = fminf(fmaxf(pos.y, g.gmin.y), g.gmax.y);
  pos.z = fminf(fmaxf(pos.z, g.gmin.z), g.gmax.z);
  return true;
}

// One particle's flight: IntegrateDev / ProcessCollisionsDev,
// kernels/dsmc_kernel.cu:1557-1657.  Returns false if the particle left.
__device__ __forceinline__ bool move_particle(const StepParams& p, float3& pos, float3& vel,
                                              uint32_t gidx, uint32_t step) {
  float3 old_pos = pos;
  pos.x = old_pos.x + vel.x * p.dt;
  pos.y = old_pos.y + vel.y * p.dt;
  pos.z = old_pos.z + vel.z * p.dt;
  PhiloxStream rng;
  rng.init(p.seed, gidx, step, kPurposeWall);
  if (p.has_geom && p.geom.nearest) {
    // nearest wall crossing along the path, repeated for the rest of the
    // flight after each re-emission (extension for diffuse bodies)
    const GeomView& G = p.geom;
    for (uint32_t b = 0; b < kCollisionLimit; b++) {
      float3 seg = make_float3(pos.x - old_pos.x, pos.y - old_pos.y, pos.z - old_pos.z);
      float dist = length3(seg);
      if (!(dist > 1e-12f)) break;
      float3 d = make_float3(seg.x / dist, seg.y / dist, seg.z / dist);
      float t;
      uint32_t e;
      if (!nearest_wall_hit(G, old_pos, d, dist, &t, &e)) break;
      float3 n = make_float3(__ldg(&G.tri[3 * (size_t)e]).w, __ldg(&G.tri[3 * (size_t)e + 1]).w,
                             __ldg(&G.tri[3 * (size_t)e + 2]).w);
      float side = (d.x * n.x + d.y * n.y + d.z * n.z) > 0.f ? -1.f : 1.f;
      float3 n_out = make_float3(side * n.x, side * n.y, side * n.z);
      float3 hp = make_float3(old_pos.x + d.x * t + n_out.x * 1e-6f, old_pos.y + d.y * t + n_out.y * 1e-6f,
                              old_pos.z + d.z * t + n_out.z * 1e-6f);
      float rest = dist - t;
      if (G.diffuse) {
        float speed = length3(vel);
        vel = diffuse_emit(n_out, G.wall_vstd, rng);
        float tau = speed > 0.f ? rest / speed : 0.f;
        pos = make_float3(hp.x + vel.x * tau, hp.y + vel.y * tau, hp.z + vel.z * tau);
      } else {
        vel = reflect3(vel, n);
        float3 r = normalize3(vel);
        pos = make_float3(hp.x + r.x * rest, hp.y + r.y * rest, hp.z + r.z * rest);
      }
      old_pos = hp;
    }
  } else if (p.has_geom) {
    const GeomView& G = p.geom;
    uint32_t st_cubid = kNone, end_cubid = kNone;
    bool collProcessed = false;
    uint32_t i = 0;
    do {
      st_cubid = coll_cell_id(G.grid, old_pos);
      end_cubid = coll_cell_id(G.grid, pos);
      if (st_cubid != kNone) {
        if (__ldg(&G.flags[st_cubid]) != 0)
          collProcessed = collide_with_geometry(G, &pos, &vel, &old_pos, st_cubid, &rng);
      }
      if (!collProcessed && st_cubid != end_cubid && end_cubid != kNone) {
        if (__ldg(&G.flags[end_cubid]) != 0)
          collProcessed = collide_with_geometry(G, &pos, &vel, &old_pos, end_cubid, &rng);
      }
    } while (collProcessed && i++ < kCollisionLimit);
  }
  if (p.face_mode == 0) {
    ref_bc(p.periodic, p.grid, pos, vel);
    return true;
  }
  return face_bc(p, pos, vel, rng);
}

// ----------------------------------------------------------- cell kernel ----

struct CellSmem {
  uint32_t* ls;
  uint32_t* s_tile;
  float* x; float* y; float* z; float* u; float* v; float* w;
  uint32_t* orig;
  uint16_t* slot;
};

__device__ __forceinline__ CellSmem carve_smem(unsigned char* base) {
  CellSmem s;
  size_t off = 0;
  s.ls = (uint32_t*)(base + off); off += (kMaxCellsPerTile + 4) * 4;
  s.s_tile = (uint32_t*)(base + off); off += kMaxScanTiles * 4;
  s.x = (float*)(base + off); off += kTileCapacity * 4;
  s.y = (float*)(base + off); off += kTileCapacity * 4;
  s.z = (float*)(base + off); off += kTileCapacity * 4;
  s.u = (float*)(base + off); off += kTileCapacity * 4;
  s.v = (float*)(base + off); off += kTileCapacity * 4;
  s.w = (float*)(base + off); off += kTileCapacity * 4;
  s.orig = (uint32_t*)(base + off); off += kTileCapacity * 4;
  s.slot = (uint16_t*)(base + off); off += kTileCapacity * 2;
  return s;
}

constexpr int kCellSmemBytes =
    (kMaxCellsPerTile + 4) * 4 + kMaxScanTiles * 4 + kTileCapacity * (7 * 4 + 2);

// Sampling of one cell from sorted velocities (SampleCellStatisticsDev,
// kernels/dsmc_kernel.cu:856-890) into the FP64 accumulators.
template <class Acc>
__device__ __forceinline__ void sample_cell(double* acc, uint32_t cells, uint32_t cell, int n,
                                            const Acc& a) {
  if (n <= 0) return;
  double su = 0, sv = 0, sw = 0, se = 0;
  for (int k = 0; k < n; k++) {
    float3 q = a.get(k);
    double x = q.x, y = q.y, z = q.z;
    su += x; sv += y; sw += z;
    se += x * x + y * y + z * z;
  }
  acc[cell] += (double)n;
  acc[(size_t)cells + cell] += su;
  acc[2 * (size_t)cells + cell] += sv;
  acc[3 * (size_t)cells + cell] += sw;
  acc[4 * (size_t)cells + cell] += se;
}

// A cell too large for the shared-memory tile: processed by the whole block
// directly in the output arrays.
__device__ void giant_cell(const StepParams& p, uint32_t cell, uint32_t s, uint32_t e,
                           uint32_t step, bool do_sample, uint32_t* s_tile, uint32_t& sel,
                           uint32_t& col, double& sum_g, uint32_t& removed) {
  const uint32_t n = e - s;
  const bool vel_only = (p.flags & kVelOnly) != 0;
  if (threadIdx.x == 0 && p.meta) atomicAdd(&p.meta->giant_cells, 1u);
  // (key, orig) order: output slot s + rank of orig among the cell's entries
  if (p.flags & kDoFixup) {
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
      uint32_t my = p.in_orig[s + i];
      uint32_t rank = 0;
      for (uint32_t j = 0; j < n; j++) rank += p.in_orig[s + j] < my;
      uint32_t d = s + rank;
      if (!vel_only) {
        p.out.x[d] = p.in.x[s + i]; p.out.y[d] = p.in.y[s + i]; p.out.z[d] = p.in.z[s + i];
      }
      p.out.u[d] = p.in.u[s + i]; p.out.v[d] = p.in.v[s + i]; p.out.w[d] = p.in.w[s + i];
    }
  } else if (p.out.u != p.in.u) {
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
      if (!vel_only) {
        p.out.x[s + i] = p.in.x[s + i]; p.out.y[s + i] = p.in.y[s + i]; p.out.z[s + i] = p.in.z[s + i];
      }
      p.out.u[s + i] = p.in.u[s + i]; p.out.v[s + i] = p.in.v[s + i]; p.out.w[s + i] = p.in.w[s + i];
    }
  }
  __threadfence_block();
  __syncthreads();
  if ((p.flags & kDoCollide) && threadIdx.x == 0) {
    GlobalVel acc{p.out.u, p.out.v, p.out.w, s};
    collide_cell(p, cell, (int)n, acc, step, sel, col, sum_g);
  }
  __threadfence_block();
  __syncthreads();
  double su = 0, sv = 0, sw = 0, se = 0;
  for (uint32_t qb = 0; qb < n; qb += blockDim.x) {
    uint32_t q = qb + threadIdx.x;
    bool active = q < n;
    float3 pos = make_float3(0.f, 0.f, 0.f), vel = pos;
    bool live = true;
    if (active) {
      uint32_t g = s + q;
      if (!vel_only) pos = make_float3(p.out.x[g], p.out.y[g], p.out.z[g]);
      vel = make_float3(p.out.u[g], p.out.v[g], p.out.w[g]);
      if (p.flags & kDoMove) live = move_particle(p, pos, vel, g, step);
      if (do_sample) {
        double x = vel.x, y = vel.y, z = vel.z;
        su += x; sv += y; sw += z;
        se += x * x + y * y + z * z;
      }
      if (!vel_only) { p.out.x[g] = pos.x; p.out.y[g] = pos.y; p.out.z[g] = pos.z; }
      p.out.u[g] = vel.x; p.out.v[g] = vel.y; p.out.w[g] = vel.z;
    }
    if (p.flags & kDoKeys) {
      bool has_key = active && live;
      unsigned m = __ballot_sync(kFull, has_key);
      if (active && !live) removed++;
      if (has_key) {
        uint32_t key = cell_id3d(p.grid, pos.x, pos.y, pos.z);
        uint32_t t = warp_ticket(p.count, key, m, s_tile);
        p.out_kt[s + q] = make_uint2(key, t);
      } else if (active) {
        p.out_kt[s + q] = make_uint2(kDeadKey, 0u);
      }
    }
  }
  if (do_sample) {
    __shared__ double red[4][kCellThreads / 32];
    su = warp_sum_f64(su); sv = warp_sum_f64(sv); sw = warp_sum_f64(sw); se = warp_sum_f64(se);
    __syncthreads();
    if (lane_id() == 0) {
      red[0][threadIdx.x / 32] = su; red[1][threadIdx.x / 32] = sv;
      red[2][threadIdx.x / 32] = sw; red[3][threadIdx.x / 32] = se;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
      for (int i = 0; i < (int)(blockDim.x / 32); i++) {
        a0 += red[0][i]; a1 += red[1][i]; a2 += red[2][i]; a3 += red[3][i];
      }
      p.acc[cell] += (double)n;
      p.acc[(size_t)p.cells + cell] += a0;
      p.acc[2 * (size_t)p.cells + cell] += a1;
      p.acc[3 * (size_t)p.cells + cell] += a2;
      p.acc[4 * (size_t)p.cells + cell] += a3;
    }
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kCellThreads, 2) k_cell(const StepParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  CellSmem S = carve_smem(smem_raw);
  const uint32_t step = p.step_override ? p.step_override : p.meta->step;
  const bool do_sample =
      (p.flags & kDoSample) &&
      ((p.flags & kSampleForce) || (p.sample_every > 0 && step % (uint32_t)p.sample_every == 0));
  const bool do_keys = (p.flags & kDoKeys) != 0;
  const bool do_fixup = (p.flags & kDoFixup) != 0;
  const bool do_move = (p.flags & kDoMove) != 0;
  const bool vel_only = (p.flags & kVelOnly) != 0;
  if (do_keys)
    for (uint32_t t = threadIdx.x; t < p.n_scan_tiles; t += blockDim.x) S.s_tile[t] = 0;

  uint32_t sel = 0, col = 0, removed = 0;
  double sum_g = 0.0;
  const int ct = p.cells_per_tile;

  for (uint32_t tile = blockIdx.x; tile < p.n_tiles; tile += gridDim.x) {
    const uint32_t c0 = tile * (uint32_t)ct;
    const uint32_t nct = min((uint32_t)ct, p.cells - c0);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i <= nct; i += blockDim.x) S.ls[i] = p.start[c0 + i];
    __syncthreads();
    uint32_t cur = 0;
    while (cur < nct) {
      const uint32_t base = S.ls[cur];
      // cells cur..cur+k-1 fit in the tile capacity
      uint32_t c = cur + 1 + threadIdx.x;
      int fits = (c <= nct) && (S.ls[c] - base <= (uint32_t)kTileCapacity);
      const uint32_t k = __syncthreads_count(fits);
      if (k == 0) {
        giant_cell(p, c0 + cur, base, S.ls[cur + 1], step, do_sample, S.s_tile, sel, col, sum_g,
                   removed);
        cur += 1;
        continue;
      }
      const uint32_t n = S.ls[cur + k] - base;
      for (uint32_t t = threadIdx.x; t < n; t += blockDim.x) {
        if (!vel_only) {
          S.x[t] = p.in.x[base + t]; S.y[t] = p.in.y[base + t]; S.z[t] = p.in.z[base + t];
        }
        S.u[t] = p.in.u[base + t]; S.v[t] = p.in.v[base + t]; S.w[t] = p.in.w[base + t];
        if (do_fixup) S.orig[t] = p.in_orig[base + t];
      }
      __syncthreads();
      // slot[sorted position] = staged index; sorted = (cell, orig) order
      for (uint32_t t = threadIdx.x; t < n; t += blockDim.x) {
        if (!do_fixup) {
          S.slot[t] = (uint16_t)t;
          continue;
        }
        // cell of staged particle t: last cc in [cur, cur+k) with ls[cc]-base <= t
        uint32_t lo = cur, hi = cur + k - 1;
        while (lo < hi) {
          uint32_t mid = (lo + hi + 1) >> 1;
          if (S.ls[mid] - base <= t) lo = mid; else hi = mid - 1;
        }
        const uint32_t s0 = S.ls[lo] - base, e0 = S.ls[lo + 1] - base;
        const uint32_t my = S.orig[t];
        uint32_t rank = 0;
        // ties (never produced by the scatter) fall back to staged order, so
        // slot[] is always a permutation of the chunk
        for (uint32_t j = s0; j < e0; j++) rank += (S.orig[j] < my) | ((S.orig[j] == my) & (j < t));
        S.slot[s0 + rank] = (uint16_t)t;
      }
      __syncthreads();
      if (p.flags & kDoCollide) {
        for (uint32_t lc = threadIdx.x; lc < k; lc += blockDim.x) {
          const uint32_t s0 = S.ls[cur + lc] - base, e0 = S.ls[cur + lc + 1] - base;
          SmemVel acc{S.u, S.v, S.w, S.slot, s0};
          collide_cell(p, c0 + cur + lc, (int)(e0 - s0), acc, step, sel, col, sum_g);
        }
        __syncthreads();
      }
      for (uint32_t qb = 0; qb < n; qb += blockDim.x) {
        const uint32_t q = qb + threadIdx.x;
        const bool active = q < n;
        float3 pos = make_float3(0.f, 0.f, 0.f), vel = pos;
        bool live = true;
        const uint32_t g = base + q;
        if (active) {
          const uint32_t j = S.slot[q];
          if (!vel_only) pos = make_float3(S.x[j], S.y[j], S.z[j]);
          vel = make_float3(S.u[j], S.v[j], S.w[j]);
          if (do_move) live = move_particle(p, pos, vel, g, step);
          if (do_sample) { S.u[j] = vel.x; S.v[j] = vel.y; S.w[j] = vel.z; }
          if (!vel_only) { p.out.x[g] = pos.x; p.out.y[g] = pos.y; p.out.z[g] = pos.z; }
          p.out.u[g] = vel.x; p.out.v[g] = vel.y; p.out.w[g] = vel.z;
        }
        if (do_keys) {
          const bool has_key = active && live;
          const unsigned m = __ballot_sync(kFull, has_key);
          if (active && !live) removed++;
          if (has_key) {
            const uint32_t key = cell_id3d(p.grid, pos.x, pos.y, pos.z);
            const uint32_t t = warp_ticket(p.count, key, m, S.s_tile);
            p.out_kt[g] = make_uint2(key, t);
          } else if (active) {
            p.out_kt[g] = make_uint2(kDeadKey, 0u);
          }
        }
      }
      if (do_sample) {
        __syncthreads();
        for (uint32_t lc = threadIdx.x; lc < k; lc += blockDim.x) {
          const uint32_t s0 = S.ls[cur + lc] - base, e0 = S.ls[cur + lc + 1] - base;
          SmemVel a{S.u, S.v, S.w, S.slot, s0};
          sample_cell(p.acc, p.cells, c0 + cur + lc, (int)(e0 - s0), a);
        }
      }
      cur += k;
      __syncthreads();
    }
  }
  __syncthreads();
  if (do_keys) flush_tile_hist(S.s_tile, p.tile_sum, p.n_scan_tiles);
  // collision and removal totals
  unsigned long long s64 = warp_sum_u64(sel), c64 = warp_sum_u64(col);
  double g = warp_sum_f64(sum_g);
  uint32_t r = warp_sum_u32(removed);
  if (lane_id() == 0 && p.meta) {
    if (s64) atomicAdd(&p.meta->selections, s64);
    if (c64) atomicAdd(&p.meta->collisions, c64);
    if (g != 0.0) atomicAdd(&p.meta->sum_g, g);
    if (r) atomicAdd(&p.meta->removed, r);
  }
  if (do_sample && p.meta && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&p.meta->samples, 1u);
}

// Move stage: free flight and boundaries for n particles in place.
__global__ void __launch_bounds__(256) k_move(const StepParams p, uint32_t n, uint32_t step) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float3 pos = make_float3(p.out.x[i], p.out.y[i], p.out.z[i]);
    float3 vel = make_float3(p.out.u[i], p.out.v[i], p.out.w[i]);
    bool live = move_particle(p, pos, vel, i, step);
    p.out.x[i] = live ? pos.x : __int_as_float(0x7fc00000);
    p.out.y[i] = pos.y; p.out.z[i] = pos.z;
    p.out.u[i] = vel.x; p.out.v[i] = vel.y; p.out.w[i] = vel.z;
  }
}

__global__ void __launch_bounds__(256) k_cell_ids(GridGeom g, const float* __restrict__ x,
                                                  const float* __restrict__ y,
                                                  const float* __restrict__ z, uint32_t n,
                                                  uint32_t* __restrict__ keys,
                                                  uint32_t* __restrict__ idx) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    keys[i] = cell_id3d(g, x[i], y[i], z[i]);
    if (idx) idx[i] = i;
  }
}

// ---------------------------------------------------------- index/scan ----

__global__ void k_index(GridGeom g, const float* __restrict__ x, const float* __restrict__ y,
                        const float* __restrict__ z, uint32_t n, uint2* __restrict__ kt,
                        uint32_t* count, uint32_t* tile_sum, uint32_t n_scan_tiles, int face_mode) {
  extern __shared__ uint32_t s_tile[];
  for (uint32_t t = threadIdx.x; t < n_scan_tiles; t += blockDim.x) s_tile[t] = 0;
  __syncthreads();
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    uint32_t i = base + threadIdx.x;
    bool active = i < n;
    bool live = false;
    uint32_t key = kDeadKey;
    if (active) {
      float px = x[i], py = y[i], pz = z[i];
      live = true;
      if (face_mode != 0 && (px < g.gmin.x || px > g.gmax.x || py < g.gmin.y || py > g.gmax.y ||
                             pz < g.gmin.z || pz > g.gmax.z))
        live = false;
      if (live) key = cell_id3d(g, px, py, pz);
    }
    unsigned m = __ballot_sync(kFull, active && live);
    if (active && live) {
      uint32_t t = warp_ticket(count, key, m, s_tile);
      kt[i] = make_uint2(key, t);
    } else if (active) {
      kt[i] = make_uint2(kDeadKey, 0u);
    }
  }
  __syncthreads();
  flush_tile_hist(s_tile, tile_sum, n_scan_tiles);
}

// Exclusive scan of per-cell counts.  Block b owns cells [b*2048, (b+1)*2048);
// its offset is the sum of the per-tile totals before it, which the producer
// kernels accumulated alongside the counts.
__global__ void __launch_bounds__(256) k_scan(uint32_t* count, uint32_t* start, uint32_t cells,
                                              const uint32_t* tile_sum, Meta* meta, int bump) {
  __shared__ uint32_t s_warp[8];
  __shared__ uint32_t s_base;
  const uint32_t b = blockIdx.x;
  uint32_t part = 0;
  for (uint32_t t = threadIdx.x; t < b; t += blockDim.x) part += tile_sum[t];
  part = warp_sum_u32(part);
  if (lane_id() == 0) s_warp[threadIdx.x / 32] = part;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t s = 0;
    for (int i = 0; i < 8; i++) s += s_warp[i];
    s_base = s;
  }
  __syncthreads();
  const uint32_t c0 = b * kScanTile + threadIdx.x * 8;
  uint32_t v[8];
  uint32_t tsum = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    v[i] = (c0 + i < cells) ? count[c0 + i] : 0u;
    tsum += v[i];
  }
  // block exclusive scan of thread sums
  uint32_t incl = tsum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(kFull, incl, o);
    if ((int)lane_id() >= o) incl += t;
  }
  __syncthreads();
  if (lane_id() == 31) s_warp[threadIdx.x / 32] = incl;
  __syncthreads();
  uint32_t warp_off = 0;
  for (uint32_t w = 0; w < threadIdx.x / 32; w++) warp_off += s_warp[w];
  uint32_t run = s_base + warp_off + incl - tsum;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    if (c0 + i < cells) {
      start[c0 + i] = run;
      count[c0 + i] = 0u;
    }
    run += v[i];
  }
  if (b == gridDim.x - 1 && threadIdx.x == blockDim.x - 1) {
    start[cells] = run;
    meta->n_scatter = meta->n_alive + meta->n_pending;
    meta->n_pending = 0;
    meta->n_alive = run;
    if (bump) {
      meta->step += 1;
      meta->particle_steps += run;
    }
  }
}

// Scatter into sorted order: dst[start[key] + ticket] = src[i], orig = i.
__global__ void __launch_bounds__(256) k_scatter(SoA src, SoA dst, const uint2* __restrict__ kt,
                                                 const uint32_t* __restrict__ start,
                                                 uint32_t* __restrict__ orig, uint32_t cells,
                                                 uint32_t* tile_sum, uint32_t n_scan_tiles,
                                                 Meta* meta, uint32_t capacity) {
  if (blockIdx.x == 0)
    for (uint32_t t = threadIdx.x; t < n_scan_tiles; t += blockDim.x) tile_sum[t] = 0;
  const uint32_t n = meta->n_scatter;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint2 k = kt[i];
    if (k.x == kDeadKey) continue;
    if (k.x >= cells) {
      atomicOr(&meta->error, kErrKeyRange);
      continue;
    }
    uint32_t d = __ldg(&start[k.x]) + k.y;
    if (d >= capacity) {
      atomicOr(&meta->error, kErrKeyRange);
      continue;
    }
    dst.x[d] = src.x[i]; dst.y[d] = src.y[i]; dst.z[d] = src.z[i];
    dst.u[d] = src.u[i]; dst.v[d] = src.v[i]; dst.w[d] = src.w[i];
    orig[d] = i;
  }
}

// ------------------------------------------------------------ sort stage ----

// Keys >= nkeys are left out of the sort (no ticket, no slot).
__global__ void k_count_keys(const uint32_t* __restrict__ keys, uint32_t n, uint32_t nkeys,
                             uint32_t* __restrict__ ticket, uint32_t* count, uint32_t* tile_sum,
                             uint32_t n_scan_tiles) {
  extern __shared__ uint32_t s_tile[];
  for (uint32_t t = threadIdx.x; t < n_scan_tiles; t += blockDim.x) s_tile[t] = 0;
  __syncthreads();
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    uint32_t i = base + threadIdx.x;
    uint32_t key = i < n ? keys[i] : kNone;
    bool active = i < n && key < nkeys;
    unsigned m = __ballot_sync(kFull, active);
    if (active) ticket[i] = warp_ticket(count, key, m, s_tile);
  }
  __syncthreads();
  flush_tile_hist(s_tile, tile_sum, n_scan_tiles);
}

__global__ void k_scatter_kv(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                             const uint32_t* __restrict__ ticket,
                             const uint32_t* __restrict__ start, uint32_t n, uint32_t nkeys,
                             uint32_t* __restrict__ tmp_val, uint32_t* __restrict__ tmp_pos) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t key = keys[i];
    if (key >= nkeys) continue;
    uint32_t d = start[key] + ticket[i];
    tmp_val[d] = vals[i];
    tmp_pos[d] = i;
  }
}

// Restores input order within each key: entry of rank r (by input position)
// among its key's entries goes to start[key] + r.
__global__ void __launch_bounds__(256) k_segment_fixup(const uint32_t* __restrict__ start,
                                                       uint32_t nkeys,
                                                       const uint32_t* __restrict__ tmp_val,
                                                       const uint32_t* __restrict__ tmp_pos,
                                                       uint32_t* __restrict__ keys_out,
                                                       uint32_t* __restrict__ vals_out) {
  constexpr int kCap = 4096;
  __shared__ uint32_t ls[257];
  __shared__ uint32_t spos[kCap];
  __shared__ uint32_t sval[kCap];
  const uint32_t ntiles = (nkeys + 255) / 256;
  for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const uint32_t c0 = tile * 256, nct = min(256u, nkeys - c0);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i <= nct; i += blockDim.x) ls[i] = start[c0 + i];
    __syncthreads();
    uint32_t cur = 0;
    while (cur < nct) {
      const uint32_t base = ls[cur];
      uint32_t c = cur + 1 + threadIdx.x;
      int fits = (c <= nct) && (ls[c] - base <= (uint32_t)kCap);
      const uint32_t k = __syncthreads_count(fits);
      if (k == 0) {
        // one key with more than kCap entries: rank from global memory
        const uint32_t s0 = base, e0 = ls[cur + 1];
        for (uint32_t i = s0 + threadIdx.x; i < e0; i += blockDim.x) {
          uint32_t my = tmp_pos[i], rank = 0;
          for (uint32_t j = s0; j < e0; j++) rank += tmp_pos[j] < my;
          keys_out[s0 + rank] = c0 + cur;
          vals_out[s0 + rank] = tmp_val[i];
        }
        cur += 1;
        __syncthreads();
        continue;
      }
      const uint32_t n = ls[cur + k] - base;
      for (uint32_t t = threadIdx.x; t < n; t += blockDim.x) {
        spos[t] = tmp_pos[base + t];
        sval[t] = tmp_val[base + t];
      }
      __syncthreads();
      for (uint32_t t = threadIdx.x; t < n; t += blockDim.x) {
        uint32_t lo = cur, hi = cur + k - 1;
        while (lo < hi) {
          uint32_t mid = (lo + hi + 1) >> 1;
          if (ls[mid] - base <= t) lo = mid; else hi = mid - 1;
        }
        const uint32_t s0 = ls[lo] - base, e0 = ls[lo + 1] - base;
        const uint32_t my = spos[t];
        uint32_t rank = 0;
        for (uint32_t j = s0; j < e0; j++) rank += spos[j] < my;
        keys_out[base + s0 + rank] = c0 + lo;
        vals_out[base + s0 + rank] = sval[t];
      }
      cur += k;
      __syncthreads();
    }
  }
}

// FindCellBoundariesDev (kernels/dsmc_kernel.cu:1734-1787): start/end per
// cell from sorted keys (cse zeroed by the caller) and the gather.
__global__ void k_bounds_reorder(const uint32_t* __restrict__ keys,
                                 const uint32_t* __restrict__ idx, uint32_t n, uint32_t ncells,
                                 uint2* cse, SoA src, SoA dst, int gather) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t h = keys[i];
    uint32_t hp = i > 0 ? keys[i - 1] : kNone;
    if (i == 0 || h != hp) {
      if (h < ncells) cse[h].x = i;
      if (i > 0 && hp < ncells) cse[hp].y = i;
    }
    if (i == n - 1 && h < ncells) cse[h].y = i + 1;
    if (gather) {
      uint32_t s = idx[i];
      dst.x[i] = src.x[s]; dst.y[i] = src.y[s]; dst.z[i] = src.z[s];
      dst.u[i] = src.u[s]; dst.v[i] = src.v[s]; dst.w[i] = src.w[s];
    }
  }
}

// Stand-alone FP64 sampling, one thread per cell (5 doubles per cell, AoS).
__global__ void k_sample_cells(const float* __restrict__ u, const float* __restrict__ v,
                               const float* __restrict__ w, const uint32_t* __restrict__ start,
                               uint32_t cells, double* acc, size_t fs, size_t cs) {
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < cells; c += gridDim.x * blockDim.x) {
    uint32_t s = start[c], e = start[c + 1];
    if (e <= s) continue;
    double su = 0, sv = 0, sw = 0, se = 0;
    for (uint32_t i = s; i < e; i++) {
      double x = u[i], y = v[i], z = w[i];
      su += x; sv += y; sw += z;
      se += x * x + y * y + z * z;
    }
    acc[c * cs] += (double)(e - s);
    acc[fs + c * cs] += su;
    acc[2 * fs + c * cs] += sv;
    acc[3 * fs + c * cs] += sw;
    acc[4 * fs + c * cs] += se;
  }
}

// ------------------------------------------------------------ init fill ----

// Initial population: part_per_cell particles per cell at uniform positions
// (GetRandomPosition, kernels/dsmc_kernel.cu:417-427) with either the
// reference's speed/angle sampler (GetRandomVelocity, :394-415) or an exact
// Maxwellian.  Random numbers come from Philox (the reference used its
// Mersenne-Twister table, which is not reproduced).
__global__ void k_init_fill(const InitParams p) {
  const uint32_t total = p.cells * p.ppc;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const uint32_t cell = i / p.ppc, k = i - cell * p.ppc;
    const uint32_t dst0 = p.cell_slot[cell];
    if (dst0 == kNone) continue;
    const uint32_t d = dst0 + k;
    const uint32_t cx = cell % p.grid.dim.x;
    const uint32_t cy = (cell / p.grid.dim.x) % p.grid.dim.y;
    const uint32_t cz = cell / (p.grid.dim.x * p.grid.dim.y);
    PhiloxStream r;
    r.init(p.seed, i, 0u, kPurposeInit);
    float3 vel;
    if (p.kind == 0) {
      float vv = p.vmp * sqrtf(-logf(r.uniform()));
      const float tetha = 2.0f * kPiF;
      vel.x = vv * sinf(r.uniform() * tetha) + p.stream.x;
      vel.y = vv * sinf(r.uniform() * tetha) + p.stream.y;
      vel.z = vv * sinf(r.uniform() * tetha) + p.stream.z;
    } else {
      float sd = (p.kind == 2 && (i & 1u)) ? p.vstd2 : p.vstd;
      float r1 = r.uniform(), r2 = r.uniform(), r3 = r.uniform(), r4 = r.uniform();
      float m1 = sd * sqrtf(-2.f * logf(r1)), m2 = sd * sqrtf(-2.f * logf(r3));
      float s1, c1, s2, c2;
      sincosf(6.2831853f * r2, &s1, &c1);
      sincosf(6.2831853f * r4, &s2, &c2);
      vel = make_float3(m1 * c1 + p.stream.x, m1 * s1 + p.stream.y, m2 * c2 + p.stream.z);
    }
    float3 cellmin = make_float3(p.grid.gmin.x + cx * p.grid.cell.x, p.grid.gmin.y + cy * p.grid.cell.y,
                                 p.grid.gmin.z + cz * p.grid.cell.z);
    float px = cellmin.x + r.uniform() * p.grid.cell.x;
    float py = cellmin.y + r.uniform() * p.grid.cell.y;
    float pz = cellmin.z + r.uniform() * p.grid.cell.z;
    p.out.x[d] = px; p.out.y[d] = py; p.out.z[d] = pz;
    p.out.u[d] = vel.x; p.out.v[d] = vel.y; p.out.w[d] = vel.z;
  }
}

// --------------------------------------------------------------- inflow ----

// Plan: number of particles each inflow face injects this step (carrying the
// fractional remainder), reserved after the particles already in the array.
__global__ void k_inject_plan(const InjectParams p, uint32_t* plan) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  float want = *p.remainder + p.inflow.number_flux * p.inflow.area * p.dt;
  uint32_t k = want > 0.f ? (uint32_t)want : 0u;
  const uint32_t have = p.meta->n_alive + p.meta->n_pending;
  if (have + k > p.capacity) {
    atomicOr(&p.meta->error, kErrCapacity);
    k = have < p.capacity ? p.capacity - have : 0u;
  }
  *p.remainder = want - (float)k;
  plan[0] = have;  // first slot
  plan[1] = k;
  p.meta->n_pending += k;
  p.meta->injected += k;
}

// Samples the inward normal speed of the drifting Maxwellian weighted by
// flux, f(z) ~ z exp(-(z - s)^2) for z = v_n / c_mp > 0, by rejection from the
// envelope (|y| + max(s,0)) exp(-y^2), y = z - s.
__device__ __forceinline__ float sample_flux_normal(float s, PhiloxStream& r) {
  const float sp = fmaxf(s, 0.f);
  const float w_abs = 1.f / (1.f + sp * 1.7724539f);
  for (int it = 0; it < 64; it++) {
    float y;
    if (r.uniform() < w_abs) {
      y = sqrtf(-logf(r.uniform()));
      if (r.uniform() < 0.5f) y = -y;
    } else {
      float a = r.uniform(), b = r.uniform();
      y = sqrtf(-logf(a)) * cosf(6.2831853f * b);  // N(0, 1/2)
    }
    float z = s + y;
    if (z <= 0.f) continue;
    if (r.uniform() * (fabsf(y) + sp) <= z) return z;
  }
  return fmaxf(s, 1e-3f);
}

__global__ void k_inject_fill(const InjectParams p, const uint32_t* plan) {
  const uint32_t step = p.meta->step;
  extern __shared__ uint32_t s_tile[];
  for (uint32_t t = threadIdx.x; t < (uint32_t)kMaxScanTiles; t += blockDim.x) s_tile[t] = 0;
  __syncthreads();
  const uint32_t first = plan[0], k = plan[1];
  const int face = p.inflow.face;
  const int ax = face >> 1;
  const float sign = (face & 1) ? -1.f : 1.f;  // inward normal along +axis for the low face
  const GridGeom& g = p.grid;
  const float cmp = p.inflow.vstd * 1.41421356f;
  const float un = sign * compc(p.inflow.stream, ax);
  const float s = un / cmp;
  for (uint32_t base = blockIdx.x * blockDim.x; base < k; base += gridDim.x * blockDim.x) {
    uint32_t i = base + threadIdx.x;
    bool active = i < k;
    bool live = false;
    uint32_t key = kDeadKey;
    float3 pos = make_float3(0, 0, 0), vel = pos;
    if (active) {
      PhiloxStream r;
      r.init(p.seed, i, step, kPurposeInject);
      float vn = sample_flux_normal(s, r) * cmp * sign;
      float a1 = r.uniform(), a2 = r.uniform();
      float rad = p.inflow.vstd * sqrtf(-2.f * logf(a1));
      float sn, cs;
      sincosf(6.2831853f * a2, &sn, &cs);
      float t1 = rad * cs, t2 = rad * sn;
      int a_t1 = (ax + 1) % 3, a_t2 = (ax + 2) % 3;
      comp(vel, ax) = vn;
      comp(vel, a_t1) = t1 + compc(p.inflow.stream, a_t1);
      comp(vel, a_t2) = t2 + compc(p.inflow.stream, a_t2);
      comp(pos, ax) = (face & 1) ? compc(g.gmax, ax) : compc(g.gmin, ax);
      comp(pos, a_t1) = compc(g.gmin, a_t1) + r.uniform() * (compc(g.gmax, a_t1) - compc(g.gmin, a_t1));
      comp(pos, a_t2) = compc(g.gmin, a_t2) + r.uniform() * (compc(g.gmax, a_t2) - compc(g.gmin, a_t2));
      float frac = r.uniform() * p.dt;
      pos.x += vel.x * frac; pos.y += vel.y * frac; pos.z += vel.z * frac;
      live = !(pos.x < g.gmin.x || pos.x > g.gmax.x || pos.y < g.gmin.y || pos.y > g.gmax.y ||
               pos.z < g.gmin.z || pos.z > g.gmax.z);
      if (live) key = cell_id3d(g, pos.x, pos.y, pos.z);
      uint32_t d = first + i;
      p.st.x[d] = pos.x; p.st.y[d] = pos.y; p.st.z[d] = pos.z;
      p.st.u[d] = vel.x; p.st.v[d] = vel.y; p.st.w[d] = vel.z;
    }
    unsigned m = __ballot_sync(kFull, active && live);
    if (active && live) {
      uint32_t t = warp_ticket(p.count, key, m, s_tile);
      p.kt[first + i] = make_uint2(key, t);
    } else if (active) {
      p.kt[first + i] = make_uint2(kDeadKey, 0u);
    }
  }
  __syncthreads();
  flush_tile_hist(s_tile, p.tile_sum, (p.cells + kScanTile - 1) / kScanTile);
}

int num_sms() {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  return sms;
}

uint32_t grid_for(uint64_t work, int threads, int per_sm) {
  uint64_t need = (work + threads - 1) / threads;
  uint64_t cap = (uint64_t)num_sms() * per_sm;
  if (need < 1) need = 1;
  return (uint32_t)(need < cap ? need : cap);
}

}  // namespace

int cell_kernel_smem_bytes() { return kCellSmemBytes; }

cudaError_t launch_index(const GridGeom& g, uint32_t cells, const float* x, const float* y,
                         const float* z, uint32_t n, uint2* kt, uint32_t* count,
                         uint32_t* tile_sum, uint32_t n_scan_tiles, int face_mode,
                         cudaStream_t stream) {
  (void)cells;
  uint32_t grid = grid_for(n, 256, 8);
  k_index<<<grid, 256, n_scan_tiles * 4, stream>>>(g, x, y, z, n, kt, count, tile_sum,
                                                   n_scan_tiles, face_mode);
  return cudaGetLastError();
}

cudaError_t launch_scan(uint32_t* count, uint32_t* start, uint32_t cells, const uint32_t* tile_sum,
                        uint32_t n_scan_tiles, Meta* meta, int bump_step, cudaStream_t stream) {
  k_scan<<<n_scan_tiles, 256, 0, stream>>>(count, start, cells, tile_sum, meta, bump_step);
  return cudaGetLastError();
}

cudaError_t launch_scatter(const SoA& src, SoA dst, const uint2* kt, const uint32_t* start,
                           uint32_t* orig, uint32_t cells, uint32_t* tile_sum,
                           uint32_t n_scan_tiles, Meta* meta, uint32_t capacity,
                           cudaStream_t stream) {
  uint32_t grid = (uint32_t)num_sms() * 8;
  k_scatter<<<grid, 256, 0, stream>>>(src, dst, kt, start, orig, cells, tile_sum, n_scan_tiles,
                                      meta, capacity);
  return cudaGetLastError();
}

cudaError_t launch_cell(const StepParams& p, cudaStream_t stream) {
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(k_cell, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kCellSmemBytes);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  uint32_t grid = (uint32_t)num_sms() * 2;
  if (grid > p.n_tiles) grid = p.n_tiles;
  if (grid == 0) return cudaSuccess;
  k_cell<<<grid, kCellThreads, kCellSmemBytes, stream>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_move(const StepParams& p, uint32_t n, uint32_t step, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  uint32_t grid = grid_for(n, 256, 8);
  k_move<<<grid, 256, 0, stream>>>(p, n, step);
  return cudaGetLastError();
}

cudaError_t launch_cell_ids(const GridGeom& g, const float* x, const float* y, const float* z,
                            uint32_t n, uint32_t* keys, uint32_t* idx, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  uint32_t grid = grid_for(n, 256, 8);
  k_cell_ids<<<grid, 256, 0, stream>>>(g, x, y, z, n, keys, idx);
  return cudaGetLastError();
}

cudaError_t launch_count_keys(const uint32_t* keys, uint32_t n, uint32_t nkeys, uint32_t* ticket, uint32_t* count,
                              uint32_t* tile_sum, uint32_t n_scan_tiles, cudaStream_t stream) {
  uint32_t grid = grid_for(n, 256, 8);
  k_count_keys<<<grid, 256, n_scan_tiles * 4, stream>>>(keys, n, nkeys, ticket, count, tile_sum,
                                                        n_scan_tiles);
  return cudaGetLastError();
}

cudaError_t launch_scatter_kv(const uint32_t* keys, const uint32_t* vals, const uint32_t* ticket,
                              const uint32_t* start, uint32_t n, uint32_t nkeys, uint32_t* tmp_val,
                              uint32_t* tmp_pos, cudaStream_t stream) {
  uint32_t grid = grid_for(n, 256, 8);
  k_scatter_kv<<<grid, 256, 0, stream>>>(keys, vals, ticket, start, n, nkeys, tmp_val, tmp_pos);
  return cudaGetLastError();
}

cudaError_t launch_segment_fixup(const uint32_t* start, uint32_t nkeys, const uint32_t* tmp_val,
                                 const uint32_t* tmp_pos, uint32_t* keys_out, uint32_t* vals_out,
                                 cudaStream_t stream) {
  uint32_t ntiles = (nkeys + 255) / 256;
  uint32_t grid = ntiles < (uint32_t)num_sms() * 4 ? ntiles : (uint32_t)num_sms() * 4;
  if (grid == 0) return cudaSuccess;
  k_segment_fixup<<<grid, 256, 0, stream>>>(start, nkeys, tmp_val, tmp_pos, keys_out, vals_out);
  return cudaGetLastError();
}

cudaError_t launch_bounds_reorder(const uint32_t* keys, const uint32_t* idx, uint32_t n,
                                  uint32_t ncells, uint32_t* cse, const float* const src[6], float* const dst[6],
                                  cudaStream_t stream) {
  SoA s{const_cast<float*>(src ? src[0] : nullptr), const_cast<float*>(src ? src[1] : nullptr),
        const_cast<float*>(src ? src[2] : nullptr), const_cast<float*>(src ? src[3] : nullptr),
        const_cast<float*>(src ? src[4] : nullptr), const_cast<float*>(src ? src[5] : nullptr)};
  SoA d{dst ? dst[0] : nullptr, dst ? dst[1] : nullptr, dst ? dst[2] : nullptr,
        dst ? dst[3] : nullptr, dst ? dst[4] : nullptr, dst ? dst[5] : nullptr};
  uint32_t grid = grid_for(n, 256, 8);
  k_bounds_reorder<<<grid, 256, 0, stream>>>(keys, idx, n, ncells, (uint2*)cse, s, d,
                                             (src && dst) ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_sample_cells(const float* u, const float* v, const float* w,
                                const uint32_t* start, uint32_t cells, double* acc,
                                size_t fstride, size_t cstride, cudaStream_t stream) {
  uint32_t grid = grid_for(cells, 256, 8);
  k_sample_cells<<<grid, 256, 0, stream>>>(u, v, w, start, cells, acc, fstride, cstride);
  return cudaGetLastError();
}

cudaError_t launch_init_fill(const InitParams& p, cudaStream_t stream) {
  uint64_t total = (uint64_t)p.cells * p.ppc;
  uint32_t grid = grid_for(total, 256, 8);
  k_init_fill<<<grid, 256, 0, stream>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_inject(const InjectParams& p, cudaStream_t stream) {
  k_inject_plan<<<1, 32, 0, stream>>>(p, p.plan);
  uint32_t grid = (uint32_t)num_sms();
  k_inject_fill<<<grid, 256, kMaxScanTiles * 4, stream>>>(p, p.plan);
  return cudaGetLastError();
}

}  // namespace dsmcb
