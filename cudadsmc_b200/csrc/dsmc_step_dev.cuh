// Device code shared by the timestep's kernels: warp helpers, RNG views,
// the NTC collision routines, boundaries and the per-particle flight.
#pragma once

#include "dsmc_kernels.cuh"

namespace dsmcb {
namespace dev {

constexpr unsigned kFull = 0xffffffffu;
// NTC selections at which a cell is collided by a whole warp (Philox mode).
constexpr uint32_t kHeavyMin = 8;

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

// Adds the lane's key to count[key] and to the block's histogram of scan
// tiles: one atomic each per lane, no return value (measured faster than
// matching the warp's equal keys first, or than one tile atomic per warp
// when the lanes share a tile).  mask: the calling lanes.
__device__ __forceinline__ void warp_count_key(uint32_t* count, uint32_t key, unsigned mask,
                                               uint32_t* s_tile) {
  (void)mask;
  atomicAdd(&count[key], 1u);
  atomicAdd(&s_tile[key >> kScanShift], 1u);
}

// Adds the lanes of `mask` holding `key` to count[key] and to the per scan
// tile totals in global memory (one atomic per distinct key and one per
// distinct scan tile per warp): for kernels without a block-wide histogram.
__device__ __forceinline__ void warp_count_key_global(uint32_t* count, uint32_t key, unsigned mask,
                                                      uint32_t* tile_sum) {
  const unsigned lane = lane_id();
  const unsigned peers = __match_any_sync(mask, key);
  if ((int)lane == __ffs(peers) - 1) atomicAdd(&count[key], (uint32_t)__popc(peers));
  const uint32_t tk = key >> kScanShift;
  const unsigned tpeers = __match_any_sync(mask, tk);
  if ((int)lane == __ffs(tpeers) - 1) atomicAdd(&tile_sum[tk], (uint32_t)__popc(tpeers));
}

// Ticket from a per-key counter, aggregated over the lanes of `mask` holding
// the same key.
__device__ __forceinline__ uint32_t warp_ticket(uint32_t* counter, uint32_t key, unsigned mask) {
  const unsigned peers = __match_any_sync(mask, key);
  const int leader = __ffs(peers) - 1;
  const unsigned lane = lane_id();
  uint32_t base = 0;
  if ((int)lane == leader) base = atomicAdd(&counter[key], (uint32_t)__popc(peers));
  base = __shfl_sync(mask, base, leader);
  return base + __popc(peers & ((1u << lane) - 1u));
}

__device__ __forceinline__ void flush_tile_hist(uint32_t* s_tile, uint32_t* tile_sum, uint32_t n) {
  for (uint32_t t = threadIdx.x; t < n; t += blockDim.x) {
    const uint32_t v = s_tile[t];
    if (v) atomicAdd(&tile_sum[t], v);
  }
}

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
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
constexpr uint32_t kPurposePairs = 0x70616972u;  // a light cell's pair choices
constexpr uint32_t kPurposeWall = 0x77616c6cu;
constexpr uint32_t kPurposeInit = 0x696e6974u;
constexpr uint32_t kPurposeInject = 0x696e6a65u;
constexpr uint32_t kPurposeHeavy = 0x68650000u;  // + lane

// ------------------------------------------------------ velocity access ----

struct SmemVel {
  float* u; float* v; float* w;
  const uint16_t* slot;
  uint32_t off;
  __device__ __forceinline__ float3 get(uint32_t k) const {
    const uint32_t j = slot[off + k];
    return make_float3(u[j], v[j], w[j]);
  }
  __device__ __forceinline__ void set(uint32_t k, float3 a) const {
    const uint32_t j = slot[off + k];
    u[j] = a.x; v[j] = a.y; w[j] = a.z;
  }
  // a distinct small index per particle of the cell (pair claims)
  __device__ __forceinline__ uint32_t claim_index(uint32_t k) const { return slot[off + k]; }
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
  __device__ __forceinline__ uint32_t claim_index(uint32_t k) const { return k; }
};

// Per-cell collision state of one cell, wherever it is staged.
struct CellState {
  float2* maxrem;  // (sigma*g)max, remainder
  uint4* seed;     // HybridTaus state (reference RNG mode)
  float4* stat4;   // optional per-cell (selections, collisions, sum g)
};

// ------------------------------------------------------------- collide ----

__device__ __forceinline__ float sigma_g(const StepParams& p, float mag) {
  if (p.hard_sphere) return mag * p.cross_section;
  return mag > 0.f ? mag * (p.cross_section * powf(p.vhs_gref / mag, p.vhs_exp)) : 0.f;
}

__device__ __forceinline__ float lg2_approx(float x) {
  float r;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float ex2_approx(float x) {
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// sigma(g) g of the Philox mode: the VHS power law as
// sigma_ref g_ref^e 2^((1 - e) log2 g) with the hardware base-2 log and
// exponential (relative error about 1e-6, far below what an acceptance test
// R < sigma g / (sigma g)max can resolve).  Every rounding step is explicit
// (no contraction), so that a CPU restatement evaluates the same steps.
__device__ __forceinline__ float sigma_g_fast(const StepParams& p, float mag) {
  if (p.hard_sphere) return __fmul_rn(mag, p.cross_section);
  return mag > 0.f ? __fmul_rn(p.vhs_k, ex2_approx(__fmul_rn(p.vhs_c1, lg2_approx(mag)))) : 0.f;
}

// |a - b| of the Philox mode with explicit rounding: sqrt(dz^2 + (dx^2 + dy^2)),
// each square-add fused.
__device__ __forceinline__ float rel_speed(float3 a, float3 b) {
  const float dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
  return sqrtf(fmaf(dz, dz, fmaf(dx, dx, __fmul_rn(dy, dy))));
}

// NTC collisions of one cell with the reference's arithmetic:
// ComputeBirdCollisionsNoMTDev, kernels/dsmc_kernel.cu:912-1000.  Particles of
// the cell are acc.get(0..n-1) in sorted order; pair members are
// start + rand % n; the pair count is evaluated in double.  In two parts: the
// pair count (which also leaves the new remainder in vmax.y) and the
// selections, so that kernels may do them apart.
__device__ __forceinline__ uint32_t ntc_pairs_reference(const StepParams& p, int partCount,
                                                        float2& vmax) {
  const float avgConc = p.ntc_local ? (float)(partCount - 1) : p.avg_conc;
  float fpc = (0.5 * partCount * avgConc * p.fnum * vmax.x * p.dt) / p.cell_volume + vmax.y;
  uint32_t pairsCount = fpc;
  vmax.y = fpc - pairsCount;
  return pairsCount;
}

template <class Rng, class Acc>
__device__ __forceinline__ void ntc_select_reference(const StepParams& p, int partCount, Acc acc,
                                                     Rng& rng, uint32_t pairsCount, float2& vmax,
                                                     float4& stat, uint32_t& col, double& sum_g) {
  for (uint32_t i = 0; i < pairsCount; i++) {
    uint32_t px = rng.u32() % (uint32_t)partCount;
    float3 v1 = acc.get(px);
    uint32_t py = rng.u32() % (uint32_t)partCount;
    float3 v2 = acc.get(py);
    float mag = length3(make_float3(v1.x - v2.x, v1.y - v2.y, v1.z - v2.z));
    float v = sigma_g(p, mag);
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
}

template <class Rng, class Acc>
__device__ __forceinline__ void ntc_reference(const StepParams& p, int partCount, Acc acc, Rng& rng,
                                              CellState cs, uint32_t& sel, uint32_t& col,
                                              double& sum_g) {
  float4 stat = make_float4(0.f, 0.f, 0.f, 0.f);
  if (cs.stat4) stat = *cs.stat4;
  float2 vmax = *cs.maxrem;
  const uint32_t pairsCount = ntc_pairs_reference(p, partCount, vmax);
  stat.x += pairsCount;
  sel += pairsCount;
  ntc_select_reference(p, partCount, acc, rng, pairsCount, vmax, stat, col, sum_g);
  *cs.maxrem = vmax;
  if (cs.stat4) *cs.stat4 = stat;
}

// Selections of a cell in the Philox mode: FP32, with the host-folded
// coefficient 0.5 fnum dt / V_c.
__device__ __forceinline__ float ntc_fpc_fast(const StepParams& p, uint32_t n, float2 vm) {
  const float avg = p.ntc_local ? (float)(n - 1) : p.avg_conc;
  return fmaf(__fmul_rn(__fmul_rn(p.ntc_coef, (float)n), avg), vm.x, vm.y);
}

// Isotropic post-collision velocities (hard sphere / VHS), accurate angles.
// Rounding steps are explicit (no contraction): cos chi = 2 R - 1,
// sin chi = sqrt(1 - cos^2 chi), the azimuth from sincospi, g'/2 added to and
// taken from the centre-of-mass velocity.
__device__ __forceinline__ void scatter_pair(float3 v1, float3 v2, float mag, float r_cos,
                                             float r_phi, float3& o1, float3& o2) {
  const float b = fmaf(2.0f, r_cos, -1.0f);
  const float a = sqrtf(fmaxf(0.f, fmaf(-b, b, 1.f)));
  float sn, cn;
  sincospif(2.0f * r_phi, &sn, &cn);
  const float h = 0.5f * mag;
  const float ah = __fmul_rn(a, h);
  const float3 ang = make_float3(__fmul_rn(b, h), __fmul_rn(ah, cn), __fmul_rn(ah, sn));
  const float3 cm = make_float3(0.5f * (v1.x + v2.x), 0.5f * (v1.y + v2.y), 0.5f * (v1.z + v2.z));
  o1 = make_float3(cm.x + ang.x, cm.y + ang.y, cm.z + ang.z);
  o2 = make_float3(cm.x - ang.x, cm.y - ang.y, cm.z - ang.z);
}

// Pair count of the Philox mode (leaves the new remainder in vm.y).
__device__ __forceinline__ uint32_t ntc_pairs_fast(const StepParams& p, uint32_t n, float2& vm) {
  const float fpc = ntc_fpc_fast(p, n, vm);
  const uint32_t M = (uint32_t)fpc;
  vm.y = fpc - (float)M;
  return M;
}

// NTC selections of one cell in the Philox mode (one lane): distinct pairs,
// acceptance sigma*g > R (sigma*g)max; returns the collisions.  The pairs
// are drawn from the cell's pair stream and the acceptance and scattering
// numbers from its collision stream, so the next pair is known before this
// one is decided: its velocities are loaded while this pair is evaluated
// (loads issued before this pair's stores; where the two pairs share a
// particle the next pair takes this pair's result instead).
template <class Acc>
__device__ __forceinline__ uint32_t ntc_select_fast(const StepParams& p, uint32_t cell, uint32_t n,
                                                    Acc acc, uint32_t step, uint32_t M, float2& vm,
                                                    double& sum_g) {
  PhiloxStreamInline r, q;
  r.init(p.seed, cell, step, kPurposeCollide);
  q.init(p.seed, cell, step, kPurposePairs);
  uint32_t ncol = 0;
  if (M == 0) return 0;
  auto draw = [&](uint32_t& a, uint32_t& b) {
    a = __umulhi(q.next(), n);
    b = a + 1u + __umulhi(q.next(), n - 1u);
    if (b >= n) b -= n;
  };
  uint32_t pi, pj;
  draw(pi, pj);
  float3 v1 = acc.get(pi), v2 = acc.get(pj);
  for (uint32_t i = 0; i < M; i++) {
    uint32_t ni = 0, nj = 0;
    float3 w1 = v1, w2 = v2;
    const bool more = i + 1 < M;
    if (more) {
      draw(ni, nj);
      w1 = acc.get(ni);
      w2 = acc.get(nj);
    }
    const float mag = rel_speed(v1, v2);
    const float v = sigma_g_fast(p, mag);
    if (v > r.uniform() * vm.x) {
      ncol++;
      sum_g += mag;
      float3 o1, o2;
      const float rc = r.uniform(), rp = r.uniform();
      scatter_pair(v1, v2, mag, rc, rp, o1, o2);
      acc.set(pi, o1);
      acc.set(pj, o2);
      if (ni == pi) w1 = o1; else if (ni == pj) w1 = o2;
      if (nj == pi) w2 = o1; else if (nj == pj) w2 = o2;
    }
    if (v > vm.x) vm.x = v;
    pi = ni;
    pj = nj;
    v1 = w1;
    v2 = w2;
  }
  return ncol;
}

template <class Acc>
__device__ __forceinline__ void ntc_fast(const StepParams& p, uint32_t cell, uint32_t n, Acc acc,
                                         uint32_t step, CellState cs, uint32_t& sel, uint32_t& col,
                                         double& sum_g) {
  float2 vm = *cs.maxrem;
  const uint32_t M = ntc_pairs_fast(p, n, vm);
  sel += M;
  const uint32_t ncol = ntc_select_fast(p, cell, n, acc, step, M, vm, sum_g);
  col += ncol;
  *cs.maxrem = vm;
  if (cs.stat4) {
    float4 s = *cs.stat4;
    s.x += M;
    s.y += ncol;
    *cs.stat4 = s;
  }
}

// One cell's collisions in the configured mode (one lane).
template <class Acc>
__device__ __forceinline__ void collide_cell(const StepParams& p, uint32_t cell, int partCount,
                                             Acc acc, uint32_t step, CellState cs, uint32_t& sel,
                                             uint32_t& col, double& sum_g) {
  if (partCount < 2) return;
  if (p.rng_kind == 0) {
    TausRng r;
    r.s = *cs.seed;
    ntc_reference(p, partCount, acc, r, cs, sel, col, sum_g);
    *cs.seed = r.s;
  } else {
    ntc_fast(p, cell, (uint32_t)partCount, acc, step, cs, sel, col, sum_g);
  }
}

// NTC selections of one dense cell by a whole warp (Philox mode).  Pairs are
// distinct particles drawn uniformly; each round processes every pair whose
// two particles are not claimed by a lower lane, the others retry with the
// same pair.  Acceptance uses (sigma*g)max as of the round's start.  M pairs
// from vmax_in; returns the new (sigma*g)max (the same in every lane).
// claim[] holds 0xffffffff for every claim index of the cell and is left so.
template <class Acc>
__device__ __forceinline__ float ntc_select_heavy_warp(const StepParams& p, uint32_t cell,
                                                       uint32_t n, Acc acc, uint32_t* claim,
                                                       uint32_t step, uint32_t M, float vmax_in,
                                                       uint32_t& col, double& sum_g) {
  const unsigned lane = lane_id();
  float vmax = vmax_in;
  PhiloxStreamInline rng;
  rng.init(p.seed, cell, step, kPurposeHeavy + lane);
  uint32_t drawn = 0, done = 0, pi = 0, pj = 0, ncol = 0;
  bool pend = false;
  while (done < M) {
    const unsigned idle = __ballot_sync(kFull, !pend);
    const uint32_t want = min((uint32_t)__popc(idle), M - drawn);
    const uint32_t r = __popc(idle & ((1u << lane) - 1u));
    if (!pend && r < want) {
      pi = __umulhi(rng.next(), n);
      pj = pi + 1u + __umulhi(rng.next(), n - 1u);
      if (pj >= n) pj -= n;
      pend = true;
    }
    drawn += want;
    uint32_t ji = 0, jj = 0;
    if (pend) {
      ji = acc.claim_index(pi);
      jj = acc.claim_index(pj);
      atomicMin(&claim[ji], lane);
      atomicMin(&claim[jj], lane);
    }
    __syncwarp();
    const bool win = pend && claim[ji] == lane && claim[jj] == lane;
    float vv = 0.f;
    if (win) {
      const float3 v1 = acc.get(pi), v2 = acc.get(pj);
      const float mag = rel_speed(v1, v2);
      vv = sigma_g_fast(p, mag);
      if (vv > rng.uniform() * vmax) {
        ncol++;
        sum_g += mag;
        float3 o1, o2;
        const float rc = rng.uniform(), rp = rng.uniform();
        scatter_pair(v1, v2, mag, rc, rp, o1, o2);
        acc.set(pi, o1);
        acc.set(pj, o2);
      }
    }
    __syncwarp();
    if (pend) {
      claim[ji] = 0xffffffffu;
      claim[jj] = 0xffffffffu;
    }
    if (win) pend = false;
    done += __popc(__ballot_sync(kFull, win));
    float mx = vv;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(kFull, mx, o));
    vmax = fmaxf(vmax, mx);
    __syncwarp();
  }
  col += ncol;
  return vmax;
}

template <class Acc>
__device__ __forceinline__ void ntc_heavy_warp(const StepParams& p, uint32_t cell, uint32_t n,
                                               Acc acc, uint32_t* claim, uint32_t step,
                                               CellState cs, uint32_t& sel, uint32_t& col,
                                               double& sum_g) {
  const unsigned lane = lane_id();
  const float2 vm = *cs.maxrem;
  const float fpc = ntc_fpc_fast(p, n, vm);
  const uint32_t M = (uint32_t)fpc;
  const uint32_t col0 = col;
  const float vmax = ntc_select_heavy_warp(p, cell, n, acc, claim, step, M, vm.x, col, sum_g);
  const uint32_t wcol = warp_sum(col - col0);
  if (lane == 0) {
    sel += M;
    *cs.maxrem = make_float2(vmax, fpc - (float)M);
    if (cs.stat4) {
      float4 s = *cs.stat4;
      s.x += M;
      s.y += wcol;
      *cs.stat4 = s;
    }
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

// One domain face (extension): specular and diffuse walls with the exact
// crossing point, outflow (particle removed), periodic wrap.  Returns false
// when the particle left the domain.
__device__ __forceinline__ bool face_axis(const StepParams& p, float& x, float& vx, float lo,
                                          float hi, int face_lo, float3& pos, float3& vel,
                                          int axis, PhiloxStream& rng) {
  int face = -1;
  float bound = 0.f;
  if (x < lo) { face = face_lo; bound = lo; }
  else if (x > hi) { face = face_lo + 1; bound = hi; }
  if (face < 0) return true;
  const int kind = p.face_kind[face];
  if (kind == 2 || kind == 4) return false;  // outflow / inflow face: leaves
  if (kind == 3) {
    x = (face & 1) ? x - (hi - lo) : x + (hi - lo);
    return true;
  }
  if (kind == 0) {
    x = fmaf(2.f, bound, -x);
    vx = -vx;
    return true;
  }
  // diffuse wall: back to the crossing point, re-emit, fly the rest
  const float tau = vx != 0.f ? (x - bound) / vx : 0.f;
  pos.x = fmaf(-vel.x, tau, pos.x); pos.y = fmaf(-vel.y, tau, pos.y); pos.z = fmaf(-vel.z, tau, pos.z);
  float3 n_in = make_float3(0.f, 0.f, 0.f);
  const float s = (face & 1) ? -1.f : 1.f;
  if (axis == 0) { pos.x = bound; n_in.x = s; }
  else if (axis == 1) { pos.y = bound; n_in.y = s; }
  else { pos.z = bound; n_in.z = s; }
  vel = diffuse_emit(n_in, p.face_vstd[face], rng);
  pos.x = fmaf(vel.x, tau, pos.x); pos.y = fmaf(vel.y, tau, pos.y); pos.z = fmaf(vel.z, tau, pos.z);
  return true;
}

__device__ __forceinline__ bool face_bc(const StepParams& p, float3& pos, float3& vel,
                                        PhiloxStream& rng) {
  const GridGeom& g = p.grid;
  if (!face_axis(p, pos.x, vel.x, g.gmin.x, g.gmax.x, 0, pos, vel, 0, rng)) return false;
  if (!face_axis(p, pos.y, vel.y, g.gmin.y, g.gmax.y, 2, pos, vel, 1, rng)) return false;
  if (!face_axis(p, pos.z, vel.z, g.gmin.z, g.gmax.z, 4, pos, vel, 2, rng)) return false;
  // a re-emitted particle that crossed another face in the rest of its
  // flight is kept inside
  pos.x = fminf(fmaxf(pos.x, g.gmin.x), g.gmax.x);
  pos.y = fminf(fmaxf(pos.y, g.gmin.y), g.gmax.y);
  pos.z = fminf(fmaxf(pos.z, g.gmin.z), g.gmax.z);
  return true;
}

// Whether the box spanned by a path from a to b overlaps the grid's box.
__device__ __forceinline__ bool path_box_meets_grid(const GridGeom& g, float3 a, float3 b) {
  return fminf(a.x, b.x) <= g.gmax.x && fmaxf(a.x, b.x) >= g.gmin.x &&
         fminf(a.y, b.y) <= g.gmax.y && fmaxf(a.y, b.y) >= g.gmin.y &&
         fminf(a.z, b.z) <= g.gmax.z && fmaxf(a.z, b.z) >= g.gmin.z;
}

// Whether this step's flight from pos may reach the body: the path is at
// least the start cell's clearance (nearest mode) or starts or ends in a
// geometry cell holding triangles (first-hit mode); a start outside the
// geometry grid counts when the path's box overlaps the grid's box.  Only
// decides which pass of the cell kernel flies the particle, never the result.
__device__ __forceinline__ bool flight_may_meet_body(const StepParams& p, float3 pos, float3 vel) {
  const GeomView& G = p.geom;
  const float3 e = make_float3(pos.x + vel.x * p.dt, pos.y + vel.y * p.dt, pos.z + vel.z * p.dt);
  if (G.nearest) {
    const uint32_t cc = coll_cell_id(G.cgrid, pos);
    if (cc != kNone) {
      const float dist = length3(make_float3(e.x - pos.x, e.y - pos.y, e.z - pos.z));
      return !(dist < geo_ld(&G.clear[cc]));
    }
    return path_box_meets_grid(G.grid, pos, e);
  }
  const uint32_t sc = coll_cell_id(G.grid, pos);
  const uint32_t ec = coll_cell_id(G.grid, e);
  return (sc != kNone && geo_ld(&G.flags[sc]) != 0) || (ec != kNone && geo_ld(&G.flags[ec]) != 0);
}

// The boundaries after the flight: the reference's functors or the per-face
// kinds.
__device__ __forceinline__ bool apply_bc(const StepParams& p, float3& pos, float3& vel,
                                         PhiloxStream& rng) {
  if (p.face_mode == 0) {
    ref_bc(p.periodic, p.grid, pos, vel);
    return true;
  }
  return face_bc(p, pos, vel, rng);
}

// Free flight and boundaries: move_particle_full's arithmetic for a path that
// cannot reach the body (flight_may_meet_body false), or without a body.
__device__ __forceinline__ bool move_free(const StepParams& p, float3& pos, float3& vel,
                                          uint32_t gidx, uint32_t step) {
  pos.x = fmaf(vel.x, p.dt, pos.x);
  pos.y = fmaf(vel.y, p.dt, pos.y);
  pos.z = fmaf(vel.z, p.dt, pos.z);
  // a particle still inside the box crossed no face: every boundary functor
  // leaves it as it is
  const GridGeom& g = p.grid;
  if (pos.x >= g.gmin.x && pos.x <= g.gmax.x && pos.y >= g.gmin.y && pos.y <= g.gmax.y && pos.z >= g.gmin.z &&
      pos.z <= g.gmax.z)
    return true;
  PhiloxStream rng;
  rng.init(p.seed, gidx, step, kPurposeWall);
  return apply_bc(p, pos, vel, rng);
}

// The deferral test of flight_may_meet_body in nearest mode, in two halves so
// that the table lookup can be issued ahead of the decision: the clearance of
// the start position's geometry cell (-1 outside the geometry grid), then the
// decision from it (the same arithmetic as flight_may_meet_body).
__device__ __forceinline__ float defer_lookup(const StepParams& p, float3 pos) {
  const uint32_t cc = coll_cell_id(p.geom.cgrid, pos);
  return cc == kNone ? -1.f : geo_ld(&p.geom.clear[cc]);
}
__device__ __forceinline__ bool defer_decide(const StepParams& p, float3 pos, float3 vel, float clr) {
  const float3 e = make_float3(pos.x + vel.x * p.dt, pos.y + vel.y * p.dt, pos.z + vel.z * p.dt);
  if (clr >= 0.f) {
    const float dist = length3(make_float3(e.x - pos.x, e.y - pos.y, e.z - pos.z));
    return !(dist < clr);
  }
  return path_box_meets_grid(p.geom.grid, pos, e);
}

// One leg of a nearest-mode flight, from old_pos to pos: its length, its
// direction and its nearest wall crossing (t along d, bin entry e, the
// crossed triangle's plane P).
struct NearestLeg {
  float3 d;
  float dist, t;
  uint32_t e;
  float4 P;
};
enum : int {
  kLegFree = 0,    // no wall crossed: the leg ends at pos
  kLegWall = 1,    // a wall crossed from the front
  kLegInside = 2,  // a face crossed from its back side: the particle is inside the body
};

// The leg's length and unit direction; false for a leg of (nearly) zero length.
__device__ __forceinline__ bool leg_path(float3 old_pos, float3 pos, NearestLeg& L) {
  const float3 seg = make_float3(pos.x - old_pos.x, pos.y - old_pos.y, pos.z - old_pos.z);
  L.dist = sqrtf(fmaf(seg.z, seg.z, fmaf(seg.x, seg.x, __fmul_rn(seg.y, seg.y))));
  if (!(L.dist > 1e-12f)) return false;
  const float idist = 1.f / L.dist;
  L.d = make_float3(__fmul_rn(seg.x, idist), __fmul_rn(seg.y, idist), __fmul_rn(seg.z, idist));
  return true;
}

// The leg's nearest wall crossing.  pretested: the clearance test of this
// leg is already done (its answer was that the leg may reach the body).  The
// mesh is closed with outward normals: a face reached from its back side
// holds a particle inside the body (left over from a fill of a cell the body
// covers in part), which is removed.
__device__ __forceinline__ int nearest_leg(const GeomView& G, float3 old_pos, float3 pos, bool pretested,
                                           NearestLeg& L) {
  if (!leg_path(old_pos, pos, L)) return kLegFree;
  if (!pretested) {
    // a path shorter than the start cell's clearance cannot reach the body
    const uint32_t cc = coll_cell_id(G.cgrid, old_pos);
    if (cc != kNone && L.dist < geo_ld(&G.clear[cc])) return kLegFree;
    // a path outside the geometry grid whose box misses the grid's box
    if (cc == kNone && !path_box_meets_grid(G.grid, old_pos, pos)) return kLegFree;
  }
  if (!nearest_wall_hit(G, old_pos, L.d, L.dist, &L.t, &L.e)) return kLegFree;
  L.P = geo_ld(&G.plane[L.e]);
  if (fmaf(L.d.z, L.P.z, fmaf(L.d.x, L.P.x, __fmul_rn(L.d.y, L.P.y))) > 0.f) return kLegInside;
  return kLegWall;
}

// The wall's answer to a front crossing: from the hit point, set off the
// wall by 1e-6 m along the outward normal, the particle flies the rest of the
// leg's length re-emitted (diffuse, at its incoming speed's time) or
// reflected (specular); old_pos becomes the hit point.
__device__ __forceinline__ void wall_response(const GeomView& G, const NearestLeg& L, float3& old_pos,
                                              float3& pos, float3& vel, PhiloxStream& rng) {
  const float3 n = make_float3(L.P.x, L.P.y, L.P.z);
  const float3 hp = make_float3(fmaf(n.x, 1e-6f, fmaf(L.d.x, L.t, old_pos.x)),
                                fmaf(n.y, 1e-6f, fmaf(L.d.y, L.t, old_pos.y)),
                                fmaf(n.z, 1e-6f, fmaf(L.d.z, L.t, old_pos.z)));
  const float rest = L.dist - L.t;
  if (G.diffuse) {
    const float speed = sqrtf(fmaf(vel.z, vel.z, fmaf(vel.x, vel.x, __fmul_rn(vel.y, vel.y))));
    vel = diffuse_emit(n, G.wall_vstd, rng);
    const float tau = speed > 0.f ? rest / speed : 0.f;
    pos = make_float3(fmaf(vel.x, tau, hp.x), fmaf(vel.y, tau, hp.y), fmaf(vel.z, tau, hp.z));
  } else {
    const float vn2 = 2.f * fmaf(vel.z, n.z, fmaf(vel.x, n.x, __fmul_rn(vel.y, n.y)));
    vel = make_float3(fmaf(-vn2, n.x, vel.x), fmaf(-vn2, n.y, vel.y), fmaf(-vn2, n.z, vel.z));
    const float sp = sqrtf(fmaf(vel.z, vel.z, fmaf(vel.x, vel.x, __fmul_rn(vel.y, vel.y))));
    const float3 r = sp > 0.f ? make_float3(vel.x / sp, vel.y / sp, vel.z / sp) : vel;
    pos = make_float3(fmaf(r.x, rest, hp.x), fmaf(r.y, rest, hp.y), fmaf(r.z, rest, hp.z));
  }
  old_pos = hp;
}

// nearest_leg out of line, for legs walked by one lane where the caller
// keeps its registers for other work.
static __device__ __noinline__ int nearest_leg_call(const GeomView& G, float3 old_pos, float3 pos, bool pretested,
                                                    NearestLeg& L) {
  return nearest_leg(G, old_pos, pos, pretested, L);
}

// The legs of a flight with nearest wall crossings, after each re-emission
// the rest of the flight (extension for bodies with diffuse walls).  first:
// the first leg's answer when it is already known (r0 >= 0: its kLeg* code
// and L0 its crossing), else r0 < 0 and the first leg is walked here
// (pretested: its clearance test is done).  Returns false if the particle
// is inside the body.
template <bool CALL>
__device__ __forceinline__ bool nearest_legs(const GeomView& G, float3& old_pos, float3& pos, float3& vel,
                                             PhiloxStream& rng, bool pretested, int r0, const NearestLeg& L0) {
  for (uint32_t b = 0; b < kCollisionLimit; b++) {
    NearestLeg L;
    int r;
    if (b == 0 && r0 >= 0) {
      L = L0;
      r = r0;
    } else if (CALL) {
      r = nearest_leg_call(G, old_pos, pos, pretested && b == 0, L);
    } else {
      r = nearest_leg(G, old_pos, pos, pretested && b == 0, L);
    }
    if (r == kLegFree) break;
    if (r == kLegInside) return false;
    float2 reach = make_float2(0.f, 2.f);
    if (G.reach) reach = geo_ld(&G.reach[L.e]);
    wall_response(G, L, old_pos, pos, vel, rng);
    // a leg within the wall's reach finds no wall (the next pass of the
    // loop would find none and stop); 1e-5 covers the rounding of the sine
    NearestLeg next;
    if (reach.x > 0.f && leg_path(old_pos, pos, next) && next.dist < reach.x &&
        fmaf(next.d.z, L.P.z, fmaf(next.d.x, L.P.x, __fmul_rn(next.d.y, L.P.y))) > reach.y + 1e-5f)
      break;
  }
  return true;
}

// One particle's flight with the body: IntegrateDev / ProcessCollisionsDev,
// kernels/dsmc_kernel.cu:1557-1657.  Returns false if the particle left.
// pretested: the caller already found that the path from pos may reach the
// body (flight_may_meet_body or its halves), so the first clearance test is
// skipped (its answer is known).  Inline in the kernel that flies only such
// flights (k_mesh_w: without a call its state stays in registers); other
// kernels call the out-of-line move_particle_full.
__device__ __forceinline__ bool move_particle_body(const StepParams& p, float3& pos, float3& vel,
                                                   uint32_t gidx, uint32_t step, bool pretested) {
  float3 old_pos = pos;
  pos.x = fmaf(vel.x, p.dt, old_pos.x);
  pos.y = fmaf(vel.y, p.dt, old_pos.y);
  pos.z = fmaf(vel.z, p.dt, old_pos.z);
  PhiloxStream rng;
  rng.init(p.seed, gidx, step, kPurposeWall);
  if (p.has_geom && p.geom.nearest) {
    // nearest wall crossing along the path, repeated for the rest of the
    // flight after each re-emission (extension for bodies with diffuse walls)
    const NearestLeg none{};
    if (!nearest_legs<false>(p.geom, old_pos, pos, vel, rng, pretested, -1, none)) return false;
  } else if (p.has_geom) {
    const GeomView& G = p.geom;
    uint32_t st_cubid = kNone, end_cubid = kNone;
    bool collProcessed = false;
    uint32_t i = 0;
    do {
      st_cubid = coll_cell_id(G.grid, old_pos);
      end_cubid = coll_cell_id(G.grid, pos);
      if (st_cubid != kNone) {
        if (geo_ld(&G.flags[st_cubid]) != 0)
          collProcessed = collide_with_geometry(G, &pos, &vel, &old_pos, st_cubid, &rng);
      }
      if (!collProcessed && st_cubid != end_cubid && end_cubid != kNone) {
        if (geo_ld(&G.flags[end_cubid]) != 0)
          collProcessed = collide_with_geometry(G, &pos, &vel, &old_pos, end_cubid, &rng);
      }
    } while (collProcessed && i++ < kCollisionLimit);
  }
  return apply_bc(p, pos, vel, rng);
}

// Out of line: only flights that may reach the body come here in the step.
static __device__ __noinline__ bool move_particle_full(const StepParams& p, float3& pos,
                                                       float3& vel, uint32_t gidx, uint32_t step,
                                                       bool pretested) {
  return move_particle_body(p, pos, vel, gidx, step, pretested);
}

// One particle's flight (free flight inline, with a body out of line).
__device__ __forceinline__ bool move_particle(const StepParams& p, float3& pos, float3& vel,
                                              uint32_t gidx, uint32_t step,
                                              bool pretested = false) {
  if (!p.has_geom) return move_free(p, pos, vel, gidx, step);
  float3 tp = pos, tv = vel;
  const bool live = move_particle_full(p, tp, tv, gidx, step, pretested);
  pos = tp;
  vel = tv;
  return live;
}

// Sampling of one cell from sorted velocities (SampleCellStatisticsDev,
// kernels/dsmc_kernel.cu:856-890) into the FP64 accumulators (SoA, 5 fields).
template <class Acc>
__device__ __forceinline__ void sample_cell(double* acc, uint32_t cells, uint32_t cell, int n,
                                            const Acc& a) {
  if (n <= 0) return;
  double su = 0, sv = 0, sw = 0, se = 0;
  for (int k = 0; k < n; k++) {
    const float3 q = a.get(k);
    const double x = q.x, y = q.y, z = q.z;
    su += x; sv += y; sw += z;
    se += x * x + y * y + z * z;
  }
  acc[cell] += (double)n;
  acc[(size_t)cells + cell] += su;
  acc[2 * (size_t)cells + cell] += sv;
  acc[3 * (size_t)cells + cell] += sw;
  acc[4 * (size_t)cells + cell] += se;
}

}  // namespace dev
}  // namespace dsmcb
