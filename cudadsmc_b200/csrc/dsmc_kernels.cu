// Kernels of the DSMC timestep other than the fused cell kernel (sm_100a):
// the cell-start scan, the scatter into sorted order, the initial keys, the
// stage kernels, the initial fill and the inflow injection.
//
// Memory plan per particle and step (SoA FP32 state, 24 B):
//   scatter: read key 4 B + state 24 B, write state 24 B + orig 4 B
//   cell:    read state 24 B + orig 4 B, write state 24 B + key 4 B
// Per-cell arrays (counts, starts, (sigma*g)max/remainder, RNG state) add a
// few bytes per particle.  All particle traffic is coalesced except the
// scatter's writes, which land near-sorted because most particles stay in or
// next to their cell between steps.
#include <algorithm>

#include "dsmc_step_dev.cuh"

namespace dsmcb {
namespace {

using namespace dev;

// Move stage: free flight and boundaries for n particles in place.
__global__ void __launch_bounds__(256) k_move(const __grid_constant__ StepParams p, uint32_t n, uint32_t step) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float3 pos = make_float3(p.out.x[i], p.out.y[i], p.out.z[i]);
    float3 vel = make_float3(p.out.u[i], p.out.v[i], p.out.w[i]);
    const bool live = move_particle(p, pos, vel, i, step);
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

// Keys and counts of a freshly uploaded state (particles outside the box are
// dead when the faces are in use).
__global__ void k_index(GridGeom g, const float* __restrict__ x, const float* __restrict__ y,
                        const float* __restrict__ z, uint32_t n, uint32_t* __restrict__ keys,
                        uint32_t* count, uint32_t* tile_sum, uint32_t n_scan_tiles, int face_mode) {
  extern __shared__ uint32_t s_tile[];
  for (uint32_t t = threadIdx.x; t < n_scan_tiles; t += blockDim.x) s_tile[t] = 0;
  __syncthreads();
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    const bool active = i < n;
    bool live = false;
    uint32_t key = kDeadKey;
    if (active) {
      const float px = x[i], py = y[i], pz = z[i];
      live = !(face_mode != 0 && (px < g.gmin.x || px > g.gmax.x || py < g.gmin.y ||
                                   py > g.gmax.y || pz < g.gmin.z || pz > g.gmax.z));
      if (live) key = cell_id3d(g, px, py, pz);
      keys[i] = key;
    }
    const unsigned m = __ballot_sync(kFull, active && live);
    if (active && live) warp_count_key(count, key, m, s_tile);
  }
  __syncthreads();
  flush_tile_hist(s_tile, tile_sum, n_scan_tiles);
}

// Exclusive scan of per-cell counts.  Block b owns cells [b*2048, (b+1)*2048);
// its offset is the sum of the per-tile totals before it, which the producer
// kernels accumulated alongside the counts.  Resets the counts and the
// scatter's cursors.
__device__ __forceinline__ void scan_body(uint32_t* count, uint32_t* cursor, uint32_t* start,
                                          uint32_t cells, const uint32_t* tile_sum, Meta* meta, int bump,
                                          const uint32_t vb, const uint32_t vg) {
  __shared__ uint32_t s_warp[8], s_part[8];
  const uint32_t b = vb;
  // the block's counts and the totals of the tiles before it, loaded together
  const uint32_t c0 = b * kScanTile + threadIdx.x * 8;
  // 8 whole counts, read and written 16 bytes at a time where the arrays
  // allow it (the stage API's workspace may be only 4-byte aligned)
  const bool vec = (((uintptr_t)count | (uintptr_t)start | (uintptr_t)cursor) & 15u) == 0;
  const bool whole = vec && c0 + 8u <= cells;
  uint32_t v[8];
  if (whole) {
    const uint4 lo = *reinterpret_cast<const uint4*>(count + c0);
    const uint4 hi = *reinterpret_cast<const uint4*>(count + c0 + 4);
    v[0] = lo.x; v[1] = lo.y; v[2] = lo.z; v[3] = lo.w;
    v[4] = hi.x; v[5] = hi.y; v[6] = hi.z; v[7] = hi.w;
  } else {
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = (c0 + i < cells) ? count[c0 + i] : 0u;
  }
  uint32_t part = 0;
  for (uint32_t t = threadIdx.x; t < b; t += blockDim.x) part += tile_sum[t];
  part = warp_sum(part);
  uint32_t tsum = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) tsum += v[i];
  uint32_t incl = tsum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(kFull, incl, o);
    if ((int)lane_id() >= o) incl += t;
  }
  if (lane_id() == 31) s_warp[threadIdx.x / 32] = incl;
  if (lane_id() == 0) s_part[threadIdx.x / 32] = part;
  __syncthreads();
  uint32_t run = incl - tsum;
#pragma unroll
  for (uint32_t w = 0; w < 8; w++) {
    run += s_part[w];
    if (w < threadIdx.x / 32) run += s_warp[w];
  }
  uint32_t st[8];
#pragma unroll
  for (int i = 0; i < 8; i++) {
    st[i] = run;
    run += v[i];
  }
  if (whole) {
    *reinterpret_cast<uint4*>(start + c0) = make_uint4(st[0], st[1], st[2], st[3]);
    *reinterpret_cast<uint4*>(start + c0 + 4) = make_uint4(st[4], st[5], st[6], st[7]);
    const uint4 z = make_uint4(0u, 0u, 0u, 0u);
    *reinterpret_cast<uint4*>(count + c0) = z;
    *reinterpret_cast<uint4*>(count + c0 + 4) = z;
    if (cursor) {
      *reinterpret_cast<uint4*>(cursor + c0) = z;
      *reinterpret_cast<uint4*>(cursor + c0 + 4) = z;
    }
  } else {
#pragma unroll
    for (int i = 0; i < 8; i++) {
      if (c0 + i < cells) {
        start[c0 + i] = st[i];
        count[c0 + i] = 0u;
        if (cursor) cursor[c0 + i] = 0u;
      }
    }
  }
  if (b == vg - 1 && threadIdx.x == blockDim.x - 1) {
    start[cells] = run;
    meta->n_scatter = meta->n_alive + meta->n_pending;
    meta->n_pending = 0;
    meta->n_alive = run;
    meta->tile_next = 0;
    meta->tile_next2 = 0;
    meta->n_defer = 0;
    meta->n_light = 0;
    meta->n_heavy = 0;
    if (bump) {
      meta->step += 1;
      meta->particle_steps += run;
    }
  }
}

__global__ void __launch_bounds__(256) k_scan(uint32_t* count, uint32_t* cursor, uint32_t* start,
                                              uint32_t cells, const uint32_t* tile_sum, Meta* meta,
                                              int bump) {
  chained_entry();
  scan_body(count, cursor, start, cells, tile_sum, meta, bump, blockIdx.x, gridDim.x);
}
__global__ void __launch_bounds__(256) k_scan_b(const __grid_constant__ BatchOf<SortArgs> bv) {
  chained_entry();
  uint32_t vb, vg;
  const SortArgs& a = bv.locate(vb, vg);
  scan_body(a.count, a.cursor, a.start, a.cells, a.tile_sum, a.meta, 1, vb, vg);
}

// Scatter into sorted order: dst[start[key] + ticket] = src[i], orig = i.  The
// tickets come from per-cell cursors (one atomic per distinct key per group of
// 32).  Each warp takes kScatterU groups of 32 consecutive particles at once,
// so that their chains of key load -> ticket atomic -> stores overlap.  With
// STATE false only orig is written: one scattered 4-byte store per particle
// instead of seven (scattered stores, not the loads or the atomics, bound this
// kernel), and the split cell kernels gather the state through orig.
constexpr int kScatterU = 4;

template <bool STATE>
__device__ __forceinline__ void scatter_body(SoA src, SoA dst, const uint32_t* __restrict__ keys,
                                             const uint32_t* __restrict__ start, uint32_t* cursor,
                                             uint32_t* __restrict__ orig, uint32_t cells,
                                             uint32_t* tile_sum, uint32_t n_scan_tiles, Meta* meta,
                                             uint32_t capacity, const uint32_t vb, const uint32_t vg) {
  if (vb == 0)
    for (uint32_t t = threadIdx.x; t < n_scan_tiles; t += blockDim.x) tile_sum[t] = 0;
  const uint32_t n = meta->n_scatter;
  const uint32_t lane = lane_id();
  const uint32_t gw = (vb * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (vg * blockDim.x) >> 5;
  constexpr int U = kScatterU;
  const uint32_t stride = nw * 32u * U;
  // keys of the next iteration load while this one's tickets are in flight
  uint32_t nkey[U];
#pragma unroll
  for (int k = 0; k < U; k++) {
    const uint32_t i = gw * 32u * U + 32u * k + lane;
    nkey[k] = i < n ? __ldcs(&keys[i]) : kDeadKey;
  }
  for (uint32_t base = gw * 32u * U; base < n; base += stride) {
    uint32_t key[U];
    float x[U], y[U], z[U], u[U], v[U], w[U];
#pragma unroll
    for (int k = 0; k < U; k++) {
      key[k] = nkey[k];
      const uint32_t i2 = base + stride + 32u * k + lane;
      nkey[k] = i2 < n ? __ldcs(&keys[i2]) : kDeadKey;
    }
#pragma unroll
    for (int k = 0; k < U; k++) {
      const uint32_t i = base + 32u * k + lane;
      x[k] = y[k] = z[k] = u[k] = v[k] = w[k] = 0.f;
      if (STATE && i < n) {
        x[k] = src.x[i]; y[k] = src.y[i]; z[k] = src.z[i];
        u[k] = src.u[i]; v[k] = src.v[i]; w[k] = src.w[i];
      }
    }
    // the ticket atomics of all groups first, then their broadcasts
    unsigned msk[U], peers[U];
    uint32_t st[U], got[U];
#pragma unroll
    for (int k = 0; k < U; k++) {
      const uint32_t i = base + 32u * k + lane;
      const bool live = key[k] < cells;
      if (i < n && key[k] != kDeadKey && !live) atomicOr(&meta->error, kErrKeyRange);
      msk[k] = __ballot_sync(kFull, live);
      st[k] = 0;
      got[k] = 0;
      peers[k] = 0;
      if (live) {
        st[k] = __ldg(&start[key[k]]);
        peers[k] = __match_any_sync(msk[k], key[k]);
        if ((int)lane == __ffs(peers[k]) - 1) got[k] = atomicAdd(&cursor[key[k]], (uint32_t)__popc(peers[k]));
      }
    }
#pragma unroll
    for (int k = 0; k < U; k++) {
      if (!(key[k] < cells)) continue;
      const uint32_t i = base + 32u * k + lane;
      const uint32_t t = __shfl_sync(msk[k], got[k], __ffs(peers[k]) - 1) +
                         __popc(peers[k] & ((1u << lane) - 1u));
      const uint32_t d = st[k] + t;
      if (d >= capacity) {
        atomicOr(&meta->error, kErrKeyRange);
        continue;
      }
      if (STATE) {
        dst.x[d] = x[k]; dst.y[d] = y[k]; dst.z[d] = z[k];
        dst.u[d] = u[k]; dst.v[d] = v[k]; dst.w[d] = w[k];
      }
      orig[d] = i;
    }
  }
}

template <bool STATE>
__global__ void __launch_bounds__(256, 4) k_scatter(SoA src, SoA dst, const uint32_t* __restrict__ keys,
                                                    const uint32_t* __restrict__ start,
                                                    uint32_t* cursor, uint32_t* __restrict__ orig,
                                                    uint32_t cells, uint32_t* tile_sum,
                                                    uint32_t n_scan_tiles, Meta* meta,
                                                    uint32_t capacity) {
  chained_entry();
  scatter_body<STATE>(src, dst, keys, start, cursor, orig, cells, tile_sum, n_scan_tiles, meta, capacity,
                      blockIdx.x, gridDim.x);
}
// orig only (the split kernels)
__global__ void __launch_bounds__(256, 4) k_scatter_b(const __grid_constant__ BatchOf<SortArgs> bv) {
  chained_entry();
  uint32_t vb, vg;
  const SortArgs& a = bv.locate(vb, vg);
  const SoA none{nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  scatter_body<false>(none, none, a.keys, a.start, a.cursor, a.orig, a.cells, a.tile_sum, a.n_scan_tiles,
                      a.meta, a.capacity, vb, vg);
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
    const uint32_t i = base + threadIdx.x;
    const uint32_t key = i < n ? keys[i] : kNone;
    const bool active = i < n && key < nkeys;
    const unsigned m = __ballot_sync(kFull, active);
    if (active) {
      const uint32_t t = warp_ticket(count, key, m);
      ticket[i] = t;
      const unsigned peers = __match_any_sync(m, key);
      if ((int)lane_id() == __ffs(peers) - 1) atomicAdd(&s_tile[key >> kScanShift], (uint32_t)__popc(peers));
    }
  }
  __syncthreads();
  flush_tile_hist(s_tile, tile_sum, n_scan_tiles);
}

__global__ void k_scatter_kv(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                             const uint32_t* __restrict__ ticket,
                             const uint32_t* __restrict__ start, uint32_t n, uint32_t nkeys,
                             uint32_t* __restrict__ tmp_val, uint32_t* __restrict__ tmp_pos) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t key = keys[i];
    if (key >= nkeys) continue;
    const uint32_t d = start[key] + ticket[i];
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
      const uint32_t c = cur + 1 + threadIdx.x;
      const int fits = (c <= nct) && (ls[c] - base <= (uint32_t)kCap);
      const uint32_t k = __syncthreads_count(fits);
      if (k == 0) {
        // one key with more than kCap entries: rank from global memory
        const uint32_t s0 = base, e0 = ls[cur + 1];
        for (uint32_t i = s0 + threadIdx.x; i < e0; i += blockDim.x) {
          const uint32_t my = tmp_pos[i];
          uint32_t rank = 0;
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
          const uint32_t mid = (lo + hi + 1) >> 1;
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
    const uint32_t h = keys[i];
    const uint32_t hp = i > 0 ? keys[i - 1] : kNone;
    if (i == 0 || h != hp) {
      if (h < ncells) cse[h].x = i;
      if (i > 0 && hp < ncells) cse[hp].y = i;
    }
    if (i == n - 1 && h < ncells) cse[h].y = i + 1;
    if (gather) {
      const uint32_t s = idx[i];
      dst.x[i] = src.x[s]; dst.y[i] = src.y[s]; dst.z[i] = src.z[s];
      dst.u[i] = src.u[s]; dst.v[i] = src.v[s]; dst.w[i] = src.w[s];
    }
  }
}

// Stand-alone FP64 sampling, one thread per cell.
__global__ void k_sample_cells(const float* __restrict__ u, const float* __restrict__ v,
                               const float* __restrict__ w, const uint32_t* __restrict__ start,
                               uint32_t cells, double* acc, size_t fs, size_t cs) {
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < cells; c += gridDim.x * blockDim.x) {
    const uint32_t s = start[c], e = start[c + 1];
    if (e <= s) continue;
    double su = 0, sv = 0, sw = 0, se = 0;
    for (uint32_t i = s; i < e; i++) {
      const double x = u[i], y = v[i], z = w[i];
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

// Per-cell fields (n, ux, uy, uz, T), cell-major, from the FP64 sampling sums
// (5 x cells, SoA) of ns passes: ProcessAndOutputStatistics' arithmetic
// (kernels/dsmc_base.cu:104-163) in double with every rounding step explicit,
// the same steps as the host code; with fields == 0 the sums themselves,
// transposed to cell-major.
__global__ void k_cell_fields(const double* __restrict__ acc, uint32_t cells, double fnum,
                              double cell_volume, uint32_t ns, double mass, int fields,
                              double* __restrict__ out) {
  const double k3 = 3.0 * 1.3806e-23;
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < cells; c += gridDim.x * blockDim.x) {
    const double N = acc[c], a1 = acc[(size_t)cells + c], a2 = acc[2 * (size_t)cells + c],
                 a3 = acc[3 * (size_t)cells + c], a4 = acc[4 * (size_t)cells + c];
    double* o = out + 5 * (size_t)c;
    if (!fields) {
      o[0] = N; o[1] = a1; o[2] = a2; o[3] = a3; o[4] = a4;
      continue;
    }
    o[0] = ns ? __ddiv_rn(__dmul_rn(fnum, N), __dmul_rn(cell_volume, (double)ns)) : 0.0;
    if (N > 0) {
      const double ux = __ddiv_rn(a1, N), uy = __ddiv_rn(a2, N), uz = __ddiv_rn(a3, N);
      const double u2 = __dadd_rn(__dadd_rn(__dmul_rn(ux, ux), __dmul_rn(uy, uy)), __dmul_rn(uz, uz));
      o[1] = ux; o[2] = uy; o[3] = uz;
      o[4] = __ddiv_rn(__dmul_rn(mass, __dsub_rn(__ddiv_rn(a4, N), u2)), k3);
    } else {
      o[1] = o[2] = o[3] = o[4] = 0.0;
    }
  }
}

// ------------------------------------------------------------ init fill ----

// Initial population: part_per_cell particles per cell at uniform positions
// (GetRandomPosition, kernels/dsmc_kernel.cu:417-427) with either the
// reference's speed/angle sampler (GetRandomVelocity, :394-415) or an exact
// Maxwellian.  Random numbers come from Philox (the reference used its
// Mersenne-Twister table, which is not reproduced).
__global__ void k_init_fill(const __grid_constant__ InitParams p) {
  const uint32_t total = p.cells * p.ppc;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const uint32_t cell = i / p.ppc, k = i - cell * p.ppc;
    const uint32_t dst0 = p.cell_slot[cell];
    if (dst0 == kNone || k >= p.cell_count[cell]) continue;
    const uint32_t d = dst0 + k;
    const uint32_t cx = cell % p.grid.dim.x;
    const uint32_t cy = (cell / p.grid.dim.x) % p.grid.dim.y;
    const uint32_t cz = cell / (p.grid.dim.x * p.grid.dim.y);
    PhiloxStream r;
    r.init(p.seed, i, 0u, kPurposeInit);
    float3 vel;
    if (p.kind == 0) {
      const float vv = p.vmp * sqrtf(-logf(r.uniform()));
      const float tetha = 2.0f * kPiF;
      vel.x = vv * sinf(r.uniform() * tetha) + p.stream.x;
      vel.y = vv * sinf(r.uniform() * tetha) + p.stream.y;
      vel.z = vv * sinf(r.uniform() * tetha) + p.stream.z;
    } else {
      float sd = (p.kind == 2 && (i & 1u)) ? p.vstd2 : p.vstd;
      float3 drift = p.stream;
      if (p.cell_state) {
        const float4 cs = p.cell_state[cell];
        drift = make_float3(cs.x, cs.y, cs.z);
        sd = cs.w;
        // a two-stream cell: a share of its particles from the free stream
        if (p.cell_mix && r.uniform() < p.cell_mix[cell]) {
          drift = p.stream;
          sd = p.vstd;
        }
      }
      const float r1 = r.uniform(), r2 = r.uniform(), r3 = r.uniform(), r4 = r.uniform();
      const float m1 = sd * sqrtf(-2.f * logf(r1)), m2 = sd * sqrtf(-2.f * logf(r3));
      float s1, c1, s2, c2;
      sincospif(2.0f * r2, &s1, &c1);
      sincospif(2.0f * r4, &s2, &c2);
      vel = make_float3(m1 * c1 + drift.x, m1 * s1 + drift.y, m2 * c2 + drift.z);
    }
    const float3 cellmin = make_float3(p.grid.gmin.x + cx * p.grid.cell.x,
                                       p.grid.gmin.y + cy * p.grid.cell.y,
                                       p.grid.gmin.z + cz * p.grid.cell.z);
    float px = cellmin.x + r.uniform() * p.grid.cell.x;
    float py = cellmin.y + r.uniform() * p.grid.cell.y;
    float pz = cellmin.z + r.uniform() * p.grid.cell.z;
    // a cell the mesh covers in part: positions inside the body are drawn
    // again (at most 64 times), then the cell's known outside point is used
    if (p.reject_inside) {
      bool in = inside_mesh(p.geom, make_float3(px, py, pz));
      for (int tries = 0; tries < 64 && in; tries++) {
        px = cellmin.x + r.uniform() * p.grid.cell.x;
        py = cellmin.y + r.uniform() * p.grid.cell.y;
        pz = cellmin.z + r.uniform() * p.grid.cell.z;
        in = inside_mesh(p.geom, make_float3(px, py, pz));
      }
      if (in && p.cell_point && p.cell_point[cell].w > 0.f) {
        const float4 q = p.cell_point[cell];
        px = q.x; py = q.y; pz = q.z;
      }
    }
    p.out.x[d] = px; p.out.y[d] = py; p.out.z[d] = pz;
    p.out.u[d] = vel.x; p.out.v[d] = vel.y; p.out.w[d] = vel.z;
  }
}


// --------------------------------------------------------------- inflow ----

// Plan: number of particles the face injects this step (carrying the
// fractional remainder), reserved after the particles already in the array.
__device__ __forceinline__ void inject_plan_body(const InjectParams& p, uint32_t* plan, const uint32_t vb) {
  if (threadIdx.x != 0 || vb != 0) return;
  const float want = fmaf(__fmul_rn(p.inflow.number_flux, p.inflow.area), p.dt, *p.remainder);
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

__global__ void k_inject_plan(const __grid_constant__ InjectParams p, uint32_t* plan) {
  chained_entry();
  inject_plan_body(p, plan, blockIdx.x);
}
__global__ void k_inject_plan_b(const __grid_constant__ BatchOf<InjectParams> bv) {
  chained_entry();
  uint32_t vb, vg;
  const InjectParams& p = bv.locate(vb, vg);
  inject_plan_body(p, p.plan, vb);
}

// Inward normal speed of the drifting Maxwellian weighted by flux,
// f(z) ~ z exp(-(z - s)^2) for z = v_n / c_mp > 0, by rejection from the
// envelope (|y| + max(s,0)) exp(-y^2), y = z - s.  Rounding steps explicit
// (no contraction).
__device__ __forceinline__ float sample_flux_normal(float s, PhiloxStream& r) {
  const float sp = fmaxf(s, 0.f);
  const float w_abs = 1.f / fmaf(sp, 1.7724539f, 1.f);
  for (int it = 0; it < 64; it++) {
    float y;
    if (r.uniform() < w_abs) {
      y = sqrtf(-logf(r.uniform()));
      if (r.uniform() < 0.5f) y = -y;
    } else {
      const float a = r.uniform(), b = r.uniform();
      y = __fmul_rn(sqrtf(-logf(a)), cospif(2.0f * b));  // N(0, 1/2)
    }
    const float z = s + y;
    if (z <= 0.f) continue;
    if (r.uniform() * (fabsf(y) + sp) <= z) return z;
  }
  return fmaxf(s, 1e-3f);
}

__device__ __forceinline__ float& comp(float3& a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }
__device__ __forceinline__ float compc(const float3& a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }

__device__ __forceinline__ void inject_fill_body(const InjectParams& p, const uint32_t* plan,
                                                 const uint32_t vb, const uint32_t vg) {
  extern __shared__ uint32_t s_tile[];
  const uint32_t step = p.meta->step;
  for (uint32_t t = threadIdx.x; t < p.n_scan_tiles; t += blockDim.x) s_tile[t] = 0;
  __syncthreads();
  const uint32_t first = plan[0], k = plan[1];
  const int face = p.inflow.face;
  const int ax = face >> 1;
  const float sign = (face & 1) ? -1.f : 1.f;  // inward normal along +axis for the low face
  const GridGeom& g = p.grid;
  const float cmp = p.inflow.vstd * 1.41421356f;
  const float s = sign * compc(p.inflow.stream, ax) / cmp;
  for (uint32_t base = vb * blockDim.x; base < k; base += vg * blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    const bool active = i < k;
    bool live = false;
    uint32_t key = kDeadKey;
    if (active) {
      float3 pos = make_float3(0, 0, 0), vel = pos;
      PhiloxStream r;
      r.init(p.seed, i, step, kPurposeInject + (uint32_t)face);
      const float vn = __fmul_rn(__fmul_rn(sample_flux_normal(s, r), cmp), sign);
      const float a1 = r.uniform(), a2 = r.uniform();
      const float rad = __fmul_rn(p.inflow.vstd, sqrtf(__fmul_rn(-2.f, logf(a1))));
      float sn, cs;
      sincospif(2.0f * a2, &sn, &cs);
      const int a_t1 = (ax + 1) % 3, a_t2 = (ax + 2) % 3;
      comp(vel, ax) = vn;
      comp(vel, a_t1) = fmaf(rad, cs, compc(p.inflow.stream, a_t1));
      comp(vel, a_t2) = fmaf(rad, sn, compc(p.inflow.stream, a_t2));
      comp(pos, ax) = (face & 1) ? compc(g.gmax, ax) : compc(g.gmin, ax);
      comp(pos, a_t1) = fmaf(r.uniform(), compc(g.gmax, a_t1) - compc(g.gmin, a_t1), compc(g.gmin, a_t1));
      comp(pos, a_t2) = fmaf(r.uniform(), compc(g.gmax, a_t2) - compc(g.gmin, a_t2), compc(g.gmin, a_t2));
      const float frac = __fmul_rn(r.uniform(), p.dt);
      pos.x = fmaf(vel.x, frac, pos.x); pos.y = fmaf(vel.y, frac, pos.y); pos.z = fmaf(vel.z, frac, pos.z);
      live = !(pos.x < g.gmin.x || pos.x > g.gmax.x || pos.y < g.gmin.y || pos.y > g.gmax.y ||
               pos.z < g.gmin.z || pos.z > g.gmax.z);
      if (live) key = cell_id3d(g, pos.x, pos.y, pos.z);
      const uint32_t d = first + i;
      p.st.x[d] = pos.x; p.st.y[d] = pos.y; p.st.z[d] = pos.z;
      p.st.u[d] = vel.x; p.st.v[d] = vel.y; p.st.w[d] = vel.z;
      p.keys[d] = key;
    }
    const unsigned m = __ballot_sync(kFull, active && live);
    if (active && live) warp_count_key(p.count, key, m, s_tile);
  }
  __syncthreads();
  flush_tile_hist(s_tile, p.tile_sum, p.n_scan_tiles);
}

__global__ void k_inject_fill(const __grid_constant__ InjectParams p, const uint32_t* plan) {
  chained_entry();
  inject_fill_body(p, plan, blockIdx.x, gridDim.x);
}
__global__ void k_inject_fill_b(const __grid_constant__ BatchOf<InjectParams> bv) {
  chained_entry();
  uint32_t vb, vg;
  const InjectParams& p = bv.locate(vb, vg);
  inject_fill_body(p, p.plan, vb, vg);
}

}  // namespace

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
  const uint64_t cap = (uint64_t)num_sms() * per_sm;
  if (need < 1) need = 1;
  return (uint32_t)(need < cap ? need : cap);
}

cudaError_t launch_index(const GridGeom& g, uint32_t cells, const float* x, const float* y,
                         const float* z, uint32_t n, uint32_t* keys, uint32_t* count,
                         uint32_t* tile_sum, uint32_t n_scan_tiles, int face_mode,
                         cudaStream_t stream) {
  (void)cells;
  const uint32_t grid = grid_for(n, 256, 8);
  k_index<<<grid, 256, n_scan_tiles * 4, stream>>>(g, x, y, z, n, keys, count, tile_sum,
                                                   n_scan_tiles, face_mode);
  return cudaGetLastError();
}

cudaError_t launch_scan(uint32_t* count, uint32_t* cursor, uint32_t* start, uint32_t cells,
                        const uint32_t* tile_sum, uint32_t n_scan_tiles, Meta* meta, int bump_step,
                        cudaStream_t stream) {
  return launch_chained(k_scan, n_scan_tiles, 256, 0, stream, true, count, cursor, start, cells, tile_sum, meta,
                        bump_step);
}

cudaError_t launch_scatter(bool with_state, const SoA& src, SoA dst, const uint32_t* keys,
                           const uint32_t* start,
                           uint32_t* cursor, uint32_t* orig, uint32_t cells, uint32_t* tile_sum,
                           uint32_t n_scan_tiles, Meta* meta, uint32_t capacity,
                           cudaStream_t stream) {
  const uint32_t grid = (uint32_t)num_sms() * 4;
  return launch_chained(with_state ? k_scatter<true> : k_scatter<false>, grid, 256, 0, stream, true, src, dst, keys,
                        start, cursor, orig, cells, tile_sum, n_scan_tiles, meta, capacity);
}

cudaError_t launch_move(const StepParams& p, uint32_t n, uint32_t step, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  const uint32_t grid = grid_for(n, 256, 8);
  k_move<<<grid, 256, 0, stream>>>(p, n, step);
  return cudaGetLastError();
}

cudaError_t launch_cell_ids(const GridGeom& g, const float* x, const float* y, const float* z,
                            uint32_t n, uint32_t* keys, uint32_t* idx, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  const uint32_t grid = grid_for(n, 256, 8);
  k_cell_ids<<<grid, 256, 0, stream>>>(g, x, y, z, n, keys, idx);
  return cudaGetLastError();
}

cudaError_t launch_count_keys(const uint32_t* keys, uint32_t n, uint32_t nkeys, uint32_t* ticket,
                              uint32_t* count, uint32_t* tile_sum, uint32_t n_scan_tiles,
                              cudaStream_t stream) {
  const uint32_t grid = grid_for(n, 256, 8);
  k_count_keys<<<grid, 256, n_scan_tiles * 4, stream>>>(keys, n, nkeys, ticket, count, tile_sum,
                                                        n_scan_tiles);
  return cudaGetLastError();
}

cudaError_t launch_scatter_kv(const uint32_t* keys, const uint32_t* vals, const uint32_t* ticket,
                              const uint32_t* start, uint32_t n, uint32_t nkeys, uint32_t* tmp_val,
                              uint32_t* tmp_pos, cudaStream_t stream) {
  const uint32_t grid = grid_for(n, 256, 8);
  k_scatter_kv<<<grid, 256, 0, stream>>>(keys, vals, ticket, start, n, nkeys, tmp_val, tmp_pos);
  return cudaGetLastError();
}

cudaError_t launch_segment_fixup(const uint32_t* start, uint32_t nkeys, const uint32_t* tmp_val,
                                 const uint32_t* tmp_pos, uint32_t* keys_out, uint32_t* vals_out,
                                 cudaStream_t stream) {
  const uint32_t ntiles = (nkeys + 255) / 256;
  const uint32_t grid = ntiles < (uint32_t)num_sms() * 4 ? ntiles : (uint32_t)num_sms() * 4;
  if (grid == 0) return cudaSuccess;
  k_segment_fixup<<<grid, 256, 0, stream>>>(start, nkeys, tmp_val, tmp_pos, keys_out, vals_out);
  return cudaGetLastError();
}

cudaError_t launch_bounds_reorder(const uint32_t* keys, const uint32_t* idx, uint32_t n,
                                  uint32_t ncells, uint32_t* cse, const float* const src[6],
                                  float* const dst[6], cudaStream_t stream) {
  SoA s{const_cast<float*>(src ? src[0] : nullptr), const_cast<float*>(src ? src[1] : nullptr),
        const_cast<float*>(src ? src[2] : nullptr), const_cast<float*>(src ? src[3] : nullptr),
        const_cast<float*>(src ? src[4] : nullptr), const_cast<float*>(src ? src[5] : nullptr)};
  SoA d{dst ? dst[0] : nullptr, dst ? dst[1] : nullptr, dst ? dst[2] : nullptr,
        dst ? dst[3] : nullptr, dst ? dst[4] : nullptr, dst ? dst[5] : nullptr};
  const uint32_t grid = grid_for(n, 256, 8);
  k_bounds_reorder<<<grid, 256, 0, stream>>>(keys, idx, n, ncells, (uint2*)cse, s, d,
                                             (src && dst) ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_cell_fields(const double* acc, uint32_t cells, double fnum, double cell_volume,
                               uint32_t ns, double mass, int fields, double* out, cudaStream_t stream) {
  k_cell_fields<<<grid_for(cells, 256, 8), 256, 0, stream>>>(acc, cells, fnum, cell_volume, ns, mass,
                                                            fields, out);
  return cudaGetLastError();
}

cudaError_t launch_sample_cells(const float* u, const float* v, const float* w,
                                const uint32_t* start, uint32_t cells, double* acc,
                                size_t fstride, size_t cstride, cudaStream_t stream) {
  const uint32_t grid = grid_for(cells, 256, 8);
  k_sample_cells<<<grid, 256, 0, stream>>>(u, v, w, start, cells, acc, fstride, cstride);
  return cudaGetLastError();
}

// One warp per cell, two of the 4x4x4 sub-cell centres per lane.
__global__ void k_outside_fraction(const GridGeom grid, const __grid_constant__ GeomView geom, uint32_t cells,
                                   float* frac, float4* point) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t warps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t cell = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); cell < cells;
       cell += warps) {
    const uint32_t cx = cell % grid.dim.x, cy = (cell / grid.dim.x) % grid.dim.y,
                   cz = cell / (grid.dim.x * grid.dim.y);
    const float3 lo = make_float3(grid.gmin.x + cx * grid.cell.x, grid.gmin.y + cy * grid.cell.y,
                                  grid.gmin.z + cz * grid.cell.z);
    const bool near = lo.x <= geom.grid.gmax.x && lo.x + grid.cell.x >= geom.grid.gmin.x &&
                      lo.y <= geom.grid.gmax.y && lo.y + grid.cell.y >= geom.grid.gmin.y &&
                      lo.z <= geom.grid.gmax.z && lo.z + grid.cell.z >= geom.grid.gmin.z;
    if (!near) {
      if (lane == 0) {
        frac[cell] = 1.f;
        point[cell] = make_float4(lo.x + 0.5f * grid.cell.x, lo.y + 0.5f * grid.cell.y,
                                  lo.z + 0.5f * grid.cell.z, 1.f);
      }
      continue;
    }
    bool out[2];
    float3 q[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const uint32_t sidx = lane * 2u + (uint32_t)h;
      q[h] = make_float3(lo.x + ((sidx & 3u) + 0.5f) * 0.25f * grid.cell.x,
                         lo.y + (((sidx >> 2) & 3u) + 0.5f) * 0.25f * grid.cell.y,
                         lo.z + ((sidx >> 4) + 0.5f) * 0.25f * grid.cell.z);
      out[h] = !inside_mesh(geom, q[h]);
    }
    const unsigned m0 = __ballot_sync(0xffffffffu, out[0]);
    const unsigned m1 = __ballot_sync(0xffffffffu, out[1]);
    const uint32_t n_out = __popc(m0) + __popc(m1);
    const int src = m0 ? __ffs(m0) - 1 : (m1 ? __ffs(m1) - 1 : 0);
    const int which = m0 ? 0 : 1;
    const float px = __shfl_sync(0xffffffffu, which ? q[1].x : q[0].x, src);
    const float py = __shfl_sync(0xffffffffu, which ? q[1].y : q[0].y, src);
    const float pz = __shfl_sync(0xffffffffu, which ? q[1].z : q[0].z, src);
    if (lane == 0) {
      frac[cell] = (float)n_out / 64.f;
      point[cell] = make_float4(px, py, pz, n_out ? 1.f : 0.f);
    }
  }
}

// Distance from q to the triangle (a, b, c): inside the prism over the
// triangle the distance to its plane, otherwise the nearest of its edges
// (closest point of each edge segment).
__device__ float point_triangle_distance(float3 q, float3 a, float3 b, float3 c) {
  const float3 ab = make_float3(b.x - a.x, b.y - a.y, b.z - a.z);
  const float3 bc = make_float3(c.x - b.x, c.y - b.y, c.z - b.z);
  const float3 ca = make_float3(a.x - c.x, a.y - c.y, a.z - c.z);
  const float3 n = make_float3(ab.y * (-ca.z) - ab.z * (-ca.y), ab.z * (-ca.x) - ab.x * (-ca.z),
                               ab.x * (-ca.y) - ab.y * (-ca.x));
  const float nn = n.x * n.x + n.y * n.y + n.z * n.z;
  auto side = [&](float3 e, float3 p0) {
    const float3 r = make_float3(q.x - p0.x, q.y - p0.y, q.z - p0.z);
    const float3 x = make_float3(e.y * r.z - e.z * r.y, e.z * r.x - e.x * r.z, e.x * r.y - e.y * r.x);
    return x.x * n.x + x.y * n.y + x.z * n.z;
  };
  if (nn > 0.f && side(ab, a) >= 0.f && side(bc, b) >= 0.f && side(ca, c) >= 0.f) {
    const float h = (q.x - a.x) * n.x + (q.y - a.y) * n.y + (q.z - a.z) * n.z;
    return fabsf(h) * rsqrtf(nn);
  }
  auto seg = [&](float3 p0, float3 e) {
    const float ee = e.x * e.x + e.y * e.y + e.z * e.z;
    float t = ee > 0.f ? ((q.x - p0.x) * e.x + (q.y - p0.y) * e.y + (q.z - p0.z) * e.z) / ee : 0.f;
    t = fminf(fmaxf(t, 0.f), 1.f);
    const float3 d = make_float3(q.x - (p0.x + t * e.x), q.y - (p0.y + t * e.y), q.z - (p0.z + t * e.z));
    return sqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
  };
  return fminf(seg(a, ab), fminf(seg(b, bc), seg(c, ca)));
}

// Clearance table on the refined grid `fine` (fac x fac x fac cells per cell
// of the triangle grid).  cdist holds each triangle-grid cell's Chebyshev
// distance in cells to the nearest cell holding triangles (-1: none at all).
// Cells at distance >= 2 keep the cell-count bound (cdist - 1) * cmin; the
// others take the exact distance from their centre to the triangles of the
// 27 triangle-grid cells around, less half their diagonal, capped by cmin
// (triangles farther out are at least one triangle-grid cell away).  All
// bounds are scaled by 0.999 to stay below the true distance.
__global__ void k_fine_clearance(const __grid_constant__ GeomView g, GridGeom fine, uint32_t fac,
                                 const int* __restrict__ cdist, float cmin, float* out) {
  const uint32_t n = fine.dim.x * fine.dim.y * fine.dim.z;
  const float hd = 0.5f * sqrtf(fine.cell.x * fine.cell.x + fine.cell.y * fine.cell.y +
                                fine.cell.z * fine.cell.z);
  for (uint32_t f = blockIdx.x * blockDim.x + threadIdx.x; f < n; f += gridDim.x * blockDim.x) {
    const uint32_t fx = f % fine.dim.x, fy = (f / fine.dim.x) % fine.dim.y,
                   fz = f / (fine.dim.x * fine.dim.y);
    const int cx = (int)(fx / fac), cy = (int)(fy / fac), cz = (int)(fz / fac);
    const int D = cdist[((uint32_t)cz * g.grid.dim.y + (uint32_t)cy) * g.grid.dim.x + (uint32_t)cx];
    float c;
    if (D < 0) {
      c = 3.0e38f;
    } else if (D >= 2) {
      c = 0.999f * (float)(D - 1) * cmin;
    } else {
      const float3 q = make_float3(fine.gmin.x + ((float)fx + 0.5f) * fine.cell.x,
                                   fine.gmin.y + ((float)fy + 0.5f) * fine.cell.y,
                                   fine.gmin.z + ((float)fz + 0.5f) * fine.cell.z);
      float best = 3.0e38f;
      for (int dz = -1; dz <= 1; dz++)
        for (int dy = -1; dy <= 1; dy++)
          for (int dx = -1; dx <= 1; dx++) {
            const int x = cx + dx, y = cy + dy, z = cz + dz;
            if (x < 0 || y < 0 || z < 0 || x >= (int)g.grid.dim.x || y >= (int)g.grid.dim.y ||
                z >= (int)g.grid.dim.z)
              continue;
            const uint2 se = g.start_end[((uint32_t)z * g.grid.dim.y + (uint32_t)y) * g.grid.dim.x + (uint32_t)x];
            for (uint32_t i = se.x; i < se.y; i++) {
              const float4 A = g.tri[kTriStride * (size_t)i], B = g.tri[kTriStride * (size_t)i + 1],
                           C = g.tri[kTriStride * (size_t)i + 2];
              best = fminf(best, point_triangle_distance(q, make_float3(A.x, A.y, A.z),
                                                         make_float3(B.x, B.y, B.z),
                                                         make_float3(C.x, C.y, C.z)));
            }
          }
      c = 0.999f * fmaxf(0.f, fminf(best - hd, cmin));
    }
    out[f] = c;
  }
}

__device__ __forceinline__ double axis_of(const double3& v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

// The slope bound of a triangle U that rises above T's plane, seen from T:
// the least k such that height(x) - tol <= k * sigma(x) at U's three
// vertices (so on all of U, both sides being linear) for one in-plane
// half-plane sigma <= 0 that holds T (an edge's outer side, or a direction
// of a vertex's normal cone: 3 edges and 7 directions per vertex).  As
// sigma(x) <= dist(x, T), every point of U then lies at most tol + k * dist
// above T's plane.  Infinity where no half-plane gives a bound.
__device__ double rise_slope(const double3 V[3], const double3 un[3], double3 n, const double3 W[3], double tol) {
  double best = 1e300;
  for (int c = 0; c < 24; c++) {
    // c < 3: edge c's outer normal (edge c runs from V[c] to V[c+1]); then 7
    // directions between the outer normals of the two edges at each vertex
    double3 u, P;
    if (c < 3) {
      u = un[c];
      P = V[c];
    } else {
      const int k = (c - 3) / 7, m = (c - 3) % 7;  // vertex k: edges k - 1 and k
      const double t = (m + 1) / 8.0;
      const double3 a = un[(k + 2) % 3], b = un[k];
      u = make_double3((1 - t) * a.x + t * b.x, (1 - t) * a.y + t * b.y, (1 - t) * a.z + t * b.z);
      const double l = sqrt(u.x * u.x + u.y * u.y + u.z * u.z);
      u = make_double3(u.x / l, u.y / l, u.z / l);
      P = V[k];
    }
    double lo = 0.0, hi = 1e300;
    bool ok = true;
    for (int q = 0; q < 3 && ok; q++) {
      const double3 d = make_double3(W[q].x - V[0].x, W[q].y - V[0].y, W[q].z - V[0].z);
      const double a = n.x * d.x + n.y * d.y + n.z * d.z - tol;
      const double b = u.x * (W[q].x - P.x) + u.y * (W[q].y - P.y) + u.z * (W[q].z - P.z);
      if (b > 1e-12) lo = fmax(lo, a / b);
      else if (b < -1e-12) hi = a > 0.0 ? -1.0 : fmin(hi, a / b);
      else ok = a <= 0.0;
    }
    if (ok && lo <= hi) best = fmin(best, lo);
  }
  return best;
}

// Reach of every bin entry's triangle T, for a particle that leaves T
// outward (re-emitted or reflected; it starts 1 um above T along T's normal):
// (r, k) such that a path shorter than r whose direction makes more than k
// with T's normal (the sine of its elevation) crosses no listed triangle.
// Every triangle U within rmax of T is listed in a cell that T's box, grown
// by rmax and one more cell, overlaps.  A U with no vertex more than tol
// above T's plane cannot be crossed from above it.  A U that rises above
// the plane either caps r by the distance between the two boxes (a lower
// bound of the distance between the triangles), or, when its slope bound
// (rise_slope) is below 1/2, raises k to that bound: a path of elevation
// above k climbs faster than U rises with the distance from T.  r is lowered
// by `slack` (the set-off and the rounding of the hit point) and by 0.1 %;
// (0, 2) where nothing is left.
__global__ void k_entry_reach(const __grid_constant__ GeomView g, uint32_t entries, float rmax, float tol,
                              float slack, float2* __restrict__ out) {
  const float grow = rmax + fmaxf(g.grid.cell.x, fmaxf(g.grid.cell.y, g.grid.cell.z));
  for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < entries; e += gridDim.x * blockDim.x) {
    const float4 A = g.tri[kTriStride * (size_t)e], B = g.tri[kTriStride * (size_t)e + 1],
                 C = g.tri[kTriStride * (size_t)e + 2];
    const float4 P = g.plane[e];
    const double3 V[3] = {make_double3(A.x, A.y, A.z), make_double3(B.x, B.y, B.z), make_double3(C.x, C.y, C.z)};
    // T's unit normal from its vertices in FP64 (the stored plane's orientation)
    const double3 e1 = make_double3(V[1].x - V[0].x, V[1].y - V[0].y, V[1].z - V[0].z);
    const double3 e2 = make_double3(V[2].x - V[0].x, V[2].y - V[0].y, V[2].z - V[0].z);
    double3 n = make_double3(e1.y * e2.z - e1.z * e2.y, e1.z * e2.x - e1.x * e2.z, e1.x * e2.y - e1.y * e2.x);
    const double nl = sqrt(n.x * n.x + n.y * n.y + n.z * n.z);
    float2 res = make_float2(0.f, 2.f);
    if (nl > 0.0) {
      n = make_double3(n.x / nl, n.y / nl, n.z / nl);
    }
    // the normal the wall response uses must agree with the vertices' one
    if (nl > 0.0 && n.x * P.x + n.y * P.y + n.z * P.z > 0.9999) {
      // in-plane outer normals of the edges V[c] -> V[c+1]
      double3 un[3];
      for (int c = 0; c < 3; c++) {
        const double3 a = V[c], b = V[(c + 1) % 3];
        const double3 d = make_double3(b.x - a.x, b.y - a.y, b.z - a.z);
        double3 u = make_double3(d.y * n.z - d.z * n.y, d.z * n.x - d.x * n.z, d.x * n.y - d.y * n.x);
        const double l = sqrt(u.x * u.x + u.y * u.y + u.z * u.z);
        u = make_double3(u.x / l, u.y / l, u.z / l);
        const double3 o = V[(c + 2) % 3];
        if (u.x * (o.x - a.x) + u.y * (o.y - a.y) + u.z * (o.z - a.z) > 0.0) u = make_double3(-u.x, -u.y, -u.z);
        un[c] = u;
      }
      const float lo[3] = {fminf(A.x, fminf(B.x, C.x)), fminf(A.y, fminf(B.y, C.y)), fminf(A.z, fminf(B.z, C.z))};
      const float hi[3] = {fmaxf(A.x, fmaxf(B.x, C.x)), fmaxf(A.y, fmaxf(B.y, C.y)), fmaxf(A.z, fmaxf(B.z, C.z))};
      const float gmn[3] = {g.grid.gmin.x, g.grid.gmin.y, g.grid.gmin.z};
      const float cs[3] = {g.grid.cell.x, g.grid.cell.y, g.grid.cell.z};
      const int dim[3] = {(int)g.grid.dim.x, (int)g.grid.dim.y, (int)g.grid.dim.z};
      int c0[3], c1[3];
      for (int k = 0; k < 3; k++) {
        c0[k] = max(0, (int)floorf((lo[k] - grow - gmn[k]) / cs[k]));
        c1[k] = min(dim[k] - 1, (int)floorf((hi[k] + grow - gmn[k]) / cs[k]));
      }
      double best = rmax, slope = 0.0;
      for (int z = c0[2]; z <= c1[2]; z++)
        for (int y = c0[1]; y <= c1[1]; y++)
          for (int x = c0[0]; x <= c1[0]; x++) {
            const uint2 se = g.start_end[((uint32_t)z * g.grid.dim.y + (uint32_t)y) * g.grid.dim.x + (uint32_t)x];
            if (se.x == kNone) continue;
            for (uint32_t j = se.x; j < se.y; j++) {
              double3 W[3];
              for (int k = 0; k < 3; k++) {
                const float4 q = g.tri[kTriStride * (size_t)j + k];
                W[k] = make_double3(q.x, q.y, q.z);
              }
              double up = -1.0;
              for (int k = 0; k < 3; k++)
                up = fmax(up, n.x * (W[k].x - V[0].x) + n.y * (W[k].y - V[0].y) + n.z * (W[k].z - V[0].z));
              if (up <= tol) continue;
              const double k_rise = rise_slope(V, un, n, W, tol);
              if (k_rise < 0.5) {
                slope = fmax(slope, k_rise);
                continue;
              }
              // no usable slope: the distance between the two boxes
              double d2 = 0.0;
              for (int k = 0; k < 3; k++) {
                const double w0 = axis_of(W[0], k), w1 = axis_of(W[1], k), w2 = axis_of(W[2], k);
                const double wl = fmin(w0, fmin(w1, w2)), wh = fmax(w0, fmax(w1, w2));
                const double gap = fmax(0.0, fmax(wl - hi[k], (double)lo[k] - wh));
                d2 += gap * gap;
              }
              best = fmin(best, sqrt(d2));
            }
          }
      const float r = fmaxf(0.f, 0.999f * (float)best - slack);
      if (r > 0.f) res = make_float2(r, __double2float_ru(slope));
    }
    out[e] = res;
  }
}

// The slab of every grid cell (GeomView::slab): n the normalised sum of the
// cell's triangle normals, [lo, hi] the range of n . v over every vertex of
// every listed triangle (FP64), widened by a margin; m = n / h, e = c / h
// with c the middle and h the half width.  Cells whose normals disagree
// (the sum shorter than half the count) pass every path.
__global__ void k_cell_slab(const __grid_constant__ GeomView g, uint32_t cells, float4* __restrict__ out) {
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < cells; c += gridDim.x * blockDim.x) {
    const uint2 se = g.start_end[c];
    float4 r = make_float4(0.f, 0.f, 0.f, 0.f);
    if (se.x != kNone && se.y > se.x) {
      double nx = 0.0, ny = 0.0, nz = 0.0;
      for (uint32_t i = se.x; i < se.y; i++) {
        const float4 P = g.plane[i];
        nx += P.x; ny += P.y; nz += P.z;
      }
      const double l = sqrt(nx * nx + ny * ny + nz * nz);
      if (l >= 0.5 * (double)(se.y - se.x)) {
        nx /= l; ny /= l; nz /= l;
        double lo = 1e300, hi = -1e300, mag = 0.0;
        for (uint32_t i = se.x; i < se.y; i++)
          for (int k = 0; k < 3; k++) {
            const float4 v = g.tri[kTriStride * (size_t)i + k];
            const double t = nx * v.x + ny * v.y + nz * v.z;
            lo = fmin(lo, t);
            hi = fmax(hi, t);
            mag = fmax(mag, fabs((double)v.x) + fabs((double)v.y) + fabs((double)v.z));
          }
        const double cmid = 0.5 * (lo + hi);
        const double h = 0.5 * (hi - lo) + 1e-6 + 1e-6 * mag;
        r = make_float4((float)(nx / h), (float)(ny / h), (float)(nz / h), (float)(cmid / h));
      }
    }
    out[c] = r;
  }
}

cudaError_t launch_cell_slab(const GeomView& g, uint32_t cells, float4* out, cudaStream_t stream) {
  if (cells == 0) return cudaSuccess;
  k_cell_slab<<<grid_for(cells, 128, 8), 128, 0, stream>>>(g, cells, out);
  return cudaGetLastError();
}

__global__ void k_clearance_at(const __grid_constant__ GeomView g, const float* __restrict__ xyz,
                               uint32_t n, float* __restrict__ out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float3 q = make_float3(xyz[3 * (size_t)i], xyz[3 * (size_t)i + 1], xyz[3 * (size_t)i + 2]);
    const uint32_t c = coll_cell_id(g.cgrid, q);
    out[i] = c == kNone ? -1.f : g.clear[c];
  }
}

cudaError_t launch_clearance_at(const GeomView& g, const float* xyz, uint32_t n, float* out,
                                cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  k_clearance_at<<<grid_for(n, 256, 8), 256, 0, stream>>>(g, xyz, n, out);
  return cudaGetLastError();
}

cudaError_t launch_entry_reach(const GeomView& g, uint32_t entries, float rmax, float tol, float slack,
                               float2* out, cudaStream_t stream) {
  if (entries == 0) return cudaSuccess;
  k_entry_reach<<<grid_for(entries, 128, 8), 128, 0, stream>>>(g, entries, rmax, tol, slack, out);
  return cudaGetLastError();
}

cudaError_t launch_fine_clearance(const GeomView& g, const GridGeom& fine, uint32_t fac,
                                  const int* cdist, float cmin, float* out, cudaStream_t stream) {
  const uint32_t n = fine.dim.x * fine.dim.y * fine.dim.z;
  k_fine_clearance<<<grid_for(n, 256, 8), 256, 0, stream>>>(g, fine, fac, cdist, cmin, out);
  return cudaGetLastError();
}

cudaError_t launch_outside_fraction(const GridGeom& grid, const GeomView& geom, uint32_t cells,
                                    float* frac, float4* point, cudaStream_t stream) {
  const uint32_t blocks = (uint32_t)std::min<uint64_t>(((uint64_t)cells + 7) / 8, 8u * num_sms());
  k_outside_fraction<<<blocks, 256, 0, stream>>>(grid, geom, cells, frac, point);
  return cudaGetLastError();
}

cudaError_t launch_init_fill(const InitParams& p, cudaStream_t stream) {
  const uint64_t total = (uint64_t)p.cells * p.ppc;
  const uint32_t grid = grid_for(total, 256, 8);
  k_init_fill<<<grid, 256, 0, stream>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_scan_b(const BatchOf<SortArgs>& bv, uint32_t blocks, cudaStream_t stream) {
  return blocks ? launch_chained(k_scan_b, blocks, 256, 0, stream, false, bv) : cudaSuccess;
}

cudaError_t launch_scatter_b(const BatchOf<SortArgs>& bv, uint32_t blocks, cudaStream_t stream) {
  return blocks ? launch_chained(k_scatter_b, blocks, 256, 0, stream, false, bv) : cudaSuccess;
}

cudaError_t launch_inject_b(const BatchOf<InjectParams>& plan, uint32_t plan_blocks,
                            const BatchOf<InjectParams>& fill, uint32_t fill_blocks, size_t fill_smem,
                            cudaStream_t stream) {
  cudaError_t e = cudaSuccess;
  if (plan_blocks) e = launch_chained(k_inject_plan_b, plan_blocks, 32, 0, stream, false, plan);
  if (!e && fill_blocks) e = launch_chained(k_inject_fill_b, fill_blocks, 256, fill_smem, stream, false, fill);
  return e;
}

cudaError_t launch_inject(const InjectParams& p, cudaStream_t stream) {
  cudaError_t e = launch_chained(k_inject_plan, 1, 32, 0, stream, true, p, p.plan);
  const uint32_t grid = (uint32_t)num_sms();
  if (!e) e = launch_chained(k_inject_fill, grid, 256, p.n_scan_tiles * 4, stream, true, p, p.plan);
  return e;
}

}  // namespace dsmcb
