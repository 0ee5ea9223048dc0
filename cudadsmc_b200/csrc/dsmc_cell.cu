// The timestep's fused cell kernel (sm_100a).
//
// Persistent CTAs (several per SM) walk tiles of cells.  A tile is processed
// in chunks of whole cells holding at most CAP particles.  The data of the
// next chunk - the particle arrays (x, y, z, u, v, w, orig), the chunk's
// per-cell collision state, and for a new tile its cell starts - is fetched
// by the tensor memory accelerator as 1D bulk copies into the other half of a
// double buffer, completing on mbarriers, while the current chunk is
// processed:
//   A  cell of every staged particle; its rank by orig inside the cell (the
//      stable order of the reference's sort); dense-cell list (Philox mode)
//   B  NTC collisions: one lane per cell, a whole warp per dense cell
//   C  flight (mesh, boundaries), next-step key and count, stores in sorted
//      order, per-cell state written back
//   D  FP64 sampling every sample_every steps
// The phases of one chunk are latency-bound; several independent CTAs per SM
// overlap them.  The (threads, capacity) variant is chosen at run time.
// Algorithmic traffic per particle: 28 B read (state + orig), 28 B written
// (state + key), plus about 24-56 B per cell of collision state.
#include "dsmc_bulk.cuh"
#include "dsmc_step_dev.cuh"

namespace dsmcb {
namespace {

using namespace dev;

constexpr int kCellArr = kMaxCellsPerTile + 4;   // float2 per-cell slots (+ slack)
constexpr int kLsArr = kMaxCellsPerTile + 8;

struct Chunk {
  uint32_t tile, c0, nct, cur, k, base, n;
  int lsb;    // ls buffer holding the tile's starts
  int buf;    // staging buffer
  int giant;  // one cell above the chunk capacity
  int valid;
  uint32_t ntile;  // the tile the CTA processes after this chunk's tile
};

// Hands out the CTA's tiles after its first (blockIdx.x): from the step's
// dynamic tile counter (tiles past the first wave go to whichever CTA asks
// first), or round robin when the launch has no counter.  Used by thread 0,
// which asks one tile ahead of need so that the atomic's latency is hidden.
struct TileSource {
  uint32_t next_static;
  __device__ __forceinline__ uint32_t grab(const StepParams& p) {
    if (p.meta) return gridDim.x + atomicAdd(&p.meta->tile_next, 1u);
    const uint32_t t = next_static;
    next_static += gridDim.x;
    return t;
  }
};

// Shared memory of one CTA; the scan-tile histogram (n_scan_tiles words)
// follows the structure.
template <int CAP>
struct __align__(128) CellSmem {
  float part[2][7][CAP + 4];
  float2 maxrem[2][kCellArr];
  uint4 seeds[2][kMaxCellsPerTile];
  uint32_t ls[3][kLsArr];        // starts of the current, next and following tile
  unsigned long long mbar[2];     // chunk data of buffer b
  unsigned long long mbar_ls[3];  // starts of ls buffer b
  Chunk cur, next;
  uint32_t nheavy;
  uint32_t nhard;
  uint32_t claim[CAP + 4];
  uint32_t cellm[kMaxCellsPerTile];
  uint16_t heavy[kMaxCellsPerTile];
  uint16_t slot[CAP];
  uint16_t hardq[CAP];  // staged particles whose flight may meet the body
  uint8_t cellof[CAP];
};

template <int CAP>
constexpr size_t smem_bytes(uint32_t n_scan_tiles) {
  return ((sizeof(CellSmem<CAP>) + 15) & ~(size_t)15) + 4 * (size_t)n_scan_tiles;
}

// --------------------------------------------------------------- chunks ----

// Chunk of tile `tile` starting at local cell `cur`: as many whole cells as
// fit CAP particles (one cell if even that one does not fit: giant).
template <int CAP>
__device__ Chunk make_chunk(const CellSmem<CAP>& S, uint32_t tile, int lsb, uint32_t cur,
                            uint32_t ct, uint32_t cells, int buf) {
  Chunk c;
  c.tile = tile;
  c.c0 = tile * ct;
  c.nct = min(ct, cells - c.c0);
  c.cur = cur;
  c.lsb = lsb;
  c.buf = buf;
  c.valid = 1;
  const uint32_t* ls = S.ls[lsb];
  const uint32_t base = ls[cur];
  uint32_t lo = 0, hi = c.nct - cur;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (ls[cur + mid] - base <= (uint32_t)CAP) lo = mid; else hi = mid - 1;
  }
  c.giant = lo == 0;
  c.k = lo == 0 ? 1u : lo;
  c.base = base;
  c.n = ls[cur + c.k] - base;
  return c;
}

__device__ __forceinline__ bool chunk_has_data(const Chunk& c) { return !c.giant && c.n > 0; }

// Element ranges of a chunk's copies.  Padded (the library's own buffers,
// allocated with 16 bytes of slack): the whole 16-byte aligned cover of the
// range.  Otherwise only the aligned interior; the ragged head and tail are
// read with plain loads after the copy (ragged_chunk), so a caller's buffer is
// never read past its end.
struct Span {
  uint32_t ia, ib;
};
__device__ __forceinline__ Span span4(uint32_t b, uint32_t e, bool padded) {
  return padded ? Span{b & ~3u, (e + 3u) & ~3u} : Span{(b + 3u) & ~3u, e & ~3u};
}
__device__ __forceinline__ Span span8(uint32_t b, uint32_t e, bool padded) {
  return padded ? Span{b & ~1u, (e + 1u) & ~1u} : Span{(b + 1u) & ~1u, e & ~1u};
}

__device__ __forceinline__ const float* part_src(const StepParams& p, int a) {
  switch (a) {
    case 0: return p.in.x;
    case 1: return p.in.y;
    case 2: return p.in.z;
    case 3: return p.in.u;
    case 4: return p.in.v;
    case 5: return p.in.w;
    default: return reinterpret_cast<const float*>(p.in_orig);
  }
}

// Issues the bulk copies of a chunk from lanes of warp 0 (the warp must be
// converged; lane 0 arms the mbarrier).
template <int CAP>
__device__ void issue_chunk(const StepParams& p, CellSmem<CAP>& S, const Chunk& c) {
  const unsigned lane = lane_id();
  const bool padded = (p.flags & kPadded) != 0;
  const bool vel_only = (p.flags & kVelOnly) != 0;
  const bool fix = (p.flags & kDoFixup) != 0;
  const bool collide = (p.flags & kDoCollide) != 0;
  const bool taus = p.rng_kind == 0;
  const uint32_t a0 = c.base & ~3u;
  const Span ps = span4(c.base, c.base + c.n, padded);
  const uint32_t pbytes = ps.ib > ps.ia ? (ps.ib - ps.ia) * 4u : 0u;
  const uint32_t cs = c.c0 + c.cur;
  const Span ms = span8(cs, cs + c.k, padded);
  const uint32_t mbytes = (collide && ms.ib > ms.ia) ? (ms.ib - ms.ia) * 8u : 0u;
  const uint32_t sbytes = (collide && taus) ? c.k * 16u : 0u;
  const uint32_t narr = vel_only ? 3u : (fix ? 7u : 6u);
  unsigned long long* m = &S.mbar[c.buf];
  if (lane == 0) mbar_expect_tx(m, pbytes * narr + mbytes + sbytes);
  __syncwarp();
  fence_proxy_async();
  const int first = vel_only ? 3 : 0;
  if (lane < narr) {
    const int a = first + (int)lane;
    if (pbytes) bulk_g2s(S.part[c.buf][a] + (ps.ia - a0), part_src(p, a) + ps.ia, pbytes, m);
  } else if (lane == 8 && mbytes) {
    bulk_g2s(S.maxrem[c.buf] + (ms.ia - (cs & ~1u)), p.maxrem + ms.ia, mbytes, m);
  } else if (lane == 9 && sbytes) {
    bulk_g2s(S.seeds[c.buf], p.seeds + cs, sbytes, m);
  }
}

// The ragged ends of a chunk's copies (not padded), by plain loads.
template <int CAP>
__device__ void ragged_chunk(const StepParams& p, CellSmem<CAP>& S, const Chunk& c) {
  const bool vel_only = (p.flags & kVelOnly) != 0;
  const bool fix = (p.flags & kDoFixup) != 0;
  const uint32_t a0 = c.base & ~3u, e = c.base + c.n;
  const Span ps = span4(c.base, e, false);
  const uint32_t narr = vel_only ? 3u : (fix ? 7u : 6u);
  const int first = vel_only ? 3 : 0;
  // head [base, min(ia, e)) and tail [max(ib, ia, base), e): at most 3 each
  const uint32_t h1 = min(ps.ia, e), t0 = max(max(ps.ib, ps.ia), c.base);
  for (uint32_t w = threadIdx.x; w < narr * 8u; w += blockDim.x) {
    const int a = first + (int)(w >> 3);
    const uint32_t r = w & 7u;
    uint32_t i = kNone;
    if (r < 4u) { if (c.base + r < h1) i = c.base + r; }
    else if (t0 + (r - 4u) < e) i = t0 + (r - 4u);
    if (i != kNone) S.part[c.buf][a][i - a0] = part_src(p, a)[i];
  }
  if ((p.flags & kDoCollide) && threadIdx.x == blockDim.x - 1) {
    const uint32_t cs = c.c0 + c.cur, ce = cs + c.k;
    const Span ms = span8(cs, ce, false);
    for (uint32_t i = cs; i < min(ms.ia, ce); i++) S.maxrem[c.buf][i - (cs & ~1u)] = p.maxrem[i];
    for (uint32_t i = max(max(ms.ib, ms.ia), cs); i < ce; i++)
      S.maxrem[c.buf][i - (cs & ~1u)] = p.maxrem[i];
  }
}

// Issues the copy of the cell starts of `tile` into ls buffer b (thread 0);
// when not padded the ragged tail is read by finish_ls after the wait.
template <int CAP>
__device__ void issue_ls(const StepParams& p, CellSmem<CAP>& S, uint32_t tile, int b) {
  const uint32_t ct = (uint32_t)p.cells_per_tile;
  const uint32_t nct = min(ct, p.cells - tile * ct);
  const uint32_t whole = (p.flags & kPadded) ? ((nct + 1u + 3u) & ~3u) : ((nct + 1u) & ~3u);
  fence_proxy_async();
  mbar_expect_tx(&S.mbar_ls[b], whole * 4u);
  if (whole) bulk_g2s(S.ls[b], p.start + tile * ct, whole * 4u, &S.mbar_ls[b]);
}
template <int CAP>
__device__ void finish_ls(const StepParams& p, CellSmem<CAP>& S, uint32_t tile, int b) {
  if (p.flags & kPadded) return;
  const uint32_t ct = (uint32_t)p.cells_per_tile;
  const uint32_t nct = min(ct, p.cells - tile * ct);
  for (uint32_t i = (nct + 1u) & ~3u; i <= nct; i++) S.ls[b][i] = p.start[tile * ct + i];
}

// ----------------------------------------------------------- giant cell ----

// A cell too large for the shared-memory chunk: processed by the whole block
// directly in the output arrays.
static __device__ __noinline__ void giant_cell(const StepParams& p, uint32_t cell, uint32_t s, uint32_t e,
                           uint32_t step, bool do_sample, uint32_t* s_tile, uint32_t& sel,
                           uint32_t& col, double& sum_g, uint32_t& removed) {
  __shared__ double red[4][32];
  const uint32_t n = e - s;
  const bool vel_only = (p.flags & kVelOnly) != 0;
  if (threadIdx.x == 0 && p.meta) atomicAdd(&p.meta->giant_cells, 1u);
  if (p.flags & kDoFixup) {
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
      const uint32_t my = p.in_orig[s + i];
      uint32_t rank = 0;
      for (uint32_t j = 0; j < n; j++) {
        const uint32_t o = p.in_orig[s + j];
        rank += (o < my) | ((o == my) & (j < i));
      }
      const uint32_t d = s + rank;
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
    CellState st{p.maxrem + cell, p.seeds ? p.seeds + cell : nullptr,
                 p.stat4 ? p.stat4 + cell : nullptr};
    collide_cell(p, cell, (int)n, acc, step, st, sel, col, sum_g);
  }
  __threadfence_block();
  __syncthreads();
  double su = 0, sv = 0, sw = 0, se = 0;
  for (uint32_t qb = 0; qb < n; qb += blockDim.x) {
    const uint32_t q = qb + threadIdx.x;
    const bool active = q < n;
    float3 pos = make_float3(0.f, 0.f, 0.f), vel = pos;
    bool live = true;
    if (active) {
      const uint32_t g = s + q;
      if (!vel_only) pos = make_float3(p.out.x[g], p.out.y[g], p.out.z[g]);
      vel = make_float3(p.out.u[g], p.out.v[g], p.out.w[g]);
      if (p.flags & kDoMove) live = move_particle(p, pos, vel, g, step);
      if (do_sample) {
        const double x = vel.x, y = vel.y, z = vel.z;
        su += x; sv += y; sw += z;
        se += x * x + y * y + z * z;
      }
      if (!vel_only) { p.out.x[g] = pos.x; p.out.y[g] = pos.y; p.out.z[g] = pos.z; }
      p.out.u[g] = vel.x; p.out.v[g] = vel.y; p.out.w[g] = vel.z;
    }
    if (p.flags & kDoKeys) {
      const bool has_key = active && live;
      const unsigned m = __ballot_sync(kFull, has_key);
      if (active && !live) removed++;
      if (has_key) {
        const uint32_t key = cell_id3d(p.grid, pos.x, pos.y, pos.z);
        warp_count_key(p.count, key, m, s_tile);
        p.out_key[s + q] = key;
      } else if (active) {
        p.out_key[s + q] = kDeadKey;
      }
    }
  }
  if (do_sample) {
    su = warp_sum(su); sv = warp_sum(sv); sw = warp_sum(sw); se = warp_sum(se);
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

// ---------------------------------------------------------------- kernel ----

template <int THREADS, int CAP, int MINB>
__global__ void __launch_bounds__(THREADS, MINB) k_cell(const __grid_constant__ StepParams p) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  CellSmem<CAP>& S = *reinterpret_cast<CellSmem<CAP>*>(smem_raw);
  uint32_t* s_tile = reinterpret_cast<uint32_t*>(smem_raw + ((sizeof(CellSmem<CAP>) + 15) & ~(size_t)15));
  const uint32_t step = p.step_override ? p.step_override : p.meta->step;
  const bool do_sample =
      (p.flags & kDoSample) &&
      ((p.flags & kSampleForce) || (p.sample_every > 0 && step % (uint32_t)p.sample_every == 0));
  const bool do_fixup = (p.flags & kDoFixup) != 0;
  const bool do_collide = (p.flags & kDoCollide) != 0;
  const bool do_keys = (p.flags & kDoKeys) != 0;
  const bool vel_only = (p.flags & kVelOnly) != 0;
  const bool padded = (p.flags & kPadded) != 0;
  const bool taus = p.rng_kind == 0;
  const bool heavy_mode = !taus && do_collide;
  const uint32_t ct = (uint32_t)p.cells_per_tile;
  const uint32_t tid = threadIdx.x;
  const uint32_t warp = tid >> 5;

  for (uint32_t t = tid; t < p.n_scan_tiles; t += blockDim.x) s_tile[t] = 0;
  for (uint32_t t = tid; t < (uint32_t)(CAP + 4); t += blockDim.x) S.claim[t] = 0xffffffffu;
  // mbarrier phase bits: bit b for chunk buffer b, bit 2+b for ls buffer b
  uint32_t phase = 0u;
  TileSource tiles{blockIdx.x + gridDim.x};
  uint32_t pending = 0;  // thread 0: the tile after the next one
  if (tid == 0) {
    mbar_init(&S.mbar[0], 1);
    mbar_init(&S.mbar[1], 1);
    mbar_init(&S.mbar_ls[0], 1);
    mbar_init(&S.mbar_ls[1], 1);
    mbar_init(&S.mbar_ls[2], 1);
    fence_mbar_init();
    S.cur.valid = 0;
    if (blockIdx.x < p.n_tiles) issue_ls(p, S, blockIdx.x, 0);
  }
  __syncthreads();
  uint32_t sel = 0, col = 0, removed = 0;
  double sum_g = 0.0;
  bool ok = true;
  if (blockIdx.x < p.n_tiles) {
    ok = mbar_wait_bounded(&S.mbar_ls[0], (phase >> 2) & 1u);
    phase ^= 4u;
  }
  if (!__syncthreads_and(ok)) {
    if (tid == 0 && p.meta) atomicOr(&p.meta->error, kErrTimeout);
    return;
  }
  if (warp == 0 && blockIdx.x < p.n_tiles) {
    if (tid == 0) {
      finish_ls(p, S, blockIdx.x, 0);
      S.cur = make_chunk(S, blockIdx.x, 0, 0, ct, p.cells, 0);
      S.cur.ntile = tiles.grab(p);
      pending = tiles.grab(p);
      if (S.cur.ntile < p.n_tiles) issue_ls(p, S, S.cur.ntile, 1);
    }
    __syncwarp();
    if (chunk_has_data(S.cur)) issue_chunk(p, S, S.cur);
  }
  __syncthreads();

  while (S.cur.valid) {
    const Chunk c = S.cur;
    // the CTA's next tile; its starts were fetched into ls buffer nb when
    // this tile's first chunk was made
    const uint32_t nt = c.ntile;
    const int nb = c.lsb == 2 ? 0 : c.lsb + 1;
    const uint32_t phase0 = phase;
    if (tid == 0) {
      S.nheavy = 0;
      S.nhard = 0;
    }
    if (chunk_has_data(c)) {
      ok = mbar_wait_bounded(&S.mbar[c.buf], (phase >> c.buf) & 1u);
      phase ^= 1u << c.buf;
    }
    // the next chunk; it may lie in the next tile, whose starts must be in
    const bool last_of_tile = c.cur + c.k >= c.nct;
    if (last_of_tile && nt < p.n_tiles) {
      ok = ok && mbar_wait_bounded(&S.mbar_ls[nb], (phase >> (2 + nb)) & 1u);
      phase ^= 1u << (2 + nb);
    }
    if (!__syncthreads_and(ok)) {
      if (tid == 0 && p.meta) atomicOr(&p.meta->error, kErrTimeout);
      // let the copies that may still be in flight (this chunk's data, the
      // next tile's starts) land before the CTA's shared memory goes away
      if (chunk_has_data(c)) mbar_wait_bounded(&S.mbar[c.buf], (phase0 >> c.buf) & 1u);
      if (nt < p.n_tiles) mbar_wait_bounded(&S.mbar_ls[nb], (phase0 >> (2 + nb)) & 1u);
      return;
    }
    if (warp == 0) {
      if (tid == 0) {
        Chunk nx;
        nx.valid = 0;
        if (!last_of_tile) {
          nx = make_chunk(S, c.tile, c.lsb, c.cur + c.k, ct, p.cells, 1 - c.buf);
          nx.ntile = nt;
        } else if (nt < p.n_tiles) {
          finish_ls(p, S, nt, nb);
          nx = make_chunk(S, nt, nb, 0, ct, p.cells, 1 - c.buf);
          nx.ntile = pending;
          pending = tiles.grab(p);
          // the following tile's starts go into the buffer this tile's
          // predecessor used
          if (nx.ntile < p.n_tiles) issue_ls(p, S, nx.ntile, nb == 2 ? 0 : nb + 1);
        }
        S.next = nx;
      }
      __syncwarp();
      if (S.next.valid && chunk_has_data(S.next)) issue_chunk(p, S, S.next);
    }
    if (chunk_has_data(c) && !padded) {
      ragged_chunk(p, S, c);
      __syncthreads();
    }
    const uint32_t* ls = S.ls[c.lsb];
    if (c.giant) {
      giant_cell(p, c.c0 + c.cur, c.base, ls[c.cur + 1], step, do_sample, s_tile, sel, col,
                 sum_g, removed);
    } else if (c.n > 0) {
      const uint32_t off = c.base - (c.base & ~3u);
      float* X = S.part[c.buf][0] + off;
      float* Y = S.part[c.buf][1] + off;
      float* Z = S.part[c.buf][2] + off;
      float* U = S.part[c.buf][3] + off;
      float* V = S.part[c.buf][4] + off;
      float* W = S.part[c.buf][5] + off;
      const uint32_t* OR = reinterpret_cast<const uint32_t*>(S.part[c.buf][6] + off);
      const uint32_t cs = c.c0 + c.cur;
      float2* MR = S.maxrem[c.buf] + (cs & 1u);
      uint4* SD = S.seeds[c.buf];
      const uint32_t base = c.base, n = c.n, cur = c.cur, k = c.k;
      // A1: cell of each staged particle; dense cells
      for (uint32_t lc = tid; lc < k; lc += blockDim.x) {
        const uint32_t s0 = ls[cur + lc] - base, e0 = ls[cur + lc + 1] - base;
        if (do_fixup)
          for (uint32_t j = s0; j < e0; j++) S.cellof[j] = (uint8_t)lc;
        if (heavy_mode) {
          const uint32_t nc = e0 - s0;
          const uint32_t m = nc >= 2 ? (uint32_t)ntc_fpc_fast(p, nc, MR[lc]) : 0u;
          S.cellm[lc] = m;
          if (m >= kHeavyMin) S.heavy[atomicAdd(&S.nheavy, 1u)] = (uint16_t)lc;
        }
      }
      __syncthreads();
      // A2: slot[sorted position] = staged index, sorted = (cell, orig)
      for (uint32_t t = tid; t < n; t += blockDim.x) {
        if (!do_fixup) {
          S.slot[t] = (uint16_t)t;
          continue;
        }
        const uint32_t lc = S.cellof[t];
        const uint32_t s0 = ls[cur + lc] - base, e0 = ls[cur + lc + 1] - base;
        const uint32_t my = OR[t];
        uint32_t rank = 0;
        for (uint32_t j = s0; j < e0; j++) {
          const uint32_t o = OR[j];
          rank += (o < my) | ((o == my) & (j < t));
        }
        S.slot[s0 + rank] = (uint16_t)t;
      }
      __syncthreads();
      // B: collisions; light cells one lane each, dense cells one warp each
      if (do_collide) {
        for (uint32_t lc = tid; lc < k; lc += blockDim.x) {
          if (heavy_mode && S.cellm[lc] >= kHeavyMin) continue;
          const uint32_t s0 = ls[cur + lc] - base, e0 = ls[cur + lc + 1] - base;
          SmemVel acc{U, V, W, S.slot, s0};
          CellState st{MR + lc, taus ? SD + lc : nullptr, p.stat4 ? p.stat4 + cs + lc : nullptr};
          collide_cell(p, cs + lc, (int)(e0 - s0), acc, step, st, sel, col, sum_g);
        }
        if (heavy_mode) {
          __syncwarp();
          const uint32_t nh = S.nheavy;
          for (uint32_t h = warp; h < nh; h += blockDim.x >> 5) {
            const uint32_t lc = S.heavy[h];
            const uint32_t s0 = ls[cur + lc] - base, e0 = ls[cur + lc + 1] - base;
            SmemVel acc{U, V, W, S.slot, s0};
            CellState st{MR + lc, nullptr, p.stat4 ? p.stat4 + cs + lc : nullptr};
            ntc_heavy_warp(p, cs + lc, e0 - s0, acc, S.claim, step, st, sel, col, sum_g);
          }
        }
        __syncthreads();
        // per-cell state back to global memory
        for (uint32_t lc = tid; lc < k; lc += blockDim.x) {
          p.maxrem[cs + lc] = MR[lc];
          if (taus) p.seeds[cs + lc] = SD[lc];
        }
      }
      // C: flight, next-step keys, stores in sorted order.  With a body,
      // particles whose path may reach it are queued in the first pass and
      // flown in a second pass by whole warps, so that the mesh traversal of
      // a few lanes does not hold up the cheap flights of the rest.
      const bool split = p.has_geom && (p.flags & kDoMove);
      const uint32_t lane = lane_id();
      for (uint32_t pass = 0; pass < (split ? 2u : 1u); pass++) {
        const uint32_t cnt = pass == 0 ? n : S.nhard;
        for (uint32_t qb = 0; qb < cnt; qb += blockDim.x) {
          const uint32_t i = qb + tid;
          const bool active = i < cnt;
          float3 pos = make_float3(0.f, 0.f, 0.f), vel = pos;
          uint32_t q = 0, j = 0;
          bool defer = false;
          if (active) {
            q = pass == 0 ? i : (uint32_t)S.hardq[i];
            j = S.slot[q];
            if (!vel_only) pos = make_float3(X[j], Y[j], Z[j]);
            vel = make_float3(U[j], V[j], W[j]);
            if (pass == 0 && split) defer = flight_may_meet_body(p, pos, vel);
          }
          const unsigned dm = __ballot_sync(kFull, defer);
          if (dm) {
            const int leader = __ffs(dm) - 1;
            uint32_t at = 0;
            if ((int)lane == leader) at = atomicAdd(&S.nhard, (uint32_t)__popc(dm));
            at = __shfl_sync(kFull, at, leader);
            if (defer) S.hardq[at + __popc(dm & ((1u << lane) - 1u))] = (uint16_t)q;
          }
          const bool go = active && !defer;
          const uint32_t g = base + q;
          bool live = true;
          if (go) {
            // pass 0 flies only paths that cannot reach the body
            if (p.flags & kDoMove)
              live = pass == 0 ? move_free(p, pos, vel, g, step) : move_particle(p, pos, vel, g, step);
            if (do_sample) { U[j] = vel.x; V[j] = vel.y; W[j] = vel.z; }
            if (!vel_only) { p.out.x[g] = pos.x; p.out.y[g] = pos.y; p.out.z[g] = pos.z; }
            p.out.u[g] = vel.x; p.out.v[g] = vel.y; p.out.w[g] = vel.z;
          }
          if (do_keys) {
            const bool has_key = go && live;
            const unsigned m = __ballot_sync(kFull, has_key);
            if (go && !live) removed++;
            if (has_key) {
              const uint32_t key = cell_id3d(p.grid, pos.x, pos.y, pos.z);
              warp_count_key(p.count, key, m, s_tile);
              p.out_key[g] = key;
            } else if (go) {
              p.out_key[g] = kDeadKey;
            }
          }
        }
        if (split && pass == 0) __syncthreads();  // the queue is complete
      }
      // D: sampling
      if (do_sample) {
        __syncthreads();
        for (uint32_t lc = tid; lc < k; lc += blockDim.x) {
          const uint32_t s0 = ls[cur + lc] - base, e0 = ls[cur + lc + 1] - base;
          SmemVel a{U, V, W, S.slot, s0};
          sample_cell(p.acc, p.cells, cs + lc, (int)(e0 - s0), a);
        }
      }
    }
    __syncthreads();
    if (tid == 0) S.cur = S.next;
    __syncthreads();
  }
  if (do_keys) flush_tile_hist(s_tile, p.tile_sum, p.n_scan_tiles);
  const unsigned long long s64 = warp_sum((unsigned long long)sel);
  const unsigned long long c64 = warp_sum((unsigned long long)col);
  const double g = warp_sum(sum_g);
  const uint32_t r = warp_sum(removed);
  if (lane_id() == 0 && p.meta) {
    if (s64) atomicAdd(&p.meta->selections, s64);
    if (c64) atomicAdd(&p.meta->collisions, c64);
    if (g != 0.0) atomicAdd(&p.meta->sum_g, g);
    if (r) atomicAdd(&p.meta->removed, r);
  }
  if (do_sample && p.meta && blockIdx.x == 0 && tid == 0) atomicAdd(&p.meta->samples, 1u);
}

// Shared-memory attribute and occupancy of a variant, per device and
// histogram size (host-side cache; a launch needs neither query again).
struct LaunchShape {
  int device = -1;
  uint32_t n_scan_tiles = 0;
  int per_sm = 0;
};

template <int THREADS, int CAP, int MINB>
cudaError_t launch_variant(const StepParams& p, cudaStream_t stream) {
  static LaunchShape cache[8];
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  LaunchShape& ls = cache[dev & 7];
  const size_t smem = smem_bytes<CAP>(p.n_scan_tiles);
  if (ls.device != dev || ls.n_scan_tiles != p.n_scan_tiles) {
    e = cudaFuncSetAttribute(k_cell<THREADS, CAP, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cell<THREADS, CAP, MINB>, THREADS,
                                                      smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    ls.device = dev;
    ls.n_scan_tiles = p.n_scan_tiles;
    ls.per_sm = per_sm;
  }
  uint32_t grid = (uint32_t)(num_sms() * ls.per_sm);
  if (grid > p.n_tiles) grid = p.n_tiles;
  if (grid == 0) return cudaSuccess;
  k_cell<THREADS, CAP, MINB><<<grid, THREADS, smem, stream>>>(p);
  return cudaGetLastError();
}

}  // namespace

// Variants 0-3: the CTA-wide kernel above; 4-7: the warp-autonomous kernel
// (dsmc_cellw.cu), which handles the full step with padded buffers (the
// collide stage, kVelOnly on caller buffers, always runs the CTA-wide one).
int cell_kernel_variants() { return 4 + cell_kernel_w_variants(); }

int cell_kernel_chunk_capacity(int variant) {
  static const int caps[4] = {2048, 1024, 512, 256};
  if (variant >= 4) return cell_kernel_w_capacity(variant - 4);
  return caps[variant < 0 ? 2 : variant];
}

bool cell_kernel_is_warp(int variant) { return variant >= 4; }

cudaError_t launch_cell(const StepParams& p, cudaStream_t stream) {
  if (p.cell_variant >= 4 && (p.flags & kPadded) && !(p.flags & kVelOnly))
    return launch_cell_w(p, p.cell_variant - 4, stream);
  switch (p.cell_variant) {
    case 0: return launch_variant<512, 2048, 1>(p, stream);
    case 1: return launch_variant<256, 1024, 2>(p, stream);
    case 3: return launch_variant<64, 256, 8>(p, stream);
    default: return launch_variant<128, 512, 4>(p, stream);
  }
}

}  // namespace dsmcb
