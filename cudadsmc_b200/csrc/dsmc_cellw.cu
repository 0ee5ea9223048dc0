// The timestep's cell work as warp-autonomous kernels (sm_100a); none has a
// CTA-wide barrier inside its loop.
//
// k_order_w (order + pair counts): warps take tiles of 32 consecutive cells
// (lane L owns cell L; tiles past the first wave come from a dynamic counter)
// and cut them into chunks of whole cells holding at most CAPW particles.  A
// chunk's orig (the pre-scatter index of every sorted slot) is staged in the
// warp's slice of shared memory by a 1-D bulk copy completing on the warp's
// mbarrier, double buffered (the next chunk's copy is in flight while the
// current one is processed); then
//   A  the chunk's state is gathered from the unsorted array through orig by
//      asynchronous 4-byte copies, while the cell of each slot (binary search
//      of the chunk's cell starts) and its rank by orig inside the cell (the
//      stable order of the reference's sort) are computed
//   B  NTC pair counts (and remainders); cells with pairs are listed
//   C  the chunk goes to the mid arrays in sorted order
// k_ntc_w: the listed cells' NTC selections in place on the mid arrays, a
// lane per light cell, a warp per dense cell (Philox mode).
// k_flight_w (flight + keys): streams the sorted particles, 32 at a time per
// warp in grid-stride order: free flight and boundaries, next-step key and
// count (warp-aggregated atomics on the per-cell counts and on the per scan
// tile totals).  Flights that may reach the body are listed instead: they
// cluster next to the body, so k_mesh_w flies them afterwards one per thread
// over the whole GPU.  k_sample_w samples (FP64) on sampling steps.
//
// The per-cell and per-particle arithmetic is that of the fused CTA-wide
// kernel (dsmc_cell.cu), in the same order, so both compute the same step for
// every cell that fits a chunk.  Gathering through orig lets the scatter write
// orig alone (one scattered 4-byte store per particle instead of seven).
//
// Traffic per particle: k_order_w orig 4 + state 24 read, 24 written;
// k_flight_w 24 read, 24 + key 4 written.  Per cell: 8 B of starts, 16 B of
// (sigma g)max read + written, 32 B more in the reference RNG mode, 80 B of
// sampling sums on sampling steps.
#include "dsmc_bulk.cuh"
#include "dsmc_step_dev.cuh"

namespace dsmcb {
namespace {

using namespace dev;

constexpr uint32_t kWarpTile = 32;  // cells per warp tile, one per lane
constexpr uint32_t kFlightQ = 64;   // per-warp queue of flights that may reach the body

template <int CAPW>
struct __align__(16) WarpSmem {
  static constexpr int kOrig = 6;  // orig's row in part
  float part[2][7][CAPW + 8];  // x y z u v w orig of a chunk, double buffered
  uint4 lbuf[2 * kWarpTile];   // light-cell list entries not yet in the global list
  uint32_t cr[kWarpTile];      // the chunk's nonempty cells in order: start | end << 16 (chunk-relative)
  unsigned long long mbar[2];
};

template <int CAPW, int WARPS>
constexpr size_t collide_smem_bytes() {
  return WARPS * sizeof(WarpSmem<CAPW>);
}

// A tile of 32 cells as the lanes see it: lane L holds the start and end of
// cell 32 t + L (cells past the last one are empty at the total count).
struct WTile {
  uint32_t t, nct, s, e;
};

__device__ __forceinline__ WTile load_tile(const StepParams& p, uint32_t t) {
  WTile w;
  w.t = t;
  w.nct = 0;
  w.s = w.e = 0;
  if (t < p.n_tiles) {
    const uint32_t c0 = t * kWarpTile;
    const uint32_t c = c0 + lane_id();
    w.nct = min(kWarpTile, p.cells - c0);
    w.s = __ldg(&p.start[min(c, p.cells)]);
    w.e = __ldg(&p.start[min(c + 1u, p.cells)]);
  }
  return w;
}

// Tiles of a warp: tile w first, then from the step's dynamic counter (or
// round robin without one).  Lane 0 asks ahead of need so that the atomic's
// latency is hidden.
struct TileQueue {
  uint32_t nwarps, next_static;
  uint32_t* counter;
  __device__ __forceinline__ uint32_t grab() {
    if (counter) return nwarps + atomicAdd(counter, 1u);
    const uint32_t t = next_static;
    next_static += nwarps;
    return t;
  }
};

// Chunk of a tile: cells [cur, cur + k) holding particles [base, base + n).
struct WChunk {
  uint32_t cur, k, base, n;
  int buf, giant, valid;
};

// As many whole cells from `cur` as fit CAPW particles (a single cell that
// does not fit is a giant chunk).  Warp-uniform; cur < T.nct.
template <int CAPW>
__device__ __forceinline__ WChunk make_wchunk(const WTile& T, uint32_t cur, int buf) {
  WChunk c;
  c.cur = cur;
  c.buf = buf;
  c.valid = 1;
  const uint32_t lane = lane_id();
  c.base = __shfl_sync(kFull, T.s, cur);
  // ends grow with the lane: the cells that fit are a prefix from cur
  const bool fits = lane >= cur && lane < T.nct && T.e - c.base <= (uint32_t)CAPW;
  const uint32_t k = __popc(__ballot_sync(kFull, fits));
  c.giant = k == 0;
  c.k = k == 0 ? 1u : k;
  c.n = __shfl_sync(kFull, T.e, cur + c.k - 1u) - c.base;
  return c;
}

// Bulk copy of a chunk's orig (the pre-scatter index of every sorted slot)
// into buffer c.buf.  The library's buffers carry 16 bytes of slack, so the
// whole 16-byte aligned cover of [base, base + n) is copied (at most CAPW + 6
// elements).
template <class Smem>
__device__ __forceinline__ void issue_wchunk(const StepParams& p, Smem& S, const WChunk& c) {
  const uint32_t ia = c.base & ~3u, ib = (c.base + c.n + 3u) & ~3u;
  const uint32_t bytes = (ib - ia) * 4u;
  const uint32_t lane = lane_id();
  if (lane == 0) mbar_expect_tx(&S.mbar[c.buf], bytes);
  __syncwarp();
  if (lane == 0) {
    fence_proxy_async();
    bulk_g2s(S.part[c.buf][Smem::kOrig], p.in_orig + ia, bytes, &S.mbar[c.buf]);
  }
}

// A cell too large for a chunk: the warp gathers it in sorted order into the
// mid arrays in global memory; its pairs are collided by one lane of k_ntc_w
// (the cell is listed as a light cell whatever its pair count).
static __device__ __noinline__ void giant_order_warp(const StepParams& p, uint32_t s, uint32_t e) {
  const uint32_t n = e - s;
  const uint32_t lane = lane_id();
  if (lane == 0 && p.meta) atomicAdd(&p.meta->giant_cells, 1u);
  for (uint32_t i = lane; i < n; i += 32) {
    const uint32_t my = p.in_orig[s + i];
    uint32_t rank = 0;
    for (uint32_t j = 0; j < n; j++) rank += (uint32_t)(p.in_orig[s + j] < my);
    const uint32_t d = s + rank;
    p.mid.x[d] = p.in.x[my]; p.mid.y[d] = p.in.y[my]; p.mid.z[d] = p.in.z[my];
    p.mid.u[d] = p.in.u[my]; p.mid.v[d] = p.in.v[my]; p.mid.w[d] = p.in.w[my];
  }
}

// Descents of orig inside a chunk (OR: its n origs).  A cell without one is
// in stable order already (its particles took their tickets in one or a few
// increasing runs, the common case) and a slot's rank there is its position;
// only cells with a descent count smaller origs.  True for the lanes whose
// nonempty cell (chunk-relative start s0, nc particles) has one.  All lanes
// call it.
template <int CAPW>
__device__ __forceinline__ bool cell_has_descent(const uint32_t* OR, uint32_t n, bool ne, uint32_t s0,
                                                 uint32_t nc) {
  const uint32_t lane = lane_id();
  uint32_t dw[CAPW / 32];
#pragma unroll
  for (int k = 0; k < CAPW / 32; k++) {
    const uint32_t t = 32u * k + lane;
    dw[k] = __ballot_sync(kFull, t > 0 && t < n && OR[t - 1] > OR[t]);
  }
  bool unsorted = false;
  if (ne && nc > 1) {
    const uint32_t lo_b = s0 + 1u, hi_b = s0 + nc;
#pragma unroll
    for (int k = 0; k < CAPW / 32; k++) {
      const uint32_t w0 = 32u * k;
      const uint32_t l = max(lo_b, w0), h = min(hi_b, w0 + 32u);
      if (l < h) {
        const uint32_t m = (uint32_t)(((1ull << (h - w0)) - 1ull) & ~((1ull << (l - w0)) - 1ull));
        unsorted |= (dw[k] & m) != 0u;
      }
    }
  }
  return unsorted;
}

// Position in stable (cell, orig) order of chunk slot t = b0 + lane (orig
// `my`; t itself for t >= n).  Its cell is the last nonempty cell starting at
// or before t, found by its ordinal among them: the lanes stand for the
// tile's cells (chunk-relative start s0, nonempty `ne`), giving the starts in
// [b0, b0 + 32) as a bit mask and the count before.  In a cell flagged with a
// descent (bit 31 of its `cr` entry: start | end << 16) the rank is the
// number of smaller origs there; ORA holds the chunk's origs from offset
// `off`.  All lanes call it.
__device__ __forceinline__ uint32_t stable_slot(const uint32_t* ORA, const uint32_t* cr, uint32_t off,
                                                uint32_t b0, uint32_t n, uint32_t my, bool ne,
                                                uint32_t s0) {
  const uint32_t lane = lane_id(), t = b0 + lane;
  const unsigned starts =
      __reduce_or_sync(kFull, (ne && s0 >= b0 && s0 < b0 + 32u) ? 1u << (s0 - b0) : 0u);
  const uint32_t before = __popc(__ballot_sync(kFull, ne && s0 < b0));
  uint32_t pos = t;
  if (t < n) {
    const uint32_t ab = cr[before + __popc(starts & (0xffffffffu >> (31u - lane))) - 1u];
    if (ab >> 31) {
      const uint32_t a = ab & 0xffffu, b = (ab >> 16) & 0x7fffu;
      uint32_t rank = 0;
      // one element per step: the lanes of a cell read the same word (a
      // broadcast), and lanes of different cells only differ in the trip
      // count (a 16-byte form with edge cases diverged in both)
      for (uint32_t j = a + off; j < b + off; j++) rank += (uint32_t)(ORA[j] < my);
      pos = a + rank;
    }
  }
  return pos;
}

// Appends e for every lane with `put` to list (one atomic per warp; all lanes
// call it).
__device__ __forceinline__ void list_cells(uint4* list, uint32_t* counter, bool put, uint4 e) {
  const uint32_t lane = lane_id();
  const unsigned m = __ballot_sync(kFull, put);
  if (!m) return;
  const int leader = __ffs(m) - 1;
  uint32_t base = 0;
  if ((int)lane == leader) base = atomicAdd(counter, (uint32_t)__popc(m));
  base = __shfl_sync(kFull, base, leader);
  if (put) list[base + __popc(m & ((1u << lane) - 1u))] = e;
}

// Adds v, summed over the block, to *dst with one atomic (every thread of the
// block calls it; s_red holds a slot per warp).  Per-warp atomics on one
// address from every warp of a full-GPU pass serialise in L2 at the end of
// the kernel, which then waits for them.
template <class T>
__device__ __forceinline__ void block_add(T* dst, T v, T* s_red) {
  v = warp_sum(v);
  if (lane_id() == 0) s_red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    T t = s_red[0];
    for (uint32_t w = 1; w < (blockDim.x >> 5); w++) t += s_red[w];
    if (t != T(0)) atomicAdd(dst, t);
  }
}

// Appends e for every lane with `put` to the warp's buffer `buf` (cnt entries,
// fewer than 32 between calls) and moves 32 at a time to the global list: one
// returning atomic on the list's counter per 32 entries instead of one per
// call, which every warp of the grid would otherwise wait on.
__device__ __forceinline__ void buffer_cells(uint4* buf, uint32_t& cnt, uint4* list,
                                             uint32_t* counter, bool put, uint4 e) {
  const uint32_t lane = lane_id();
  const unsigned m = __ballot_sync(kFull, put);
  if (put) buf[cnt + __popc(m & ((1u << lane) - 1u))] = e;
  cnt += __popc(m);
  if (cnt >= 32) {
    __syncwarp();
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(counter, 32u);
    base = __shfl_sync(kFull, base, 0);
    list[base + lane] = buf[lane];
    cnt -= 32;
    __syncwarp();
    if (lane < cnt) buf[lane] = buf[32 + lane];
    __syncwarp();
  }
}

// The rest of the buffer (cnt < 32 entries) to the global list.
__device__ __forceinline__ void flush_cells(const uint4* buf, uint32_t cnt, uint4* list,
                                            uint32_t* counter) {
  if (!cnt) return;
  const uint32_t lane = lane_id();
  __syncwarp();
  uint32_t base = 0;
  if (lane == 0) base = atomicAdd(counter, cnt);
  base = __shfl_sync(kFull, base, 0);
  if (lane < cnt) list[base + lane] = buf[lane];
}

// ---------------------------------------------------- order + pair counts ----

// The order kernel's body for block vb of vg (the launch's grid, or a
// member's share of a batched launch).
template <int CAPW, int WARPS>
__device__ __forceinline__ void order_body(const StepParams& p, const uint32_t vb, const uint32_t vg) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  using Smem = WarpSmem<CAPW>;
  Smem& S = reinterpret_cast<Smem*>(smem_raw)[warp];
  const bool do_fixup = (p.flags & kDoFixup) != 0;
  const bool do_collide = (p.flags & kDoCollide) != 0;
  const bool taus = p.rng_kind == 0;
  const bool heavy_mode = !taus && do_collide;
  if (lane == 0) {
    mbar_init(&S.mbar[0], 1);
    mbar_init(&S.mbar[1], 1);
    fence_mbar_init();
  }
  __syncwarp();

  const uint32_t nwarps = vg * WARPS;
  const uint32_t gw = vb * WARPS + warp;
  TileQueue tq{nwarps, gw + nwarps, p.meta ? &p.meta->tile_next : nullptr};
  WTile A = load_tile(p, gw);
  uint32_t pend = 0, tb = 0;
  if (lane == 0 && gw < p.n_tiles) {
    tb = tq.grab();
    pend = tq.grab();
  }
  tb = __shfl_sync(kFull, gw < p.n_tiles ? tb : 0xffffffffu, 0);
  WTile B = load_tile(p, tb);

  uint32_t phase = 0;  // bit b: parity of the next phase of buffer b
  uint32_t sel = 0;
  uint32_t lcnt = 0;   // entries in S.lbuf
  WChunk C;
  C.valid = 0;
  // the previous chunk, gathered into its buffer's state rows by copies that
  // may still be in flight, written out once the next chunk's gathers are
  // issued (P.valid == 0: none)
  WChunk P;
  P.valid = 0;
  // writes chunk (base, n) from state buffer b to the mid arrays
  auto write_chunk = [&](uint32_t b, uint32_t base, uint32_t n) {
    const uint32_t o = base & 3u;
    const float* X = S.part[b][0] + o;
    const float* Y = S.part[b][1] + o;
    const float* Z = S.part[b][2] + o;
    const float* U = S.part[b][3] + o;
    const float* V = S.part[b][4] + o;
    const float* W = S.part[b][5] + o;
    for (uint32_t q = lane; q < n; q += 32) {
      const uint32_t g = base + q;
      p.mid.x[g] = X[q]; p.mid.y[g] = Y[q]; p.mid.z[g] = Z[q];
      p.mid.u[g] = U[q]; p.mid.v[g] = V[q]; p.mid.w[g] = W[q];
    }
  };
  // the pending chunk, once every gather but the newest group has landed
  // (all of them with `all`)
  auto write_pending = [&](bool all) {
    if (!P.valid) return;
    if (all) cp_async_wait_all();
    else cp_async_wait_prior();
    __syncwarp();
    write_chunk(P.buf, P.base, P.n);
    __syncwarp();
    P.valid = 0;
  };
  // (sigma g)max and remainder of a chunk's cells, loaded one chunk ahead
  float2 mr_c = make_float2(0.f, 0.f);
  auto load_cell_state = [&](const WChunk& K, uint32_t tile, float2& mr) {
    if (do_collide && K.valid && !K.giant && K.n && lane >= K.cur && lane < K.cur + K.k)
      mr = p.maxrem[tile * kWarpTile + lane];
  };
  if (A.t < p.n_tiles) {
    C = make_wchunk<CAPW>(A, 0, 0);
    if (!C.giant && C.n) issue_wchunk(p, S, C);
    load_cell_state(C, A.t, mr_c);
  }

  while (C.valid) {
    // the chunk after this one, and its copy into the other buffer
    WChunk N;
    N.valid = 0;
    bool n_in_b = false;
    if (C.cur + C.k < A.nct) {
      N = make_wchunk<CAPW>(A, C.cur + C.k, C.buf ^ 1);
    } else if (B.t < p.n_tiles) {
      N = make_wchunk<CAPW>(B, 0, C.buf ^ 1);
      n_in_b = true;
    }
    const bool n_copy = N.valid && !N.giant && N.n;
    if (n_copy) issue_wchunk(p, S, N);
    float2 mr_n = make_float2(0.f, 0.f);
    load_cell_state(N, n_in_b ? B.t : A.t, mr_n);

    const uint32_t c0 = A.t * kWarpTile;
    const uint32_t cell = c0 + lane;
    const bool mine = lane >= C.cur && lane < C.cur + C.k;
    const uint32_t s0 = A.s - C.base, nc = A.e - A.s;  // meaningful for `mine`
    const bool ne = mine && nc > 0;
    const uint32_t ne_idx = __popc(__ballot_sync(kFull, ne) & ((1u << lane) - 1u));
    if (!C.giant && C.n) {
      if (ne) S.cr[ne_idx] = s0 | ((s0 + nc) << 16);
      const uint32_t par = (phase >> C.buf) & 1u;
      bool ok = mbar_wait_bounded(&S.mbar[C.buf], par);
      phase ^= 1u << C.buf;
      if (!__all_sync(kFull, ok)) {
        if (lane == 0 && p.meta) atomicOr(&p.meta->error, kErrTimeout);
        // this chunk's and the next chunk's copies may still be in flight:
        // let them land (again bounded) before the shared memory goes away
        mbar_wait_bounded(&S.mbar[C.buf], par);
        if (n_copy) mbar_wait_bounded(&S.mbar[N.buf], (phase >> N.buf) & 1u);
        cp_async_wait_all();
        P.valid = 0;
        break;
      }
    }
    __syncwarp();

    if (C.giant) {
      // the chunk after it reuses the pending chunk's buffer
      write_pending(true);
      giant_order_warp(p, C.base, C.base + C.n);
      if (do_collide) {
        // the giant cell's pair count, from lane C.cur's (sigma g)max
        const uint32_t gc = c0 + C.cur;
        uint32_t M = 0;
        if (lane == C.cur) {
          float2 vm = p.maxrem[gc];
          M = taus ? ntc_pairs_reference(p, (int)C.n, vm) : ntc_pairs_fast(p, C.n, vm);
          p.maxrem[gc] = vm;
          sel += M;
        }
        buffer_cells(S.lbuf, lcnt, p.ntc_light, &p.meta->n_light, lane == C.cur && M > 0,
                     make_uint4(gc, C.base, C.n, M));
      }
    } else if (C.n > 0) {
      // a pending chunk in this chunk's buffer (an empty chunk came between)
      if (P.valid && P.buf == C.buf) write_pending(true);
      const uint32_t off = C.base & 3u;
      const uint32_t* OR = reinterpret_cast<const uint32_t*>(S.part[C.buf][Smem::kOrig] + off);
      // element j of the chunk sits at ORA[j + off]
      const uint32_t* ORA = reinterpret_cast<const uint32_t*>(S.part[C.buf][Smem::kOrig]);
      const uint32_t base = C.base, n = C.n;
      float* X = S.part[C.buf][0] + off;
      float* Y = S.part[C.buf][1] + off;
      float* Z = S.part[C.buf][2] + off;
      float* U = S.part[C.buf][3] + off;
      float* V = S.part[C.buf][4] + off;
      float* W = S.part[C.buf][5] + off;
      // A: each particle's sorted position, sorted = (cell, orig), then the
      // gather of its state through orig straight to that position
      // (asynchronous 4-byte copies, in flight while the pair counts run).
      // The origs are distinct, so a particle's rank in its cell is the
      // number of smaller origs there.
      // (strips of 32 slots without a cell that has a descent keep their
      // order)
      bool desc = false;
      if (do_fixup) {
        desc = cell_has_descent<CAPW>(OR, n, ne, s0, nc);
        if (desc) S.cr[ne_idx] |= 0x80000000u;
        __syncwarp();
      }
      const bool any_desc = __any_sync(kFull, desc);
      for (uint32_t b0 = 0; b0 < n; b0 += 32) {
        const uint32_t t = b0 + lane;
        const uint32_t my = t < n ? OR[t] : 0u;
        const bool rank = any_desc && __any_sync(kFull, desc && s0 < b0 + 32u && s0 + nc > b0);
        const uint32_t pos = rank ? stable_slot(ORA, S.cr, off, b0, n, my, ne, s0) : t;
        if (t < n) {
          cp_async4(X + pos, p.in.x + my);
          cp_async4(Y + pos, p.in.y + my);
          cp_async4(Z + pos, p.in.z + my);
          cp_async4(U + pos, p.in.u + my);
          cp_async4(V + pos, p.in.v + my);
          cp_async4(W + pos, p.in.w + my);
        }
      }
      // B: pair counts (the new remainder is stored now); cells with pairs
      // are listed for k_ntc_w, light ones to get a lane, dense ones a warp
      if (do_collide) {
        uint32_t M = 0;
        if (mine && nc >= 2) {
          float2 vm = mr_c;
          M = taus ? ntc_pairs_reference(p, (int)nc, vm) : ntc_pairs_fast(p, nc, vm);
          p.maxrem[cell] = vm;
          sel += M;
        }
        const bool heavy = heavy_mode && M >= kHeavyMin;
        const uint4 e = make_uint4(cell, base + s0, nc, M);
        buffer_cells(S.lbuf, lcnt, p.ntc_light, &p.meta->n_light, M > 0 && !heavy, e);
        list_cells(p.ntc_heavy, &p.meta->n_heavy, heavy, e);
      }
      cp_async_commit();
      // C: the previous chunk, in sorted order, to the mid arrays while this
      // one's gathers are in flight; this one waits for the next
      write_pending(false);
      P = C;
    }
    __syncwarp();
    if (n_in_b) {
      A = B;
      const uint32_t t2 = __shfl_sync(kFull, pend, 0);
      B = load_tile(p, t2);
      if (lane == 0 && t2 < p.n_tiles) pend = tq.grab();
    }
    C = N;
    mr_c = mr_n;
  }
  write_pending(true);
  if (do_collide) flush_cells(S.lbuf, lcnt, p.ntc_light, &p.meta->n_light);
  __shared__ unsigned long long s_red[WARPS];
  if (p.meta) block_add(&p.meta->selections, (unsigned long long)sel, s_red);
}

template <int CAPW, int WARPS, int MINB>
__global__ void __launch_bounds__(WARPS * 32, MINB) k_order_w(const __grid_constant__ StepParams p) {
  chained_entry();
  order_body<CAPW, WARPS>(p, blockIdx.x, gridDim.x);
}
template <int CAPW, int WARPS, int MINB>
__global__ void __launch_bounds__(WARPS * 32, MINB) k_order_wb(const __grid_constant__ BatchOf<StepParams> bv) {
  chained_entry();
  uint32_t vb, vg;
  const StepParams& p = bv.locate(vb, vg);
  order_body<CAPW, WARPS>(p, vb, vg);
}

// ------------------------------------------------------- NTC selections ----

constexpr uint32_t kNtcClaim = 256;  // claim slots per warp: the largest chunk

// The NTC selections of the cells k_order_w listed, in place on the sorted
// post-collision state p.mid: a lane per light cell, a warp per dense cell
// (at most kNtcClaim particles: larger cells were collided by k_order_w).
// The pair counts and remainders come from k_order_w; this kernel updates
// (sigma g)max (and the HybridTaus state in the reference RNG mode) with the
// same arithmetic and random streams as the fused path.  The grid is one
// wave: dense cells (the longest chains) go first, a warp each, then warps
// claim light cells 32 at a time, so that the warps that finish early take
// more (with a static split the blocks holding both a second round of light
// cells and a dense cell set the kernel's length).
template <int WARPS>
__device__ __forceinline__ void ntc_body(const StepParams& p, const uint32_t vb, const uint32_t vg) {
  __shared__ uint32_t s_claim[WARPS][kNtcClaim];
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const uint32_t step = p.step_override ? p.step_override : p.meta->step;
  const bool taus = p.rng_kind == 0;
  for (uint32_t t = lane; t < kNtcClaim; t += 32) s_claim[warp][t] = 0xffffffffu;
  __syncwarp();
  uint32_t col = 0;
  double sum_g = 0.0;
  const uint32_t nl = p.meta->n_light, nh = p.meta->n_heavy;
  const uint32_t gw = vb * WARPS + warp, nw = vg * WARPS;
  for (uint32_t h = gw; h < nh; h += nw) {
    const uint4 e = p.ntc_heavy[h];
    GlobalVel acc{p.mid.u, p.mid.v, p.mid.w, e.y};
    const float2 vm = p.maxrem[e.x];  // .y: the remainder k_order_w stored
    const float vmax =
        ntc_select_heavy_warp(p, e.x, e.z, acc, s_claim[warp], step, e.w, vm.x, col, sum_g);
    __syncwarp();
    if (lane == 0) p.maxrem[e.x] = make_float2(vmax, vm.y);
  }
  uint32_t* claims = &p.meta->tile_next2;
  uint32_t next = 0;
  if (lane == 0) next = atomicAdd(claims, 32u);
  for (uint32_t base = __shfl_sync(kFull, next, 0); base < nl;) {
    // the claim after this one, asked for ahead of need
    if (lane == 0) next = atomicAdd(claims, 32u);
    const uint32_t i = base + lane;
    base = __shfl_sync(kFull, next, 0);
    if (i >= nl) continue;
    const uint4 e = p.ntc_light[i];  // cell, first sorted slot, count, pairs
    GlobalVel acc{p.mid.u, p.mid.v, p.mid.w, e.y};
    float2 vm = p.maxrem[e.x];
    if (taus) {
      TausRng r;
      r.s = p.seeds[e.x];
      float4 stat = make_float4(0.f, 0.f, 0.f, 0.f);
      ntc_select_reference(p, (int)e.z, acc, r, e.w, vm, stat, col, sum_g);
      p.seeds[e.x] = r.s;
    } else {
      col += ntc_select_fast(p, e.x, e.z, acc, step, e.w, vm, sum_g);
    }
    p.maxrem[e.x] = vm;
  }
  __shared__ unsigned long long s_col[WARPS];
  __shared__ double s_g[WARPS];
  if (p.meta) {
    block_add(&p.meta->collisions, (unsigned long long)col, s_col);
    block_add(&p.meta->sum_g, sum_g, s_g);
  }
}

template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_ntc_w(const __grid_constant__ StepParams p) {
  chained_entry();
  ntc_body<WARPS>(p, blockIdx.x, gridDim.x);
}
template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_ntc_wb(const __grid_constant__ BatchOf<StepParams> bv) {
  chained_entry();
  uint32_t vb, vg;
  const StepParams& p = bv.locate(vb, vg);
  ntc_body<WARPS>(p, vb, vg);
}

// ------------------------------------------------ flight + keys + sample ----

// Next-step key and count of a flown particle (all lanes; `go`: this lane
// flew one), its state stored at g.  The count goes to count[key]; the scan
// tile's total to the block's histogram s_tile when given (flushed by the
// caller), else straight to tile_sum.  Per group the tile atomic lands on one
// of a few hundred addresses: from every warp of a full-GPU pass these
// serialise in L2 (70 of the flight kernel's 125 us on 3.7M particles), so
// the streaming kernels count tiles in shared memory.
__device__ __forceinline__ void finish_flight(const StepParams& p, bool go, bool live, uint32_t g,
                                              float3 pos, float3 vel, uint32_t& removed,
                                              uint32_t* s_tile = nullptr) {
  if (go) {
    p.out.x[g] = pos.x; p.out.y[g] = pos.y; p.out.z[g] = pos.z;
    p.out.u[g] = vel.x; p.out.v[g] = vel.y; p.out.w[g] = vel.z;
  }
  if (p.flags & kDoKeys) {
    const bool has_key = go && live;
    const unsigned m = __ballot_sync(kFull, has_key);
    if (go && !live) removed++;
    if (has_key) {
      const uint32_t key = cell_id3d(p.grid, pos.x, pos.y, pos.z);
      if (s_tile)
        warp_count_key(p.count, key, m, s_tile);
      else
        warp_count_key_global(p.count, key, m, p.tile_sum);
      p.out_key[g] = key;
    } else if (go) {
      p.out_key[g] = kDeadKey;
    }
  }
}

// Appends q[from, from + cnt) (cnt <= 32) to the step's list of flights that
// may reach the body (one atomic per call).
__device__ __forceinline__ void list_deferred(const StepParams& p, const uint32_t* q, uint32_t from,
                                              uint32_t cnt) {
  const uint32_t lane = lane_id();
  uint32_t base = 0;
  if (lane == 0) base = atomicAdd(&p.meta->n_defer, cnt);
  base = __shfl_sync(kFull, base, 0);
  if (lane < cnt) p.defer_list[base + lane] = q[from + lane];
}

// Free flights of the sorted particles [0, n_alive), read from p.mid (the
// state k_order_w and k_ntc_w produced) and written to p.out.  Each warp
// takes a contiguous run of groups of 32 (the work per particle is even once
// the flights that may reach the body are listed for k_mesh_w, which spreads
// them over the whole GPU: they cluster next to the body); a warp's listed
// flights are then neighbours, so each 32-entry chunk of the list holds
// flights through the same few geometry cells for one warp of k_mesh_w.  The
// state of a group is loaded two iterations ahead, and in nearest mode the
// clearance lookup of its deferral test one iteration ahead, so that both
// latencies are covered.
template <int WARPS>
__device__ __forceinline__ void flight_body(const StepParams& p, const uint32_t vb, const uint32_t vg) {
  __shared__ uint32_t s_q[WARPS][kFlightQ];
  extern __shared__ uint32_t s_tile[];  // this block's next-step counts per scan tile
  for (uint32_t t = threadIdx.x; t < p.n_scan_tiles; t += blockDim.x) s_tile[t] = 0;
  __syncthreads();
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const uint32_t step = p.step_override ? p.step_override : p.meta->step;
  const uint32_t n = p.meta->n_alive;
  const bool do_move = (p.flags & kDoMove) != 0;
  const bool split = p.has_geom && do_move;
  const bool piped = split && p.geom.nearest;
  uint32_t* q = s_q[warp];
  // this warp's groups: per of the ceil(n / 32) groups from gb, particles [gb * 32, end)
  const uint32_t ngroups = (n + 31u) / 32u, nwarps = vg * WARPS;
  const uint32_t per = (ngroups + nwarps - 1u) / nwarps;
  const uint32_t gb = min((vb * WARPS + warp) * per, ngroups);
  const uint32_t end = min(min(gb + per, ngroups) * 32u, n);
  const uint32_t stride = 32u;
  const uint32_t g0 = gb * 32u + lane;
  auto load = [&](uint32_t g, float3& pos, float3& vel) {
    if (g < end) {
      pos = make_float3(p.mid.x[g], p.mid.y[g], p.mid.z[g]);
      vel = make_float3(p.mid.u[g], p.mid.v[g], p.mid.w[g]);
    }
  };
  const float3 zero = make_float3(0.f, 0.f, 0.f);
  float3 pos0 = zero, vel0 = zero;  // group g
  float3 pos1 = zero, vel1 = zero;  // group g + stride
  float3 pos2 = zero, vel2 = zero;  // group g + 2 stride
  load(g0, pos0, vel0);
  load(g0 + stride, pos1, vel1);
  float clr0 = -1.f;
  if (piped && g0 < end) clr0 = defer_lookup(p, pos0);
  uint32_t removed = 0, nq = 0;
  for (uint32_t g = g0; g - lane < end; g += stride) {
    const bool active = g < end;
    load(g + 2u * stride, pos2, vel2);
    float clr1 = -1.f;
    if (piped && g + stride < end) clr1 = defer_lookup(p, pos1);
    float3 pos = pos0, vel = vel0;
    bool defer = false;
    if (active && split)
      defer = piped ? defer_decide(p, pos, vel, clr0) : flight_may_meet_body(p, pos, vel);
    const unsigned dm = __ballot_sync(kFull, defer);
    if (defer) q[nq + __popc(dm & ((1u << lane) - 1u))] = g;
    nq += __popc(dm);
    const bool go = active && !defer;
    bool live = true;
    // a path that cannot reach the body
    if (go && do_move) live = move_free(p, pos, vel, g, step);
    finish_flight(p, go, live, g, pos, vel, removed, s_tile);
    if (nq >= 32) {
      __syncwarp();
      nq -= 32;
      list_deferred(p, q, nq, 32);
      __syncwarp();
    }
    pos0 = pos1; vel0 = vel1; clr0 = clr1;
    pos1 = pos2; vel1 = vel2;
  }
  if (nq) {
    __syncwarp();
    list_deferred(p, q, 0, nq);
  }
  __shared__ uint32_t s_rm[WARPS];
  if (p.meta) block_add(&p.meta->removed, removed, s_rm);
  __syncthreads();
  flush_tile_hist(s_tile, p.tile_sum, p.n_scan_tiles);
}

template <int WARPS, int MINB>
__global__ void __launch_bounds__(WARPS * 32, MINB) k_flight_w(const __grid_constant__ StepParams p) {
  chained_entry();
  flight_body<WARPS>(p, blockIdx.x, gridDim.x);
}
template <int WARPS, int MINB>
__global__ void __launch_bounds__(WARPS * 32, MINB) k_flight_wb(const __grid_constant__ BatchOf<StepParams> bv) {
  chained_entry();
  uint32_t vb, vg;
  const StepParams& p = bv.locate(vb, vg);
  flight_body<WARPS>(p, vb, vg);
}

// Paired form of k_flight_w: lane L flies particles 2L and 2L+1 of each group
// of 64, with 8-byte loads and stores (half the memory instructions) and two
// independent chains per lane.  A deferred particle's slot gets its unmoved
// state and a dead key here; k_mesh_w, which runs after this kernel, writes
// both again.
constexpr uint32_t kFlightQ2 = 128;

template <int WARPS, int MINB>
__global__ void __launch_bounds__(WARPS * 32, MINB) k_flight_pw(const __grid_constant__ StepParams p) {
  chained_entry();
  __shared__ uint32_t s_q[WARPS][kFlightQ2];
  extern __shared__ uint32_t s_tile[];  // this block's next-step counts per scan tile
  for (uint32_t t = threadIdx.x; t < p.n_scan_tiles; t += blockDim.x) s_tile[t] = 0;
  __syncthreads();
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const uint32_t step = p.step_override ? p.step_override : p.meta->step;
  const uint32_t n = p.meta->n_alive;
  const bool do_move = (p.flags & kDoMove) != 0;
  const bool do_keys = (p.flags & kDoKeys) != 0;
  const bool split = p.has_geom && do_move;
  uint32_t* q = s_q[warp];
  const uint32_t stride = gridDim.x * WARPS * 64u;
  struct Pair {
    float2 x, y, z, u, v, w;
  };
  // state of particles g, g + 1 (g even; g + 1 only below n)
  auto load = [&](uint32_t g, Pair& s) {
    if (g + 1u < n) {
      s.x = *reinterpret_cast<const float2*>(p.mid.x + g);
      s.y = *reinterpret_cast<const float2*>(p.mid.y + g);
      s.z = *reinterpret_cast<const float2*>(p.mid.z + g);
      s.u = *reinterpret_cast<const float2*>(p.mid.u + g);
      s.v = *reinterpret_cast<const float2*>(p.mid.v + g);
      s.w = *reinterpret_cast<const float2*>(p.mid.w + g);
    } else if (g < n) {
      s.x.x = p.mid.x[g]; s.y.x = p.mid.y[g]; s.z.x = p.mid.z[g];
      s.u.x = p.mid.u[g]; s.v.x = p.mid.v[g]; s.w.x = p.mid.w[g];
    }
  };
  const uint32_t g0 = (blockIdx.x * WARPS + warp) * 64u + 2u * lane;
  Pair nxt{};
  load(g0, nxt);
  uint32_t removed = 0, nq = 0;
  for (uint32_t g = g0; g - 2u * lane < n; g += stride) {
    const Pair cur = nxt;
    load(g + stride, nxt);
    float3 pos[2] = {make_float3(cur.x.x, cur.y.x, cur.z.x), make_float3(cur.x.y, cur.y.y, cur.z.y)};
    float3 vel[2] = {make_float3(cur.u.x, cur.v.x, cur.w.x), make_float3(cur.u.y, cur.v.y, cur.w.y)};
    bool active[2] = {g < n, g + 1u < n};
    bool defer[2] = {false, false};
#pragma unroll
    for (int k = 0; k < 2; k++)
      if (active[k] && split) defer[k] = flight_may_meet_body(p, pos[k], vel[k]);
#pragma unroll
    for (int k = 0; k < 2; k++) {
      const unsigned dm = __ballot_sync(kFull, defer[k]);
      if (defer[k]) q[nq + __popc(dm & ((1u << lane) - 1u))] = g + k;
      nq += __popc(dm);
    }
    bool live[2] = {true, true};
    uint32_t key[2] = {kDeadKey, kDeadKey};
#pragma unroll
    for (int k = 0; k < 2; k++) {
      const bool go = active[k] && !defer[k];
      // a path that cannot reach the body
      if (go && do_move) live[k] = move_free(p, pos[k], vel[k], g + k, step);
      if (do_keys) {
        const bool has_key = go && live[k];
        const unsigned m = __ballot_sync(kFull, has_key);
        if (go && !live[k]) removed++;
        if (has_key) {
          key[k] = cell_id3d(p.grid, pos[k].x, pos[k].y, pos[k].z);
          warp_count_key(p.count, key[k], m, s_tile);
        }
      }
    }
    if (active[1]) {
      *reinterpret_cast<float2*>(p.out.x + g) = make_float2(pos[0].x, pos[1].x);
      *reinterpret_cast<float2*>(p.out.y + g) = make_float2(pos[0].y, pos[1].y);
      *reinterpret_cast<float2*>(p.out.z + g) = make_float2(pos[0].z, pos[1].z);
      *reinterpret_cast<float2*>(p.out.u + g) = make_float2(vel[0].x, vel[1].x);
      *reinterpret_cast<float2*>(p.out.v + g) = make_float2(vel[0].y, vel[1].y);
      *reinterpret_cast<float2*>(p.out.w + g) = make_float2(vel[0].z, vel[1].z);
      if (do_keys) *reinterpret_cast<uint2*>(p.out_key + g) = make_uint2(key[0], key[1]);
    } else if (active[0]) {
      p.out.x[g] = pos[0].x; p.out.y[g] = pos[0].y; p.out.z[g] = pos[0].z;
      p.out.u[g] = vel[0].x; p.out.v[g] = vel[0].y; p.out.w[g] = vel[0].z;
      if (do_keys) p.out_key[g] = key[0];
    }
    while (nq >= 32) {
      __syncwarp();
      nq -= 32;
      list_deferred(p, q, nq, 32);
      __syncwarp();
    }
  }
  if (nq) {
    __syncwarp();
    list_deferred(p, q, 0, nq);
  }
  __shared__ uint32_t s_rm[WARPS];
  if (p.meta) block_add(&p.meta->removed, removed, s_rm);
  __syncthreads();
  flush_tile_hist(s_tile, p.tile_sum, p.n_scan_tiles);
}

// The listed flights, one particle per thread over the whole grid (the list's
// order does not matter: each particle's flight, key and count are its own).
//
// With nearest wall crossings the first leg of the warp's 32 flights is
// walked together: each lane lists the grid cells its path visits (the same
// walk as nearest_wall_hit), the warp then tests the planes of all those
// cells' triangles 32 at a time whatever flight and cell they belong to, the
// vertices of the triangles that pass in rounds of 32, and keeps per flight
// and cell the nearest crossing (the least (t, entry)).  Each lane then
// applies nearest_wall_hit's rule to its own cells in order - the running
// nearest crossing, the walk stopped at the first cell whose exit lies
// beyond it - so the answer is the one the lane alone would find, while the
// warp's memory rounds follow the total work rather than the slowest lane's
// cells times the most planes of a cell.  Paths over more than kCoopCells
// cells walk alone.  The rest of each flight (re-emission, later legs,
// boundaries) follows per lane.
constexpr int kCoopCells = 6;
constexpr int kCoopUnroll = 4;  // plane loads per lane per round
constexpr int kMeshWarps = 8;

struct MeshCoop {
  float ox[32], oy[32], oz[32], dx[32], dy[32], dz[32], dist[32];
  uint32_t cstart[32][kCoopCells];      // first entry of each visited cell
  uint32_t cpre[32][kCoopCells + 1];    // the lane's entries before cell j
  float texit[32][kCoopCells];
  uint32_t lpre[33];                    // the warp's entries before lane L
  unsigned long long best[32][kCoopCells];  // nearest (t bits, entry) per lane and cell
  uint2 cand[64];                       // candidate (entry, lane | cell << 8)
};

// The candidates cand[0, c) (c <= 32): the crossing of each with its lane's
// segment, kept if nearer than that cell's best.
__device__ __forceinline__ void coop_crossings(const GeomView& G, MeshCoop& S, uint32_t c) {
  const uint32_t lane = lane_id();
  if (lane < c) {
    const uint2 q = S.cand[lane];
    const uint32_t L = q.y & 0xffu, j = q.y >> 8;
    const float3 o = make_float3(S.ox[L], S.oy[L], S.oz[L]);
    const float3 d = make_float3(S.dx[L], S.dy[L], S.dz[L]);
    float t;
    if (entry_crossing(G, q.x, o, d, S.dist[L], &t)) {
      // +0 for -0: the key's order is the order of t, then of the entry
      const float tp = t + 0.f;
      atomicMin(&S.best[L][j], ((unsigned long long)__float_as_uint(tp) << 32) | q.x);
    }
  }
  __syncwarp();
}

// The first leg's nearest crossing for every lane of the warp (all lanes
// call it; walk = the lane has a leg).  Returns the lane's kLeg* code with
// L's t, e and P set; -1 when the lane's path is too long for the joint walk.
__device__ __forceinline__ int coop_first_leg(const GeomView& G, MeshCoop& S, bool walk, float3 o,
                                              NearestLeg& L) {
  const uint32_t lane = lane_id();
  DdaWalk w;
  if (walk) walk = dda_begin(G.grid, o, L.d, L.dist, w);
  int nc = 0;
  bool alone = false;
  if (walk) {
    const int max_iter = dda_max_iter(G.grid);
    for (int it = 0; it < max_iter; it++) {
      DdaNext nx;
      const bool more = dda_peek(w, nx);
      if (nc == kCoopCells) {
        alone = true;
        break;
      }
      S.cstart[lane][nc] = dda_cell(G.grid, w.X.i, w.Y.i, w.Z.i);
      S.texit[lane][nc] = nx.texit;
      nc++;
      if (!more) break;
      dda_take(w, nx);
    }
  }
  if (alone) nc = 0;
  S.ox[lane] = o.x; S.oy[lane] = o.y; S.oz[lane] = o.z;
  S.dx[lane] = L.d.x; S.dy[lane] = L.d.y; S.dz[lane] = L.d.z;
  S.dist[lane] = L.dist;
  // the visited cells' entry ranges and slabs, loaded together; a cell whose
  // slab the path stays outside contributes no entries
  uint2 se[kCoopCells];
  bool pass[kCoopCells];
#pragma unroll
  for (int j = 0; j < kCoopCells; j++) {
    se[j] = j < nc ? geo_ld(&G.start_end[S.cstart[lane][j]]) : make_uint2(0u, 0u);
    pass[j] = true;
  }
  if (G.slab) {
    float4 sl[kCoopCells];
#pragma unroll
    for (int j = 0; j < kCoopCells; j++)
      sl[j] = j < nc ? geo_ld(&G.slab[S.cstart[lane][j]]) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int j = 0; j < kCoopCells; j++) pass[j] = slab_may_cross(sl[j], o, L.d, L.dist);
  }
  uint32_t tot = 0;
#pragma unroll
  for (int j = 0; j < kCoopCells; j++) {
    const uint32_t cnt = (j < nc && se[j].x != kNone && pass[j]) ? se[j].y - se[j].x : 0u;
    S.cstart[lane][j] = se[j].x;
    S.cpre[lane][j] = tot;
    S.best[lane][j] = ~0ull;
    tot += cnt;
  }
  S.cpre[lane][kCoopCells] = tot;
  // the warp's exclusive prefix over lanes
  uint32_t incl = tot;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t v = __shfl_up_sync(kFull, incl, d);
    if ((int)lane >= d) incl += v;
  }
  S.lpre[lane] = incl - tot;
  if (lane == 31) S.lpre[32] = incl;
  __syncwarp();
  const uint32_t total = S.lpre[32];
  // the planes of all listed entries, kCoopUnroll per lane per round
  uint32_t nq = 0;
  for (uint32_t base = 0; base < total; base += 32u * kCoopUnroll) {
    float4 P[kCoopUnroll];
    uint32_t ent[kCoopUnroll], own[kCoopUnroll];
#pragma unroll
    for (int u = 0; u < kCoopUnroll; u++) {
      const uint32_t k = base + 32u * u + lane;
      ent[u] = kNone;
      own[u] = 0;
      P[u] = make_float4(0.f, 0.f, 0.f, 1.f);
      if (k < total) {
        // the lane that owns item k: the last with lpre <= k
        uint32_t lo = 0, hi = 32;
        while (hi - lo > 1) {
          const uint32_t mid = (lo + hi) >> 1;
          if (S.lpre[mid] <= k) lo = mid; else hi = mid;
        }
        const uint32_t r = k - S.lpre[lo];
        uint32_t j = 0;
        while (j + 1 < kCoopCells && S.cpre[lo][j + 1] <= r) j++;
        ent[u] = S.cstart[lo][j] + (r - S.cpre[lo][j]);
        own[u] = lo | (j << 8);
        P[u] = geo_ld(&G.plane[ent[u]]);
      }
    }
#pragma unroll
    for (int u = 0; u < kCoopUnroll; u++) {
      bool c = false;
      if (ent[u] != kNone) {
        const uint32_t Lw = own[u] & 0xffu;
        c = plane_may_cross(P[u], make_float3(S.ox[Lw], S.oy[Lw], S.oz[Lw]),
                            make_float3(S.dx[Lw], S.dy[Lw], S.dz[Lw]), S.dist[Lw]);
      }
      const unsigned m = __ballot_sync(kFull, c);
      if (c) S.cand[nq + __popc(m & ((1u << lane) - 1u))] = make_uint2(ent[u], own[u]);
      nq += __popc(m);
      __syncwarp();
      if (nq >= 32) {
        coop_crossings(G, S, 32);
        nq -= 32;
        if (lane < nq) S.cand[lane] = S.cand[32 + lane];
        __syncwarp();
      }
    }
  }
  if (nq) coop_crossings(G, S, nq);
  // nearest_wall_hit's rule over the lane's own cells, in walk order
  float best = 3.0e38f;
  uint32_t best_i = kNone;
  for (int j = 0; j < nc; j++) {
    const unsigned long long b = S.best[lane][j];
    if (b != ~0ull) {
      const float t = __uint_as_float((uint32_t)(b >> 32));
      if (t < best) {
        best = t;
        best_i = (uint32_t)b;
      }
    }
    if (best <= S.texit[lane][j]) break;
  }
  __syncwarp();
  if (alone) return -1;
  if (!walk || best_i == kNone) return kLegFree;
  L.t = best;
  L.e = best_i;
  L.P = geo_ld(&G.plane[best_i]);
  if (fmaf(L.d.z, L.P.z, fmaf(L.d.x, L.P.x, __fmul_rn(L.d.y, L.P.y))) > 0.f) return kLegInside;
  return kLegWall;
}

// COOP: the form with the joint first leg, for nearest wall crossings (the
// launch has kMeshWarps warps per CTA); the other flies each listed flight
// alone (first-hit mode).
template <bool COOP>
__device__ __forceinline__ void mesh_body(const StepParams& p, const uint32_t vb, const uint32_t vg) {
  const uint32_t step = p.step_override ? p.step_override : p.meta->step;
  const uint32_t n = p.meta->n_defer;
  uint32_t removed = 0;
  __shared__ MeshCoop s_coop[COOP ? kMeshWarps : 1];
  MeshCoop& S = s_coop[COOP ? (threadIdx.x >> 5) % kMeshWarps : 0];
  const bool coop = COOP && p.has_geom && p.geom.nearest;
  for (uint32_t base = vb * blockDim.x; base < n; base += vg * blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    const bool go = i < n;
    uint32_t g = 0;
    float3 pos = make_float3(0.f, 0.f, 0.f), vel = pos;
    bool live = true;
    if (go) {
      g = p.defer_list[i];
      pos = make_float3(p.mid.x[g], p.mid.y[g], p.mid.z[g]);
      vel = make_float3(p.mid.u[g], p.mid.v[g], p.mid.w[g]);
    }
    if (coop) {
      // move_particle_body's nearest branch, the first leg walked jointly
      const GeomView& G = p.geom;
      float3 old_pos = pos;
      pos.x = fmaf(vel.x, p.dt, old_pos.x);
      pos.y = fmaf(vel.y, p.dt, old_pos.y);
      pos.z = fmaf(vel.z, p.dt, old_pos.z);
      NearestLeg L0;
      const bool leg = go && leg_path(old_pos, pos, L0);
      if (!leg) L0.d = make_float3(0.f, 0.f, 0.f), L0.dist = 0.f;
      const int r0 = coop_first_leg(G, S, leg, old_pos, L0);
      if (go) {
        PhiloxStream rng;
        rng.init(p.seed, g, step, kPurposeWall);
        // listed because the path may reach the body: the first clearance
        // test is already done
        // (later legs, and first legs too long for the joint walk, walk
        // alone through a call)
        live = nearest_legs<false>(G, old_pos, pos, vel, rng, true, r0, L0) && apply_bc(p, pos, vel, rng);
      }
    } else if (!COOP && go) {
      // listed because the path may reach the body: the first clearance test
      // is already done
      live = move_particle_body(p, pos, vel, g, step, true);
    }
    finish_flight(p, go, live, g, pos, vel, removed);
  }
  __shared__ uint32_t s_rm[8];
  if (p.meta) block_add(&p.meta->removed, removed, s_rm);
}

template <int MINB, bool COOP>
__global__ void __launch_bounds__(32 * kMeshWarps, MINB) k_mesh_w(const __grid_constant__ StepParams p) {
  chained_entry();
  mesh_body<COOP>(p, blockIdx.x, gridDim.x);
}
template <int MINB, bool COOP>
__global__ void __launch_bounds__(32 * kMeshWarps, MINB) k_mesh_wb(const __grid_constant__ BatchOf<StepParams> bv) {
  chained_entry();
  uint32_t vb, vg;
  const StepParams& p = bv.locate(vb, vg);
  mesh_body<COOP>(p, vb, vg);
}

// FP64 sampling after the flights, one cell per thread (the reference's
// SampleCellStatisticsDev order: each cell's particles in sorted order, with
// their velocities after the move); returns at once on other steps.
// A kernel of the step must not complete before the one it follows: a
// chained kernel after it (the next step's scan, launched directly) waits
// only for it.  In a captured step graph this kernel is the graph's last
// (graph_tail; only the inflow kernels, which run beside the mesh kernel by
// design, may follow it), and the next replay waits for the whole graph: on
// a step without sampling it then ends without waiting for the mesh kernel.
// The step counter it reads first was bumped by the step's scan kernel,
// which completed before the kernel this one follows began.
__device__ __forceinline__ void sample_body(const StepParams& p, const uint32_t vb, const uint32_t vg) {
  if (p.graph_tail) {
    const uint32_t step = p.step_override ? p.step_override : __ldcg(&p.meta->step);
    const bool idle = !(p.flags & kDoSample) ||
                      (!(p.flags & kSampleForce) && !(p.sample_every > 0 && step % (uint32_t)p.sample_every == 0));
    if (idle) return;
  }
  chained_entry();
  const uint32_t step = p.step_override ? p.step_override : p.meta->step;
  const bool do_sample =
      (p.flags & kDoSample) &&
      ((p.flags & kSampleForce) || (p.sample_every > 0 && step % (uint32_t)p.sample_every == 0));
  if (!do_sample) return;
  for (uint32_t c = vb * blockDim.x + threadIdx.x; c < p.cells; c += vg * blockDim.x) {
    const uint32_t s = __ldg(&p.start[c]), e = __ldg(&p.start[c + 1]);
    GlobalVel a{p.out.u, p.out.v, p.out.w, s};
    sample_cell(p.acc, p.cells, c, (int)(e - s), a);
  }
  if (p.meta && vb == 0 && threadIdx.x == 0) atomicAdd(&p.meta->samples, 1u);
}

__global__ void __launch_bounds__(256) k_sample_w(const __grid_constant__ StepParams p) {
  sample_body(p, blockIdx.x, gridDim.x);
}
__global__ void __launch_bounds__(256) k_sample_wb(const __grid_constant__ BatchOf<StepParams> bv) {
  uint32_t vb, vg;
  const StepParams& p = bv.locate(vb, vg);
  sample_body(p, vb, vg);
}

// ------------------------------------------------------------- launches ----

struct LaunchShapeW {
  int device = -1;
  uint32_t n_scan_tiles = 0;
  int per_sm = 0;
};

template <int CAPW, int WARPS, int MINB>
cudaError_t launch_order_w(const StepParams& p, cudaStream_t stream) {
  static LaunchShapeW cache[8];
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  LaunchShapeW& ls = cache[dev & 7];
  const size_t smem = collide_smem_bytes<CAPW, WARPS>();
  if (ls.device != dev) {
    e = cudaFuncSetAttribute(k_order_w<CAPW, WARPS, MINB>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_order_w<CAPW, WARPS, MINB>,
                                                      WARPS * 32, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    ls.device = dev;
    ls.per_sm = per_sm;
  }
  uint32_t grid = (uint32_t)(num_sms() * ls.per_sm);
  const uint32_t need = (p.n_tiles + WARPS - 1) / WARPS;
  if (grid > need) grid = need;
  if (grid == 0) return cudaSuccess;
  return launch_chained(k_order_w<CAPW, WARPS, MINB>, grid, WARPS * 32, smem, stream, true, p);
}

constexpr int kFlightWarps = 8;

template <int MINB>
cudaError_t launch_flight_w(const StepParams& p, cudaStream_t stream) {
  static LaunchShapeW cache[8];
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  LaunchShapeW& ls = cache[dev & 7];
  if (ls.device != dev) {
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_flight_w<kFlightWarps, MINB>,
                                                      kFlightWarps * 32, kMaxScanTiles * 4);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    ls.device = dev;
    ls.per_sm = per_sm;
  }
  // a full wave of warps: the particle count is known only on the device
  return launch_chained(k_flight_w<kFlightWarps, MINB>, (uint32_t)(num_sms() * ls.per_sm), kFlightWarps * 32,
                        p.n_scan_tiles * 4u, stream, true, p);
}

template <int MINB>
cudaError_t launch_flight_pw(const StepParams& p, cudaStream_t stream) {
  static LaunchShapeW cache[8];
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  LaunchShapeW& ls = cache[dev & 7];
  if (ls.device != dev) {
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_flight_pw<kFlightWarps, MINB>,
                                                      kFlightWarps * 32, kMaxScanTiles * 4);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    ls.device = dev;
    ls.per_sm = per_sm;
  }
  return launch_chained(k_flight_pw<kFlightWarps, MINB>, (uint32_t)(num_sms() * ls.per_sm), kFlightWarps * 32,
                        p.n_scan_tiles * 4u, stream, true, p);
}

constexpr int kNtcWarps = 8;

cudaError_t launch_ntc_w(const StepParams& p, cudaStream_t stream) {
  static LaunchShapeW cache[8];
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  LaunchShapeW& ls = cache[dev & 7];
  if (ls.device != dev) {
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ntc_w<kNtcWarps>, kNtcWarps * 32, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    ls.device = dev;
    ls.per_sm = per_sm;
  }
  return launch_chained(k_ntc_w<kNtcWarps>, (uint32_t)(num_sms() * ls.per_sm), kNtcWarps * 32, 0, stream, true, p);
}

template <int MINB, bool COOP>
cudaError_t launch_mesh_w(const StepParams& p, cudaStream_t stream) {
  static LaunchShapeW cache[8];
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  LaunchShapeW& ls = cache[dev & 7];
  if (ls.device != dev) {
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mesh_w<MINB, COOP>, 32 * kMeshWarps, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    ls.device = dev;
    ls.per_sm = per_sm;
  }
  return launch_chained(k_mesh_w<MINB, COOP>, (uint32_t)(num_sms() * ls.per_sm), 32 * kMeshWarps, 0, stream, true, p);
}

cudaError_t launch_sample_w(const StepParams& p, cudaStream_t stream) {
  return launch_chained(k_sample_w, grid_for(p.cells, 256, 8), 256, 0, stream, true, p);
}

}  // namespace

// Split variants (cell_kernel_variants() numbers them after the fused
// CTA-wide ones): (particles per warp chunk, warps per CTA, CTAs per SM the
// registers are capped for) of the order kernel and the flight kernel's form
// (8 warps per CTA): 0 (256, 4, 4; one particle per lane), 1 (128, 4, 5;
// one), 2 (128, 8, 3; pairs), 3 (128, 4, 6; pairs).
int cell_kernel_w_variants() { return 4; }

int cell_kernel_w_capacity(int v) {
  static const int caps[4] = {256, 128, 128, 128};
  return caps[v < 0 || v > 3 ? 1 : v];
}

uint32_t cell_kernel_w_tile() { return kWarpTile; }

cudaError_t launch_split_stage(const StepParams& p, int v, int stage, cudaStream_t stream) {
  switch (stage) {
    case 0:
      switch (v) {
        case 0: return launch_order_w<256, 4, 4>(p, stream);
        case 2: return launch_order_w<128, 8, 3>(p, stream);
        case 3: return launch_order_w<128, 4, 6>(p, stream);
        default: return launch_order_w<128, 4, 5>(p, stream);
      }
    case 1:
      if (p.flags & kDoCollide) return launch_ntc_w(p, stream);
      return cudaSuccess;
    case 2:
      // 0, 1: single particles per lane; 2, 3: pairs (different register caps)
      switch (v) {
        case 2: return launch_flight_pw<3>(p, stream);
        case 3: return launch_flight_pw<4>(p, stream);
        default: return launch_flight_w<4>(p, stream);
      }
    case 3:
      // flights that may reach the body (listed only with a body and the move)
      if (p.has_geom && (p.flags & kDoMove))
        return p.geom.nearest ? launch_mesh_w<2, true>(p, stream) : launch_mesh_w<2, false>(p, stream);
      return cudaSuccess;
    default:
      if (p.flags & kDoSample) return launch_sample_w(p, stream);
      return cudaSuccess;
  }
}

// Batched forms of the split kernels for ensembles: the order kernel in the
// (128 particles, 4 warps, 5 CTAs per SM) shape, single-particle flights.
cudaError_t cell_batch_waves(uint32_t wave[5], size_t flight_smem) {
  const size_t osmem = collide_smem_bytes<128, 4>();
  cudaError_t e = cudaFuncSetAttribute(k_order_wb<128, 4, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)osmem);
  if (e != cudaSuccess) return e;
  int per[5] = {0, 0, 0, 0, 0};
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per[0], k_order_wb<128, 4, 5>, 128, osmem);
  if (!e) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per[1], k_ntc_wb<kNtcWarps>, kNtcWarps * 32, 0);
  if (!e)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per[2], k_flight_wb<kFlightWarps, 4>, kFlightWarps * 32,
                                                      flight_smem);
  if (!e) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per[3], k_mesh_wb<2, true>, 32 * kMeshWarps, 0);
  per[4] = 8;
  if (e != cudaSuccess) return e;
  for (int k = 0; k < 5; k++) {
    if (per[k] < 1) return cudaErrorInvalidConfiguration;
    wave[k] = (uint32_t)(num_sms() * per[k]);
  }
  return cudaSuccess;
}

cudaError_t launch_cell_stage_b(int stage, const BatchOf<StepParams>& bv, uint32_t blocks, size_t flight_smem,
                                bool coop_mesh, cudaStream_t stream) {
  if (blocks == 0) return cudaSuccess;
  switch (stage) {
    case 0: return launch_chained(k_order_wb<128, 4, 5>, blocks, 128, collide_smem_bytes<128, 4>(), stream, false, bv);
    case 1: return launch_chained(k_ntc_wb<kNtcWarps>, blocks, kNtcWarps * 32, 0, stream, false, bv);
    case 2: return launch_chained(k_flight_wb<kFlightWarps, 4>, blocks, kFlightWarps * 32, flight_smem, stream, false, bv);
    case 3:
      return coop_mesh ? launch_chained(k_mesh_wb<2, true>, blocks, 32 * kMeshWarps, 0, stream, false, bv)
                       : launch_chained(k_mesh_wb<2, false>, blocks, 32 * kMeshWarps, 0, stream, false, bv);
    default: return launch_chained(k_sample_wb, blocks, 256, 0, stream, false, bv);
  }
}

cudaError_t launch_cell_w(const StepParams& p, int v, cudaStream_t stream) {
  for (int stage = 0; stage < 5; stage++) {
    const cudaError_t e = launch_split_stage(p, v, stage, stream);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace dsmcb
