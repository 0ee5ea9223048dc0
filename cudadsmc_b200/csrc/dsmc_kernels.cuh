// Kernel parameter blocks and launch helpers for the DSMC timestep.
//
// One timestep (dsmc_step) is three launches on the handle's stream:
//   scan     per-cell particle counts -> exclusive cell starts (counts reset)
//   scatter  each particle to start[key] + a per-cell ticket in the sorted
//            array, with its position in the unsorted array (`orig`)
//   cell     per tile of cells, staged in shared memory by bulk copies: the
//            stable (key, orig) order restored inside each cell, NTC
//            collisions, free flight with mesh and boundary collisions,
//            optional FP64 sampling, and the next step's cell key (+ count).
// The cell kernel writes the state back in sorted order, which is the array the
// next step's scatter reads: the reference's sort + reorder + collide + move
// sequence (include/gpu_dsmc.inl:220-274) with two passes over particle memory.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "dsmc_device.cuh"

namespace dsmcb {

// Launches `kernel` with programmatic stream serialization: its CTAs may be
// dispatched while the previous kernel in the stream drains; the kernel must
// call chained_entry() before touching memory.  Kernel nodes captured into
// a graph keep the programmatic edge.  The batched (ensemble) stages launch
// with chained = false: there the early CTAs of the next stage cost more than
// they save (1.78 against 2.10 ms per step of the 64-member ensemble), while
// a single instance gains about 1 %.
template <typename... KArgs, typename... Args>
inline cudaError_t launch_chained(void (*kernel)(KArgs...), uint32_t grid, uint32_t block, size_t smem,
                                  cudaStream_t stream, bool chained, Args... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = chained ? 1 : 0;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}

constexpr int kMaxCellsPerTile = 256;
constexpr int kScanTile = 2048;       // cells per scan block (256 threads x 8)
constexpr int kScanShift = 11;
constexpr int kMaxScanTiles = 2048;   // => at most 4M cells

// Device-side counters shared by the step's kernels.
struct Meta {
  uint32_t n_alive;   // particles placed in cells by the last scan
  uint32_t n_pending; // particles appended after them since (inflow)
  uint32_t n_scatter; // particles the current step's scatter reads
  uint32_t step;      // timestep counter (reference m_state->stepCount)
  uint32_t error;     // error bits (kErr*)
  unsigned long long selections;
  unsigned long long collisions;
  double sum_g;
  uint32_t giant_cells;  // cells handled by the out-of-shared-memory path
  uint32_t samples;      // sampling passes
  uint32_t injected;     // particles injected by the inflow faces (total)
  uint32_t removed;      // particles removed through outflow faces (total)
  uint32_t tile_next;    // the cell kernel's dynamic tile counter (reset by the scan)
  uint32_t tile_next2;   // the NTC kernel's claims of light cells (reset by the scan)
  uint32_t n_defer;      // flights listed for the mesh kernel this step (reset by the scan)
  uint32_t n_light;      // cells listed for the NTC kernel, one lane each (reset by the scan)
  uint32_t n_heavy;      // cells listed for the NTC kernel, one warp each (reset by the scan)
  unsigned long long particle_steps;  // sum over steps of the particles placed by the scan
};

enum : uint32_t {
  kErrCapacity = 1u,   // injection would exceed the buffer capacity
  kErrKeyRange = 2u,   // a key >= cells reached the scatter
  kErrTimeout = 4u,    // a bounded wait on a tile copy ran out
};

struct SoA {
  float* x; float* y; float* z; float* u; float* v; float* w;
};

enum : int {
  kDoFixup = 1,    // restore (key, orig) order inside each cell
  kDoCollide = 2,
  kDoMove = 4,
  kDoKeys = 8,     // next-step key + count + tile histogram
  kDoSample = 16,  // FP64 sampling after the move (every sample_every steps)
  kSampleForce = 32,  // sample regardless of the step counter
  kVelOnly = 64,      // stage only velocities (collide stage)
  kPadded = 128,      // buffers carry 16 bytes of slack: whole aligned copies
};

// Inflow description for a face that injects (extension).
struct Inflow {
  int face;            // 0..5 (-x,+x,-y,+y,-z,+z); -1: none
  float number_flux;   // simulator particles per unit area per second
  float3 stream;       // free-stream velocity
  float vstd;          // sqrt(k T / m)
  float area;
};

struct StepParams {
  GridGeom grid;
  uint32_t cells;
  float cell_volume;
  float cross_section;
  float fnum;
  float avg_conc;
  float dt;
  float ntc_coef;  // 0.5 fnum dt / V_c (FP32 selection count of the Philox mode)
  int periodic;
  int hard_sphere;
  float vhs_exp;   // 2*omega - 1
  float vhs_gref;
  // Philox mode: sigma(g) g = vhs_k 2^(vhs_c1 log2 g), vhs_c1 = 1 - vhs_exp,
  // vhs_k = cross_section vhs_gref^vhs_exp (both rounded from double)
  float vhs_k, vhs_c1;
  int ntc_local;
  int rng_kind;    // 0 HybridTaus per cell (reference), 1 Philox
  uint2 seed;
  int face_mode;
  int face_kind[6];
  float face_vstd[6];
  int has_geom;
  GeomView geom;

  // buffers
  SoA in;             // state the cell kernel reads (sorted by scatter)
  const uint32_t* in_orig;
  SoA out;            // state the cell kernel writes (sorted order)
  SoA mid;            // split variants: the sorted post-collision state between
                      // the collide kernel (which gathers it from `in` through
                      // in_orig) and the flight kernel (which writes `out`)
  uint32_t* out_key;  // next-step cell key (kDeadKey: left the domain)
  const uint32_t* start;   // cells+1 exclusive starts
  uint32_t* count;         // per-cell counters for the next step
  uint32_t* tile_sum;      // per scan tile counters for the next step
  uint32_t n_scan_tiles;
  float2* maxrem;
  uint4* seeds;
  float4* stat4;           // optional per-cell (selections, collisions, sum g)
  double* acc;             // 5 x cells FP64 accumulators (SoA), optional
  Meta* meta;
  int flags;
  int sample_every;
  int cells_per_tile;
  uint32_t n_tiles;
  uint32_t step_override;  // 0: use meta->step
  int cell_variant;        // (threads, chunk capacity) of the cell kernel
  uint4* ntc_light;        // split variants: (cell, first sorted slot, count, pairs) of
  uint4* ntc_heavy;        // the cells with NTC pairs this step (cells entries each)
  uint32_t* defer_list;    // split variants: flights that may reach the body
                           // (capacity entries; the orig buffer, dead once the
                           // collide kernel has read it)
  int graph_tail;          // 1: the sampling kernel ends a captured step graph (nothing
                           // after it in the graph reads the step's keys or counts)
};

// A batched launch: one grid for several members (instances of the step),
// member m owning blocks [block0[m], block0[m + 1]) of it; each block runs the
// member's kernel body with its index and count inside that share, as if the
// member's kernel had been launched alone with that grid.
template <class T>
struct BatchOf {
  const T* items;          // per member, in device memory
  const uint32_t* block0;  // members + 1 block offsets
  uint32_t members;
  __device__ __forceinline__ const T& locate(uint32_t& vb, uint32_t& vg) const {
    uint32_t lo = 0, hi = members;  // the last member whose first block is at or before this one
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (block0[mid] <= blockIdx.x) lo = mid;
      else hi = mid;
    }
    vb = blockIdx.x - block0[lo];
    vg = block0[lo + 1] - block0[lo];
    return items[lo];
  }
};

// Per member, the arrays of the scan and the scatter (batched launches).
struct SortArgs {
  uint32_t* count;
  uint32_t* cursor;
  uint32_t* start;
  uint32_t* tile_sum;
  uint32_t* orig;
  const uint32_t* keys;
  Meta* meta;
  uint32_t cells, n_scan_tiles, capacity;
};

// Launchers (all asynchronous on `stream`).
cudaError_t launch_index(const GridGeom& g, uint32_t cells, const float* x, const float* y,
                         const float* z, uint32_t n, uint32_t* keys, uint32_t* count,
                         uint32_t* tile_sum, uint32_t n_scan_tiles, int face_mode,
                         cudaStream_t stream);
cudaError_t launch_scan(uint32_t* count, uint32_t* cursor, uint32_t* start, uint32_t cells,
                        const uint32_t* tile_sum, uint32_t n_scan_tiles, Meta* meta, int bump_step,
                        cudaStream_t stream);
// with_state = false: only orig (the split cell kernels gather the state).
cudaError_t launch_scatter(bool with_state, const SoA& src, SoA dst, const uint32_t* keys,
                           const uint32_t* start,
                           uint32_t* cursor, uint32_t* orig, uint32_t cells, uint32_t* tile_sum,
                           uint32_t n_scan_tiles, Meta* meta, uint32_t capacity,
                           cudaStream_t stream);
// The timestep's fused cell kernel (also the collide stage with kVelOnly).
cudaError_t launch_cell(const StepParams& p, cudaStream_t stream);
// Variants of the cell kernel.  CTA-wide: 0 (512 threads, 2048 particles per
// chunk, 1 CTA/SM), 1 (256, 1024, 2), 2 (128, 512, 4), 3 (64, 256, up to 8).
// Warp-autonomous (particles per warp chunk, warps per CTA, CTAs per SM):
// 4 (256, 4, 4), 5 (128, 4, 5), 6 (128, 8, 3), 7 (128, 4, 6).
int cell_kernel_variants();
int cell_kernel_chunk_capacity(int variant);
// Variants at or above 4 use the warp-autonomous kernel, whose tiles are
// cell_kernel_w_tile() cells (one per lane).
bool cell_kernel_is_warp(int variant);
int cell_kernel_w_variants();
int cell_kernel_w_capacity(int v);
uint32_t cell_kernel_w_tile();
cudaError_t launch_cell_w(const StepParams& p, int v, cudaStream_t stream);
// One kernel of the split variants: 0 order (gather, stable order, pair
// counts), 1 NTC selections, 2 flight, 3 mesh flights, 4 sampling
// (launch_cell_w runs the five in order).
cudaError_t launch_split_stage(const StepParams& p, int v, int stage, cudaStream_t stream);
// Free flight + boundaries in place on p.out for n particles (move stage);
// particles that leave through an outflow face get x = NaN.
cudaError_t launch_move(const StepParams& p, uint32_t n, uint32_t step, cudaStream_t stream);
// keys[i] = cell id of particle i, idx[i] = i (cell-index stage).
cudaError_t launch_cell_ids(const GridGeom& g, const float* x, const float* y, const float* z,
                            uint32_t n, uint32_t* keys, uint32_t* idx, cudaStream_t stream);

// Sort stage pieces (dsmc_stage_sort).
cudaError_t launch_count_keys(const uint32_t* keys, uint32_t n, uint32_t nkeys, uint32_t* ticket,
                              uint32_t* count, uint32_t* tile_sum, uint32_t n_scan_tiles,
                              cudaStream_t stream);
cudaError_t launch_scatter_kv(const uint32_t* keys, const uint32_t* vals, const uint32_t* ticket,
                              const uint32_t* start, uint32_t n, uint32_t nkeys, uint32_t* tmp_val,
                              uint32_t* tmp_pos, cudaStream_t stream);
cudaError_t launch_segment_fixup(const uint32_t* start, uint32_t nkeys, const uint32_t* tmp_val,
                                 const uint32_t* tmp_pos, uint32_t* keys_out, uint32_t* vals_out,
                                 cudaStream_t stream);
cudaError_t launch_bounds_reorder(const uint32_t* keys, const uint32_t* idx, uint32_t n,
                                  uint32_t ncells, uint32_t* cse, const float* const src[6],
                                  float* const dst[6], cudaStream_t stream);
// acc[field * fstride + cell * cstride] += sums (field 0..4: n, u, v, w, |v|^2)
// The -mt collisions (dsmc_mt.cu): twister set-up (InitTwisterFast for
// twisters [0, n)), InitMaximums, and the NTC selections of the listed cells
// drawn from each cell's twister in place of k_ntc_w's.
cudaError_t launch_mt_init(const uint4* cfg, uint32_t* state, uint32_t n, cudaStream_t stream);
cudaError_t launch_mt_maximums(const uint4* cfg, uint32_t* state, float2* maxrem, float max_rel_vel,
                               uint32_t n, cudaStream_t stream);
cudaError_t launch_ntc_mt(const StepParams& p, uint32_t* mt_state, const uint4* mt_cfg,
                          cudaStream_t stream);

// Per-cell fields (or, with fields == 0, the sums) cell-major from the FP64
// sampling sums.
cudaError_t launch_cell_fields(const double* acc, uint32_t cells, double fnum, double cell_volume,
                               uint32_t ns, double mass, int fields, double* out, cudaStream_t stream);
cudaError_t launch_sample_cells(const float* u, const float* v, const float* w,
                                const uint32_t* start, uint32_t cells, double* acc,
                                size_t fstride, size_t cstride, cudaStream_t stream);

// Initial fill (dsmc_init_state).
struct InitParams {
  GridGeom grid;
  uint32_t cells;
  uint32_t ppc;
  int kind;          // 0 reference sampler, 1 Maxwellian, 2 bimodal
  float vstd;        // sqrt(kT/m)
  float vstd2;       // bimodal second temperature
  float vmp;         // sqrt(2kT/m), reference sampler
  float3 stream;
  uint2 seed;
  const uint32_t* cell_slot;  // per cell: first particle index, kNone = skipped cell
  const uint32_t* cell_count; // per cell: particles to fill (<= ppc)
  const float4* cell_state;   // optional per cell (u, v, w, sqrt(kT/m)) of the Maxwellian
  const float* cell_mix;      // optional per cell (with cell_state): the fraction of particles
                              // drawn from the free stream (stream, vstd) instead
  int reject_inside;          // redraw positions that fall inside the mesh
  GeomView geom;
  const float4* cell_point;   // optional per cell: a point outside the mesh (w = 1) or none (w = 0)
  SoA out;
};
cudaError_t launch_init_fill(const InitParams& p, cudaStream_t stream);
// Fraction of every cell outside the mesh (64 stratified points per cell)
// and one outside point per cell (w = 1; w = 0 if none was found).
cudaError_t launch_outside_fraction(const GridGeom& grid, const GeomView& geom, uint32_t cells,
                                    float* frac, float4* point, cudaStream_t stream);

// Clearance table of the deferral test on `fine` (the triangle grid refined
// by fac), from the triangle grid's CSR and its cell distances cdist.
cudaError_t launch_fine_clearance(const GeomView& g, const GridGeom& fine, uint32_t fac,
                                  const int* cdist, float cmin, float* out, cudaStream_t stream);

// Per bin entry, (path length, least elevation sine) below and above which
// a path leaving its triangle outward crosses no listed triangle
// (k_entry_reach); (0, 2) where none.
cudaError_t launch_entry_reach(const GeomView& g, uint32_t entries, float rmax, float tol, float slack,
                               float2* out, cudaStream_t stream);

// The slab of every cell of the triangle grid (k_cell_slab; GeomView::slab).
cudaError_t launch_cell_slab(const GeomView& g, uint32_t cells, float4* out, cudaStream_t stream);

// out[i] = clearance table entry at point i (xyz interleaved), -1 outside.
cudaError_t launch_clearance_at(const GeomView& g, const float* xyz, uint32_t n, float* out,
                                cudaStream_t stream);

// Inflow injection: appends particles after the ones in cells and counts them
// for the next scan.
struct InjectParams {
  GridGeom grid;
  uint32_t cells;
  Inflow inflow;
  float dt;
  uint2 seed;
  uint32_t capacity;
  float* remainder;  // device float carrying the fractional particle count
  SoA st;            // the array the next scatter reads
  uint32_t* keys;
  uint32_t* count;
  uint32_t* tile_sum;
  uint32_t n_scan_tiles;
  uint32_t* plan;    // 2 words of device scratch: first slot, count
  Meta* meta;
};
cudaError_t launch_inject(const InjectParams& p, cudaStream_t stream);

int num_sms();
uint32_t grid_for(uint64_t work, int threads, int per_sm);

// Batched launches of the step's kernels over the members of an ensemble
// (BatchOf; every member's blocks run its own parameters).
cudaError_t launch_scan_b(const BatchOf<SortArgs>& bv, uint32_t blocks, cudaStream_t stream);
cudaError_t launch_scatter_b(const BatchOf<SortArgs>& bv, uint32_t blocks, cudaStream_t stream);
// One block of 32 threads per entry for the plan; the fill's blocks shared
// among the entries.
cudaError_t launch_inject_b(const BatchOf<InjectParams>& plan, uint32_t plan_blocks,
                            const BatchOf<InjectParams>& fill, uint32_t fill_blocks, size_t fill_smem,
                            cudaStream_t stream);
// Full-wave block counts of the batched cell stages: order, NTC, flight, mesh,
// sampling.
cudaError_t cell_batch_waves(uint32_t wave[5], size_t flight_smem);
// Stage 0 order, 1 NTC, 2 flight, 3 mesh, 4 sampling.  coop_mesh: every
// member with a body uses nearest wall crossings (the mesh stage walks first
// legs a warp at a time).
cudaError_t launch_cell_stage_b(int stage, const BatchOf<StepParams>& bv, uint32_t blocks, size_t flight_smem,
                                bool coop_mesh, cudaStream_t stream);

}  // namespace dsmcb
