// C ABI of the B200 DSMC timestep (declared in include/dsmc_b200.h).
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "dsmc_b200.h"
#include "dsmc_geomgrid.hpp"
#include "dsmc_host.hpp"
#include "dsmc_kernels.cuh"

using dsmcb::GridGeom;
using dsmcb::Meta;
using dsmcb::SoA;

struct dsmc_handle {
  dsmc_config cfg{};
  int device = 0;
  cudaStream_t stream = nullptr;

  uint32_t ppc = 0, cells = 0, capacity = 0, n_scan_tiles = 0, n_tiles = 0, cells_per_tile = 0;
  int variant = 5;  // cell-kernel variant (dsmc_set_kernel_variant)
  float cell_size[3]{}, cell_volume = 0.f, cross_section = 0.f, max_rel_vel = 0.f;
  float vhs_gref = 0.f;
  GridGeom grid{};

  float* A[6]{};
  float* B[6]{};
  uint32_t* orig = nullptr;
  uint4* ntc_list = nullptr;  // 2 x cells entries: light then dense cells with NTC pairs
  uint32_t* keys = nullptr;    // next-step cell key per particle
  uint32_t* cursor = nullptr;  // per-cell ticket counters of the scatter
  uint32_t* count = nullptr;
  uint32_t* start = nullptr;
  uint32_t* tile_sum = nullptr;
  float2* maxrem = nullptr;
  uint4* seeds = nullptr;
  // -mt mode (dsmc_set_twisters): per cell a Mersenne Twister, 21 state
  // words and one parameter record; the NTC selections draw from it
  uint32_t* mt_state = nullptr;
  uint4* mt_cfg = nullptr;
  bool mt_on = false;
  double* acc = nullptr;
  double* cellbuf = nullptr;  // per-cell fields / sums, cell-major, for readback (on first use)
  Meta* meta = nullptr;
  float* inj_rem = nullptr;
  uint32_t* inj_plan = nullptr;

  bool has_geom = false;
  dsmcb::GeomGrid ggrid;
  uint32_t* gflags = nullptr;
  float* gclear = nullptr;
  float2* greach = nullptr;  // per bin entry (null: the mesh's scale is too large for it)
  float4* gslab = nullptr;   // per cell of the triangle grid
  uint2* gse = nullptr;
  float4* gtri = nullptr;
  float4* gplane = nullptr;
  GridGeom gcgrid{};  // grid of the clearance table gclear

  bool has_state = false;
  uint64_t step = 0;
  double sim_time = 0.0;
  uint64_t gen = 0;  // bumped whenever captured launches of this handle go stale

  std::vector<dsmcb::Inflow> inflows;

  cudaGraphExec_t graph_exec = nullptr;
  cudaGraph_t graph = nullptr;
  float graph_dt = -1.f;

  // the inflow branch: injection runs on `side` beside the NTC, flight,
  // mesh and sampling kernels (forked after the order kernel, joined at the
  // end of the step)
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;

  // per-kernel event timing (dsmc_profile)
  bool profiling = false;
  uint32_t prof_mask = 0xff;  // slots that get events while profiling
  // graph replay with per-kernel events: event-record nodes are captured
  // around the profiled kernels, and before every replay they are pointed at
  // fresh events of ev[]
  bool capturing = false;
  std::vector<cudaEvent_t> cap_ev;        // placeholders used during capture (pairs)
  std::vector<int> cap_slot;              // kernel slot of each captured pair
  std::vector<cudaGraphNode_t> gev_node;  // the graph's event-record nodes, 2 per pair
  uint32_t graph_prof_mask = 0;           // profiled slots the graph was captured with
  std::vector<cudaEvent_t> ev;      // pairs
  std::vector<int> ev_kernel;       // kernel id of each pair
  size_t ev_used = 0;
  // slots: 0 scan, 1 scatter, 2 cell (fused) / order (split), 3 injection,
  // 4 flight, 5 mesh flights, 6 sampling, 7 NTC selections (split)
  double prof_ms[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  uint32_t prof_n[8] = {0, 0, 0, 0, 0, 0, 0, 0};

  std::string err;
};

namespace {

std::string g_create_error;

int fail(dsmc_handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  else g_create_error = msg;
  return code;
}

int cuda_fail(dsmc_handle* h, cudaError_t e, const char* where) {
  return fail(h, e == cudaErrorMemoryAllocation ? DSMC_ERR_OOM : DSMC_ERR_CUDA,
              std::string(where) + ": " + cudaGetErrorString(e));
}

#define CK(h, call, where)                              \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return cuda_fail(h, e_, where); \
  } while (0)

void drop_graph(dsmc_handle* h) {
  h->gen++;
  h->graph_prof_mask = 0;
  h->cap_slot.clear();
  h->gev_node.clear();
  if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
  if (h->graph) cudaGraphDestroy(h->graph);
  h->graph_exec = nullptr;
  h->graph = nullptr;
  h->graph_dt = -1.f;
}

// Cell-kernel variant and the tile size that goes with it: tiles of about one
// shared-memory chunk of particles (32..256 cells); the warp-autonomous
// variants use tiles of 32 cells, one per lane.
void apply_variant(dsmc_handle* h, int v) {
  h->variant = v;
  const uint64_t cap = (uint64_t)dsmcb::cell_kernel_chunk_capacity(v);
  uint32_t ct = dsmcb::kMaxCellsPerTile;
  while (ct > 32 && (uint64_t)ct * std::max<uint32_t>(h->ppc, 1) > cap) ct >>= 1;
  if (dsmcb::cell_kernel_is_warp(v)) ct = dsmcb::cell_kernel_w_tile();
  h->cells_per_tile = ct;
  h->n_tiles = (h->cells + ct - 1) / ct;
  drop_graph(h);
}

uint64_t splitmix64(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

template <class T>
cudaError_t dalloc(T** p, size_t n) {
  return cudaMalloc((void**)p, n * sizeof(T) + 16);
}

void free_all(dsmc_handle* h) {
  if (h->ev_fork) cudaEventDestroy(h->ev_fork);
  if (h->ev_join) cudaEventDestroy(h->ev_join);
  if (h->side) cudaStreamDestroy(h->side);
  h->ev_fork = h->ev_join = nullptr;
  h->side = nullptr;
  for (cudaEvent_t e : h->ev) cudaEventDestroy(e);
  h->ev.clear();
  for (cudaEvent_t e : h->cap_ev) cudaEventDestroy(e);
  h->cap_ev.clear();
  if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
  if (h->graph) cudaGraphDestroy(h->graph);
  h->graph_exec = nullptr;
  h->graph = nullptr;
  for (int i = 0; i < 6; i++) {
    cudaFree(h->A[i]);
    cudaFree(h->B[i]);
    h->A[i] = h->B[i] = nullptr;
  }
  void* ps[] = {h->orig, h->ntc_list, h->keys, h->cursor, h->count, h->start, h->tile_sum, h->maxrem, h->seeds,
                h->acc, h->cellbuf, h->meta, h->inj_rem, h->inj_plan, h->gflags, h->gclear, h->greach, h->gslab,
                h->gse, h->gtri, h->gplane, h->mt_state, h->mt_cfg};
  for (void* p : ps) cudaFree(p);
  h->mt_state = nullptr;
  h->mt_cfg = nullptr;
  h->mt_on = false;
}

SoA soa_of(float* const a[6]) { return SoA{a[0], a[1], a[2], a[3], a[4], a[5]}; }

// VHS reference speed for sigma(g) = sigma_ref (g_ref / g)^(2 omega - 1):
// g_ref = sqrt(2 k T_ref / m_r) * Gamma(5/2 - omega)^(-1/(2 omega - 1)), m_r = m/2.
float vhs_gref_of(const dsmc_config& c) {
  double w = c.gas_omega;
  if (std::fabs(w - 0.5) < 1e-9) return 0.f;
  double mr = 0.5 * c.gas_mass;
  double g0 = std::sqrt(2.0 * 1.380649e-23 * c.gas_tref / mr);
  return (float)(g0 * std::pow(std::tgamma(2.5 - w), -1.0 / (2.0 * w - 1.0)));
}

// The Philox mode's VHS coefficients: sigma(g) g = vhs_k 2^(vhs_c1 log2 g),
// vhs_c1 = 2 - 2 omega, vhs_k = sigma_ref g_ref^(2 omega - 1), evaluated in
// double and rounded once.
void set_vhs_fast(dsmcb::StepParams& p, float cross_section, float omega, float gref) {
  p.vhs_k = 0.f;
  p.vhs_c1 = 0.f;
  if (p.hard_sphere || !(gref > 0.f) || !(cross_section > 0.f)) return;
  const double e = 2.0 * (double)omega - 1.0;
  p.vhs_c1 = (float)(1.0 - e);
  p.vhs_k = (float)((double)cross_section * std::pow((double)gref, e));
}

dsmcb::StepParams base_params(dsmc_handle* h, float dt) {
  dsmcb::StepParams p{};
  p.grid = h->grid;
  p.cells = h->cells;
  p.cell_volume = h->cell_volume;
  p.cross_section = h->cross_section;
  p.fnum = h->cfg.fnum;
  p.avg_conc = (float)h->ppc;
  p.dt = dt;
  p.ntc_coef = (float)(0.5 * (double)h->cfg.fnum * dt / (double)h->cell_volume);
  p.periodic = h->cfg.periodic;
  p.hard_sphere = std::fabs(h->cfg.gas_omega - 0.5f) < 1e-9f;
  p.vhs_exp = 2.f * h->cfg.gas_omega - 1.f;
  p.vhs_gref = h->vhs_gref;
  set_vhs_fast(p, h->cross_section, h->cfg.gas_omega, h->vhs_gref);
  p.ntc_local = h->cfg.ntc_local;
  p.rng_kind = h->cfg.rng;
  p.seed = make_uint2((uint32_t)h->cfg.seed, (uint32_t)(h->cfg.seed >> 32));
  p.face_mode = h->cfg.face_mode;
  for (int i = 0; i < 6; i++) {
    p.face_kind[i] = h->cfg.face_kind[i];
    p.face_vstd[i] = std::sqrt(1.3806e-23f * h->cfg.face_temp[i] / h->cfg.gas_mass);
  }
  p.has_geom = h->has_geom && h->cfg.geometry;
  if (p.has_geom) {
    const auto& g = h->ggrid;
    p.geom.grid.gmin = make_float3(g.bbox[0], g.bbox[1], g.bbox[2]);
    p.geom.grid.gmax = make_float3(g.bbox[3], g.bbox[4], g.bbox[5]);
    p.geom.grid.cell = make_float3(g.cell[0], g.cell[1], g.cell[2]);
    p.geom.grid.dim = make_uint3(g.dim[0], g.dim[1], g.dim[2]);
    p.geom.flags = h->gflags;
    p.geom.start_end = h->gse;
    p.geom.tri = h->gtri;
    p.geom.plane = h->gplane;
    p.geom.clear = h->gclear;
    p.geom.reach = h->greach;
    p.geom.slab = h->gslab;
    p.geom.cgrid = h->gcgrid;
    p.geom.diffuse = h->cfg.wall_diffuse;
    p.geom.nearest = h->cfg.geom_nearest;
    p.geom.wall_vstd = std::sqrt(1.3806e-23f * h->cfg.wall_temp / h->cfg.gas_mass);
  }
  p.start = h->start;
  p.count = h->count;
  p.tile_sum = h->tile_sum;
  p.n_scan_tiles = h->n_scan_tiles;
  p.maxrem = h->maxrem;
  p.seeds = h->seeds;
  p.stat4 = nullptr;
  p.acc = h->acc;
  p.meta = h->meta;
  p.sample_every = h->cfg.sample_every;
  p.cells_per_tile = (int)h->cells_per_tile;
  p.n_tiles = h->n_tiles;
  p.step_override = 0;
  return p;
}

constexpr size_t kProfPairs = 4096;

void prof_flush(dsmc_handle* h) {
  if (!h->ev_used) return;
  cudaEventSynchronize(h->ev[2 * (h->ev_used - 1) + 1]);
  for (size_t i = 0; i < h->ev_used; i++) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, h->ev[2 * i], h->ev[2 * i + 1]) == cudaSuccess) {
      h->prof_ms[h->ev_kernel[i]] += ms;
      h->prof_n[h->ev_kernel[i]] += 1;
    }
  }
  h->ev_used = 0;
}

// Profiled launches a captured step may hold (each kernel slot at most twice).
constexpr size_t kCapPairs = 16;

// Launches `launch` with CUDA events around it when the handle is profiling.
template <class F>
cudaError_t timed(dsmc_handle* h, int kernel, F launch) {
  if (!h->profiling || !((h->prof_mask >> kernel) & 1u)) return launch();
  if (h->capturing) {
    // event-record nodes around the kernel, with placeholder events (created
    // before the capture); a plain record inside a capture makes no node
    const size_t k = h->cap_slot.size();
    if (h->cap_ev.size() < 2 * (k + 1)) return cudaErrorInvalidValue;
    h->cap_slot.push_back(kernel);
    cudaError_t e = cudaEventRecordWithFlags(h->cap_ev[2 * k], h->stream, cudaEventRecordExternal);
    if (!e) e = launch();
    if (!e) e = cudaEventRecordWithFlags(h->cap_ev[2 * k + 1], h->stream, cudaEventRecordExternal);
    return e;
  }
  if (h->ev_used == kProfPairs) prof_flush(h);
  size_t i = h->ev_used++;
  h->ev_kernel[i] = kernel;
  cudaEventRecord(h->ev[2 * i], h->stream);
  cudaError_t e = launch();
  cudaEventRecord(h->ev[2 * i + 1], h->stream);
  return e;
}

// The side stream and events of the inflow branch (created on first use,
// outside any stream capture).
cudaError_t ensure_side(dsmc_handle* h) {
  if (h->side) return cudaSuccess;
  cudaError_t e = cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking);
  if (!e) e = cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming);
  if (!e) e = cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming);
  return e;
}

// Inflow injection of every inflow face on `stream` (timed when on the
// handle's stream).
dsmcb::InjectParams inject_params(dsmc_handle* h, const dsmcb::Inflow& in, float dt, uint2 seed) {
  dsmcb::InjectParams ip{};
  ip.grid = h->grid;
  ip.cells = h->cells;
  ip.inflow = in;
  ip.dt = dt;
  ip.seed = seed;
  ip.capacity = h->capacity;
  ip.remainder = h->inj_rem + in.face;
  ip.st = soa_of(h->A);
  ip.keys = h->keys;
  ip.count = h->count;
  ip.tile_sum = h->tile_sum;
  ip.n_scan_tiles = h->n_scan_tiles;
  ip.plan = h->inj_plan + 2 * in.face;
  ip.meta = h->meta;
  return ip;
}

cudaError_t enqueue_inflow(dsmc_handle* h, float dt, uint2 seed, cudaStream_t stream) {
  for (const auto& in : h->inflows) {
    const dsmcb::InjectParams ip = inject_params(h, in, dt, seed);
    const cudaError_t e = stream == h->stream
                              ? timed(h, 3, [&] { return dsmcb::launch_inject(ip, stream); })
                              : dsmcb::launch_inject(ip, stream);
    if (e) return e;
  }
  return cudaSuccess;
}

// The cell kernels' parameters of one timestep (split: the split kernels,
// which gather the state from A through orig; else the fused kernel, which
// reads it scattered into B).
dsmcb::StepParams step_params(dsmc_handle* h, float dt, bool split) {
  dsmcb::StepParams p = base_params(h, dt);
  p.in = split ? soa_of(h->A) : soa_of(h->B);
  p.mid = soa_of(h->B);
  p.in_orig = h->orig;
  p.out = soa_of(h->A);
  p.out_key = h->keys;
  p.flags = dsmcb::kDoFixup | dsmcb::kDoCollide | dsmcb::kDoMove | dsmcb::kDoKeys | dsmcb::kPadded;
  if (h->cfg.sample_every > 0) p.flags |= dsmcb::kDoSample;
  p.cell_variant = h->variant;
  p.defer_list = h->orig;
  p.ntc_light = h->ntc_list;
  p.ntc_heavy = h->ntc_list + h->cells;
  return p;
}

// One timestep: scan -> scatter -> cell (-> inflow injection).  With the split
// kernels the injection runs on the side stream once the order kernel has
// gathered the old state: it writes only slots past the sorted particles and
// adds to the counts atomically, so it overlaps the NTC, flight, mesh and
// sampling kernels, which touch only the sorted particles.
cudaError_t enqueue_step(dsmc_handle* h, float dt) {
  cudaError_t e;
  e = timed(h, 0, [&] {
    return dsmcb::launch_scan(h->count, h->cursor, h->start, h->cells, h->tile_sum,
                              h->n_scan_tiles, h->meta, 1, h->stream);
  });
  if (e) return e;
  // the split cell kernels gather the state through orig themselves; the
  // fused one reads it scattered into B
  const bool split = dsmcb::cell_kernel_is_warp(h->variant);
  e = timed(h, 1, [&] {
    return dsmcb::launch_scatter(!split, soa_of(h->A), soa_of(h->B), h->keys, h->start, h->cursor,
                                 h->orig, h->cells, h->tile_sum, h->n_scan_tiles, h->meta,
                                 h->capacity, h->stream);
  });
  if (e) return e;
  dsmcb::StepParams p = step_params(h, dt, split);
  // the sampling kernel closes a captured graph (the graph replay after it
  // waits for every node of this one)
  p.graph_tail = h->capturing ? 1 : 0;
  // the inflow branch (not while the injection itself is being timed: its
  // events are on the handle's stream)
  const bool fork = split && !h->inflows.empty() && h->side &&
                    !(h->profiling && ((h->prof_mask >> 3) & 1u));
  if (split) {
    static const int slot[5] = {2, 7, 4, 5, 6};
    for (int stage = 0; stage < 5; stage++) {
      e = timed(h, slot[stage], [&] {
        if (stage == 1 && h->mt_on) return dsmcb::launch_ntc_mt(p, h->mt_state, h->mt_cfg, h->stream);
        return dsmcb::launch_split_stage(p, h->variant - 4, stage, h->stream);
      });
      if (e) return e;
      if (stage == 0 && fork) {
        e = cudaEventRecord(h->ev_fork, h->stream);
        if (!e) e = cudaStreamWaitEvent(h->side, h->ev_fork, 0);
        if (!e) e = enqueue_inflow(h, dt, p.seed, h->side);
        if (!e) e = cudaEventRecord(h->ev_join, h->side);
        if (e) return e;
      }
    }
    if (fork) return cudaStreamWaitEvent(h->stream, h->ev_join, 0);
  } else {
    // the -mt selections exist for the split kernels only (dsmc_set_twisters
    // selects one)
    if (h->mt_on) return cudaErrorInvalidValue;
    e = timed(h, 2, [&] { return dsmcb::launch_cell(p, h->stream); });
    if (e) return e;
  }
  return enqueue_inflow(h, dt, p.seed, h->stream);
}

// Inflow fluxes of the faces marked DSMC_FACE_INFLOW: number flux of a
// drifting Maxwellian through a face, n c_mp / (2 sqrt(pi)) [exp(-s^2) +
// sqrt(pi) s (1 + erf(s))], s = U.n_in / c_mp, in simulator particles.
void setup_inflows(dsmc_handle* h) {
  h->inflows.clear();
  if (!h->cfg.face_mode) return;
  const dsmc_config& c = h->cfg;
  double vstd = std::sqrt(1.3806e-23 * c.temp / c.gas_mass);
  double cmp = std::sqrt(2.0) * vstd;
  for (int f = 0; f < 6; f++) {
    if (c.face_kind[f] != DSMC_FACE_INFLOW) continue;
    int ax = f >> 1;
    double sign = (f & 1) ? -1.0 : 1.0;
    double un = sign * c.stream_vel[ax];
    double s = un / cmp;
    double flux = c.density * cmp / (2.0 * std::sqrt(M_PI)) *
                  (std::exp(-s * s) + std::sqrt(M_PI) * s * (1.0 + std::erf(s)));
    int a1 = (ax + 1) % 3, a2 = (ax + 2) % 3;
    double area = (double)(c.grid_max[a1] - c.grid_min[a1]) * (c.grid_max[a2] - c.grid_min[a2]);
    dsmcb::Inflow in{};
    in.face = f;
    in.number_flux = (float)(flux / c.fnum);
    in.stream = make_float3(c.stream_vel[0], c.stream_vel[1], c.stream_vel[2]);
    in.vstd = (float)vstd;
    in.area = (float)area;
    h->inflows.push_back(in);
  }
}

int check_device_flags(dsmc_handle* h) {
  uint32_t err = 0;
  CK(h, cudaMemcpy(&err, &h->meta->error, 4, cudaMemcpyDeviceToHost), "read error flags");
  if (err) {
    std::string m = "device error flags:";
    if (err & dsmcb::kErrCapacity) m += " particle capacity exceeded (raise capacity_factor);";
    if (err & dsmcb::kErrKeyRange) m += " cell key out of range;";
    if (err & dsmcb::kErrTimeout) m += " a bulk copy did not complete within a second;";
    return fail(h, DSMC_ERR_DEVICE, m);
  }
  return DSMC_OK;
}

int reindex(dsmc_handle* h, uint32_t n) {
  CK(h, cudaMemsetAsync(h->count, 0, (h->cells + 1) * sizeof(uint32_t), h->stream), "memset");
  CK(h, cudaMemsetAsync(h->tile_sum, 0, h->n_scan_tiles * sizeof(uint32_t), h->stream), "memset");
  CK(h, dsmcb::launch_index(h->grid, h->cells, h->A[0], h->A[1], h->A[2], n, h->keys, h->count,
                            h->tile_sum, h->n_scan_tiles, h->cfg.face_mode, h->stream),
     "index kernel");
  uint32_t m2[2] = {n, 0u};
  CK(h, cudaMemcpyAsync(h->meta, m2, sizeof(m2), cudaMemcpyHostToDevice, h->stream), "meta");
  CK(h, cudaStreamSynchronize(h->stream), "index sync");
  h->has_state = true;
  return DSMC_OK;
}

int read_meta(dsmc_handle* h, Meta& m) {
  CK(h, cudaStreamSynchronize(h->stream), "sync");
  CK(h, cudaMemcpy(&m, h->meta, sizeof(Meta), cudaMemcpyDeviceToHost), "read meta");
  return DSMC_OK;
}

}  // namespace

extern "C" {

const char* dsmc_status_string(int s) {
  switch (s) {
    case DSMC_OK: return "ok";
    case DSMC_ERR_ARG: return "invalid argument";
    case DSMC_ERR_CONFIG: return "configuration error";
    case DSMC_ERR_CUDA: return "CUDA error";
    case DSMC_ERR_OOM: return "out of device memory";
    case DSMC_ERR_STATE: return "call out of order";
    case DSMC_ERR_CAPACITY: return "particle capacity exceeded";
    case DSMC_ERR_IO: return "I/O error";
    case DSMC_ERR_DEVICE: return "device error flag";
  }
  return "unknown status";
}

const char* dsmc_last_error(const dsmc_handle* h) {
  if (!h) return g_create_error.empty() ? dsmcb::g_config_error.c_str() : g_create_error.c_str();
  return h->err.c_str();
}

int dsmc_config_default(dsmc_config* cfg) {
  if (!cfg) return DSMC_ERR_ARG;
  return dsmcb::config_default(cfg);
}

int dsmc_config_read_xml(const char* path, dsmc_config* cfg) {
  if (!path || !cfg) return DSMC_ERR_ARG;
  g_create_error.clear();
  return dsmcb::config_read_xml(path, cfg);
}

int dsmc_config_from_args(int argc, const char* const* argv, dsmc_config* cfg, float* run_for) {
  if (!cfg || (argc > 0 && !argv)) return DSMC_ERR_ARG;
  g_create_error.clear();
  return dsmcb::config_from_args(argc, argv, cfg, run_for);
}

int dsmc_create(const dsmc_config* cfg, dsmc_handle** out) {
  if (!cfg || !out) return fail(nullptr, DSMC_ERR_ARG, "null argument");
  *out = nullptr;
  const dsmc_config& c = *cfg;
  for (int k = 0; k < 3; k++) {
    if (c.grid_dim[k] <= 0 || !(c.grid_max[k] > c.grid_min[k]))
      return fail(nullptr, DSMC_ERR_CONFIG, "grid dims must be > 0 and max > min");
  }
  if (!(c.fnum > 0) || !(c.density > 0) || !(c.gas_mass > 0) || !(c.gas_diam > 0))
    return fail(nullptr, DSMC_ERR_CONFIG, "density, fnum, gas mass and diameter must be > 0");
  if (c.gas_omega < 0.5f || c.gas_omega > 1.0f)
    return fail(nullptr, DSMC_ERR_CONFIG, "VHS omega must lie in [0.5, 1]");
  if (c.rng != DSMC_RNG_TAUS && c.rng != DSMC_RNG_PHILOX)
    return fail(nullptr, DSMC_ERR_CONFIG, "unknown rng");
  uint64_t cells64 = (uint64_t)c.grid_dim[0] * c.grid_dim[1] * c.grid_dim[2];
  if (cells64 > (uint64_t)dsmcb::kMaxScanTiles * dsmcb::kScanTile)
    return fail(nullptr, DSMC_ERR_CONFIG, "too many cells (max 4194304)");

  dsmc_handle* h = new dsmc_handle();
  h->cfg = c;
  cudaGetDevice(&h->device);
  h->cells = (uint32_t)cells64;
  // settings_t / main (src/sim_settings.cpp:100-103, kernels/dsmc.cu:324-330)
  for (int k = 0; k < 3; k++)
    h->cell_size[k] = (c.grid_max[k] - c.grid_min[k]) / (float)(uint32_t)c.grid_dim[k];
  h->cell_volume = h->cell_size[0] * h->cell_size[1] * h->cell_size[2];
  h->ppc = c.part_per_cell ? c.part_per_cell : (uint32_t)(c.density * h->cell_volume / c.fnum);
  // InitSimulationProperties (kernels/dsmc_kernel.cu:323-331)
  const float pi_f = 3.14159265358979f;
  h->cross_section = (float)(double)(pi_f * c.gas_diam * c.gas_diam);
  h->max_rel_vel = (float)(double)(c.gas_diam * c.gas_diam * pi_f * sqrtf((float)(c.temp / 300.0)) * 300);
  h->vhs_gref = vhs_gref_of(c);
  h->grid.gmin = make_float3(c.grid_min[0], c.grid_min[1], c.grid_min[2]);
  h->grid.gmax = make_float3(c.grid_max[0], c.grid_max[1], c.grid_max[2]);
  h->grid.cell = make_float3(h->cell_size[0], h->cell_size[1], h->cell_size[2]);
  h->grid.dim = make_uint3(c.grid_dim[0], c.grid_dim[1], c.grid_dim[2]);
  h->n_scan_tiles = (h->cells + dsmcb::kScanTile - 1) / dsmcb::kScanTile;
  apply_variant(h, h->variant);
  float capf = c.capacity_factor < 1.f ? 1.f : c.capacity_factor;
  // the Maxwellian and bimodal starts fill the fractional part of n V_c / F_N too
  const double ppc_f = c.part_per_cell ? (double)c.part_per_cell
                                       : (double)c.density * h->cell_volume / c.fnum;
  uint64_t cap = (uint64_t)std::ceil(std::max(ppc_f, (double)h->ppc + 1.0) * h->cells * capf) + 1024;
  if (cap > 0xF0000000ull) {
    delete h;
    return fail(nullptr, DSMC_ERR_CONFIG, "particle capacity exceeds 32-bit indexing");
  }
  h->capacity = (uint32_t)cap;
  setup_inflows(h);

  cudaError_t e = cudaSuccess;
  for (int i = 0; i < 6 && !e; i++) {
    e = dalloc(&h->A[i], h->capacity);
    if (!e) e = dalloc(&h->B[i], h->capacity);
  }
  if (!e) e = dalloc(&h->orig, h->capacity);
  if (!e) e = dalloc(&h->keys, h->capacity);
  if (!e) e = dalloc(&h->ntc_list, 2 * (size_t)h->cells);
  if (!e) e = dalloc(&h->cursor, h->cells + 1);
  if (!e) e = dalloc(&h->count, h->cells + 1);
  if (!e) e = dalloc(&h->start, h->cells + 1);
  if (!e) e = dalloc(&h->tile_sum, h->n_scan_tiles);
  if (!e) e = dalloc(&h->maxrem, h->cells);
  if (!e) e = dalloc(&h->seeds, h->cells);
  if (!e) e = dalloc(&h->acc, 5 * (size_t)h->cells);
  if (!e) e = dalloc(&h->meta, 1);
  if (!e) e = dalloc(&h->inj_rem, 6);
  if (!e) e = dalloc(&h->inj_plan, 12);
  if (e) {
    std::string m = std::string("allocation: ") + cudaGetErrorString(e);
    free_all(h);
    delete h;
    return fail(nullptr, e == cudaErrorMemoryAllocation ? DSMC_ERR_OOM : DSMC_ERR_CUDA, m);
  }
  cudaMemset(h->count, 0, (h->cells + 1) * sizeof(uint32_t));
  cudaMemset(h->start, 0, (h->cells + 1) * sizeof(uint32_t));
  cudaMemset(h->tile_sum, 0, h->n_scan_tiles * sizeof(uint32_t));
  cudaMemset(h->acc, 0, 5 * (size_t)h->cells * sizeof(double));
  cudaMemset(h->meta, 0, sizeof(Meta));
  cudaMemset(h->inj_rem, 0, 6 * sizeof(float));
  // per-cell (sigma*g)max and remainder (InitMaximums, kernels/dsmc_kernel.cu:1104-1120)
  // and HybridTaus seeds (CreateRandomSeedsUint4, :1846-1886), from the seed
  std::vector<float2> mr(h->cells);
  std::vector<uint4> sd(h->cells);
  uint64_t s = c.seed ^ 0x5eed5eed12345678ull;
  for (uint32_t i = 0; i < h->cells; i++) {
    mr[i].x = h->max_rel_vel;
    mr[i].y = (float)((splitmix64(s) >> 40) * (1.0 / 16777216.0));
    uint32_t v[4];
    for (int k = 0; k < 4; k++) v[k] = (uint32_t)(splitmix64(s) % (4294967296ull - 129)) + 128;
    sd[i] = make_uint4(v[0], v[1], v[2], v[3]);
  }
  cudaMemcpy(h->maxrem, mr.data(), h->cells * sizeof(float2), cudaMemcpyHostToDevice);
  cudaMemcpy(h->seeds, sd.data(), h->cells * sizeof(uint4), cudaMemcpyHostToDevice);
  e = cudaDeviceSynchronize();
  if (e) {
    std::string m = std::string("init: ") + cudaGetErrorString(e);
    free_all(h);
    delete h;
    return fail(nullptr, DSMC_ERR_CUDA, m);
  }
  *out = h;
  return DSMC_OK;
}

int dsmc_destroy(dsmc_handle* h) {
  if (!h) return DSMC_ERR_ARG;
  cudaStreamSynchronize(h->stream);
  if (h->side) cudaStreamSynchronize(h->side);
  free_all(h);
  delete h;
  return DSMC_OK;
}

int dsmc_set_stream(dsmc_handle* h, void* stream) {
  if (!h) return DSMC_ERR_ARG;
  h->stream = (cudaStream_t)stream;
  drop_graph(h);
  return DSMC_OK;
}

int dsmc_sync(dsmc_handle* h) {
  if (!h) return DSMC_ERR_ARG;
  CK(h, cudaStreamSynchronize(h->stream), "stream sync");
  return check_device_flags(h);
}

int dsmc_get_info(dsmc_handle* h, dsmc_info* info) {
  if (!h || !info) return DSMC_ERR_ARG;
  Meta m{};
  int st = read_meta(h, m);
  if (st) return st;
  info->part_per_cell = h->ppc;
  info->cells = h->cells;
  info->capacity = h->capacity;
  info->num_particles = h->has_state ? m.n_alive + m.n_pending : 0;
  for (int k = 0; k < 3; k++) info->cell_size[k] = h->cell_size[k];
  info->cell_volume = h->cell_volume;
  info->cross_section = h->cross_section;
  info->max_rel_vel = h->max_rel_vel;
  info->step = h->step;
  info->samples = m.samples;
  info->sim_time = h->sim_time;
  info->particle_steps = m.particle_steps;
  info->injected = m.injected;
  info->removed = m.removed;
  info->giant_cells = m.giant_cells;
  info->mesh_flights = m.n_defer;
  return DSMC_OK;
}

int dsmc_profile(dsmc_handle* h, int enable) {
  if (!h) return DSMC_ERR_ARG;
  if (enable) {
    if (h->ev.empty()) {
      h->ev.resize(2 * kProfPairs);
      h->ev_kernel.resize(kProfPairs);
      for (auto& e : h->ev) CK(h, cudaEventCreate(&e), "event create");
    }
    h->ev_used = 0;
    for (int k = 0; k < 8; k++) { h->prof_ms[k] = 0; h->prof_n[k] = 0; }
  } else {
    prof_flush(h);
  }
  h->profiling = enable != 0;
  h->prof_mask = 0xff;
  return DSMC_OK;
}

int dsmc_profile_mask(dsmc_handle* h, uint32_t slots) {
  if (!h || !h->profiling) return fail(h, DSMC_ERR_STATE, "dsmc_profile_mask needs an open window");
  h->prof_mask = slots & 0xffu;
  return DSMC_OK;
}

int dsmc_profile_read(dsmc_handle* h, double ms[4], uint32_t launches[4]) {
  if (!h || !ms || !launches) return DSMC_ERR_ARG;
  prof_flush(h);
  for (int k = 0; k < 4; k++) { ms[k] = h->prof_ms[k]; launches[k] = h->prof_n[k]; }
  // the cell work of the split variants: order + NTC + flight + mesh + sampling
  for (int k = 4; k < 8; k++) ms[2] += h->prof_ms[k];
  h->profiling = false;
  return DSMC_OK;
}

int dsmc_profile_read_kernels(dsmc_handle* h, int n, double* ms, uint32_t* launches) {
  if (!h || !ms || !launches || n < 1) return DSMC_ERR_ARG;
  prof_flush(h);
  for (int k = 0; k < n; k++) {
    ms[k] = k < 8 ? h->prof_ms[k] : 0.0;
    launches[k] = k < 8 ? h->prof_n[k] : 0u;
  }
  h->profiling = false;
  return DSMC_OK;
}

int dsmc_build_geometry_grid(const float* verts, uint32_t nverts, const uint32_t* tris,
                             uint32_t ntris, const int grid_dim[3], float bbox[6], float cell[3],
                             uint32_t* cell_count, uint32_t* tri_ids, uint64_t cap, uint8_t* flags,
                             uint64_t* n_entries) {
  if (!verts || !tris || !grid_dim || grid_dim[0] <= 0 || grid_dim[1] <= 0 || grid_dim[2] <= 0)
    return DSMC_ERR_ARG;
  for (uint32_t i = 0; i < 3 * ntris; i++)
    if (tris[i] >= nverts) return DSMC_ERR_ARG;
  dsmcb::GeomGrid g;
  dsmcb::build_geometry_grid(verts, nverts, tris, ntris, grid_dim, g);
  if (bbox) std::memcpy(bbox, g.bbox, sizeof(g.bbox));
  if (cell) std::memcpy(cell, g.cell, sizeof(g.cell));
  if (cell_count) std::memcpy(cell_count, g.count.data(), g.count.size() * 4);
  if (flags) std::memcpy(flags, g.flags.data(), g.flags.size());
  if (tri_ids) {
    size_t n = std::min<size_t>(cap, g.tri_ids.size());
    std::memcpy(tri_ids, g.tri_ids.data(), n * 4);
  }
  if (n_entries) *n_entries = g.tri_ids.size();
  return DSMC_OK;
}

// The face normals of the mesh when the caller gives none.
static const float* normals_or_faces(const float* verts, uint32_t nverts, const uint32_t* tris,
                                     uint32_t ntris, const float* normals, std::vector<float>& nrm) {
  if (normals) return normals;
  std::vector<float> v(verts, verts + 3 * (size_t)nverts);
  std::vector<uint32_t> t(tris, tris + 3 * (size_t)ntris);
  dsmcb::face_normals(v, t, nrm);
  return nrm.data();
}

static void free_geometry(dsmcb::GeomDevice& gd) {
  cudaFree(gd.flags);
  cudaFree(gd.se);
  cudaFree(gd.tri);
  cudaFree(gd.plane);
  gd = dsmcb::GeomDevice{};
}

// Takes over the device arrays of a built grid (h->ggrid holds its host copy)
// and fills the clearance table.
static int install_geometry(dsmc_handle* h, dsmcb::GeomDevice& gd) {
  const auto& g = h->ggrid;
  const uint32_t gc = g.dim[0] * g.dim[1] * g.dim[2];
  // Chebyshev cell distance of every cell to the nearest cell holding
  // triangles (multi-source BFS over the 26-neighbourhood): (distance - 1) x
  // the smallest cell size bounds the distance from any point of the cell to
  // the surface; the clearance table refines it next to the body
  std::vector<int> dist(gc, -1);
  std::vector<uint32_t> queue;
  queue.reserve(gc);
  for (uint32_t c = 0; c < gc; c++)
    if (g.count[c]) { dist[c] = 0; queue.push_back(c); }
  for (size_t qi = 0; qi < queue.size(); qi++) {
    const uint32_t c = queue[qi];
    const int cx = (int)(c % g.dim[0]), cy = (int)((c / g.dim[0]) % g.dim[1]),
              cz = (int)(c / (g.dim[0] * g.dim[1]));
    for (int dz = -1; dz <= 1; dz++)
      for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) {
          const int x = cx + dx, y = cy + dy, z = cz + dz;
          if (x < 0 || y < 0 || z < 0 || x >= (int)g.dim[0] || y >= (int)g.dim[1] || z >= (int)g.dim[2])
            continue;
          const uint32_t nc = ((uint32_t)z * g.dim[1] + (uint32_t)y) * g.dim[0] + (uint32_t)x;
          if (dist[nc] < 0) { dist[nc] = dist[c] + 1; queue.push_back(nc); }
        }
  }
  const float cmin = std::min(g.cell[0], std::min(g.cell[1], g.cell[2]));
  // the clearance table lives on the triangle grid refined by cfac (2 unless
  // that would pass 16.8M cells); it is filled on the device below
  const uint32_t cfac = (uint64_t)gc * 8 <= (16u << 20) ? 2u : 1u;
  const uint32_t fc = gc * cfac * cfac * cfac;
  cudaFree(h->gflags);
  cudaFree(h->gclear);
  cudaFree(h->greach);
  h->greach = nullptr;
  cudaFree(h->gslab);
  h->gslab = nullptr;
  cudaFree(h->gse);
  cudaFree(h->gtri);
  cudaFree(h->gplane);
  h->gflags = gd.flags;
  h->gse = gd.se;
  h->gtri = gd.tri;
  h->gplane = gd.plane;
  h->gclear = nullptr;
  gd = dsmcb::GeomDevice{};
  h->has_geom = false;
  CK(h, dalloc(&h->gclear, fc), "geometry alloc");
  {
    h->gcgrid.gmin = make_float3(g.bbox[0], g.bbox[1], g.bbox[2]);
    h->gcgrid.gmax = make_float3(g.bbox[3], g.bbox[4], g.bbox[5]);
    h->gcgrid.cell = make_float3(g.cell[0] / cfac, g.cell[1] / cfac, g.cell[2] / cfac);
    h->gcgrid.dim = make_uint3(g.dim[0] * cfac, g.dim[1] * cfac, g.dim[2] * cfac);
    dsmcb::GeomView gv{};
    gv.grid.gmin = h->gcgrid.gmin;
    gv.grid.gmax = h->gcgrid.gmax;
    gv.grid.cell = make_float3(g.cell[0], g.cell[1], g.cell[2]);
    gv.grid.dim = make_uint3(g.dim[0], g.dim[1], g.dim[2]);
    gv.start_end = h->gse;
    gv.tri = h->gtri;
    int* ddist = nullptr;
    CK(h, cudaMalloc(&ddist, gc * sizeof(int)), "geometry alloc");
    cudaError_t ce = cudaMemcpy(ddist, dist.data(), gc * sizeof(int), cudaMemcpyHostToDevice);
    if (!ce) ce = dsmcb::launch_fine_clearance(gv, h->gcgrid, cfac, ddist, cmin, h->gclear, nullptr);
    if (!ce) ce = cudaDeviceSynchronize();
    cudaFree(ddist);
    CK(h, ce, "clearance table");
    // Per bin entry, how far and how steeply a particle leaving the entry's
    // triangle must fly for the traversal to find no wall.  The set-off of
    // 1 um from the wall must stay several roundings of a coordinate: bodies
    // within 2 m of the origin.
    float mag = 0.f;
    for (int k = 0; k < 6; k++) mag = std::max(mag, std::fabs(g.bbox[k]));
    const size_t entries = g.tri_ids.size();
    gv.plane = h->gplane;
    if (mag < 2.0f && entries) {
      CK(h, dalloc(&h->greach, entries), "geometry alloc");
      ce = dsmcb::launch_entry_reach(gv, (uint32_t)entries, cmin, 1e-7f, 4e-6f, h->greach, nullptr);
      if (!ce) ce = cudaDeviceSynchronize();
      CK(h, ce, "entry reach");
    }
    // per cell, the slab that holds its triangles (the mesh kernel's cell
    // pre-test)
    CK(h, dalloc(&h->gslab, gc), "geometry alloc");
    ce = dsmcb::launch_cell_slab(gv, gc, h->gslab, nullptr);
    if (!ce) ce = cudaDeviceSynchronize();
    CK(h, ce, "cell slabs");
  }
  h->has_geom = true;
  h->cfg.geometry = 1;
  drop_graph(h);
  return DSMC_OK;
}

// The grid of a mesh, binned on the device (dsmc_geomgrid.cu).
int dsmc_set_mesh(dsmc_handle* h, const float* verts, uint32_t nverts, const uint32_t* tris,
                  uint32_t ntris, const float* normals, const int grid_dim[3]) {
  if (!h || !verts || !tris || !grid_dim || ntris == 0) return fail(h, DSMC_ERR_ARG, "bad mesh");
  for (int k = 0; k < 3; k++)
    if (grid_dim[k] <= 0) return fail(h, DSMC_ERR_ARG, "geometry grid dims must be > 0");
  for (uint32_t i = 0; i < 3 * ntris; i++)
    if (tris[i] >= nverts) return fail(h, DSMC_ERR_ARG, "triangle index out of range");
  std::vector<float> nrm;
  normals = normals_or_faces(verts, nverts, tris, ntris, normals, nrm);
  dsmcb::geometry_grid_frame(verts, nverts, grid_dim, h->ggrid);
  dsmcb::GeomDevice gd;
  const cudaError_t e = dsmcb::build_geometry_device(h->ggrid, verts, nverts, tris, ntris, normals, gd);
  if (e) {
    free_geometry(gd);
    return fail(h, DSMC_ERR_CUDA, std::string("geometry grid build: ") + cudaGetErrorString(e));
  }
  return install_geometry(h, gd);
}

int dsmc_set_geometry_grid(dsmc_handle* h, const float bbox[6], const float cell[3],
                           const int dim[3], const uint32_t* cell_count, const uint32_t* tri_ids,
                           const uint8_t* flags, const float* verts, uint32_t nverts,
                           const uint32_t* tris, uint32_t ntris, const float* normals) {
  if (!h || !bbox || !cell || !dim || !cell_count || !flags || !verts || !tris)
    return fail(h, DSMC_ERR_ARG, "null argument");
  for (int k = 0; k < 3; k++)
    if (dim[k] <= 0) return fail(h, DSMC_ERR_ARG, "geometry grid dims must be > 0");
  auto& g = h->ggrid;
  std::memcpy(g.bbox, bbox, sizeof(g.bbox));
  std::memcpy(g.cell, cell, sizeof(g.cell));
  for (int k = 0; k < 3; k++) g.dim[k] = (uint32_t)dim[k];
  uint32_t gc = g.dim[0] * g.dim[1] * g.dim[2];
  g.count.assign(cell_count, cell_count + gc);
  g.flags.assign(flags, flags + gc);
  size_t total = 0;
  for (uint32_t c = 0; c < gc; c++) total += g.count[c];
  if (total && !tri_ids) return fail(h, DSMC_ERR_ARG, "tri_ids missing");
  g.tri_ids.assign(tri_ids, tri_ids + total);
  for (uint32_t t : g.tri_ids)
    if (t >= ntris) return fail(h, DSMC_ERR_ARG, "triangle id out of range");
  for (uint32_t i = 0; i < 3 * ntris; i++)
    if (tris[i] >= nverts) return fail(h, DSMC_ERR_ARG, "triangle index out of range");
  std::vector<float> nrm;
  normals = normals_or_faces(verts, nverts, tris, ntris, normals, nrm);
  // the given binning to the device, then the same entry records
  std::vector<uint32_t> start((size_t)gc + 1, 0u), fl(gc);
  for (uint32_t c = 0; c < gc; c++) {
    start[c + 1] = start[c] + g.count[c];
    fl[c] = g.flags[c] ? 1u : 0u;
  }
  dsmcb::GeomDevice gd;
  uint32_t *d_start = nullptr, *d_ids = nullptr, *d_tris = nullptr;
  float *d_verts = nullptr, *d_normals = nullptr;
  auto up = [](auto** p, const auto* src, size_t n) {
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), (n ? n : 1) * sizeof(**p));
    if (!e && n) e = cudaMemcpy(*p, src, n * sizeof(**p), cudaMemcpyHostToDevice);
    return e;
  };
  cudaError_t e = up(&d_start, start.data(), start.size());
  if (!e) e = up(&d_ids, g.tri_ids.data(), total);
  if (!e) e = up(&d_tris, tris, 3 * (size_t)ntris);
  if (!e) e = up(&d_verts, verts, 3 * (size_t)nverts);
  if (!e) e = up(&d_normals, normals, 3 * (size_t)ntris);
  if (!e) e = up(&gd.flags, fl.data(), fl.size());
  if (!e) e = dsmcb::geometry_entries_device(d_start, d_ids, gc, (uint32_t)total, d_verts, d_tris,
                                             d_normals, gd);
  if (!e) e = cudaDeviceSynchronize();
  cudaFree(d_start);
  cudaFree(d_ids);
  cudaFree(d_tris);
  cudaFree(d_verts);
  cudaFree(d_normals);
  if (e) {
    free_geometry(gd);
    return fail(h, DSMC_ERR_CUDA, std::string("geometry upload: ") + cudaGetErrorString(e));
  }
  return install_geometry(h, gd);
}

int dsmc_get_geometry_grid(dsmc_handle* h, float bbox[6], float cell[3], int dim[3],
                           uint32_t* cell_count, uint32_t* tri_ids, float* planes, uint64_t cap,
                           uint8_t* flags, uint64_t* n_entries) {
  if (!h) return DSMC_ERR_ARG;
  if (!h->has_geom) return fail(h, DSMC_ERR_STATE, "no geometry grid (dsmc_set_mesh)");
  const auto& g = h->ggrid;
  if (bbox) std::memcpy(bbox, g.bbox, sizeof(g.bbox));
  if (cell) std::memcpy(cell, g.cell, sizeof(g.cell));
  if (dim)
    for (int k = 0; k < 3; k++) dim[k] = (int)g.dim[k];
  if (cell_count) std::memcpy(cell_count, g.count.data(), g.count.size() * 4);
  if (flags) std::memcpy(flags, g.flags.data(), g.flags.size());
  const size_t n = std::min<size_t>(cap, g.tri_ids.size());
  if (tri_ids) std::memcpy(tri_ids, g.tri_ids.data(), n * 4);
  if (planes && n) CK(h, cudaMemcpy(planes, h->gplane, n * sizeof(float4), cudaMemcpyDeviceToHost), "read planes");
  if (n_entries) *n_entries = g.tri_ids.size();
  return DSMC_OK;
}

int dsmc_get_entry_reach(dsmc_handle* h, float* out, uint64_t cap, uint64_t* n_entries) {
  if (!h) return DSMC_ERR_ARG;
  if (!h->has_geom) return fail(h, DSMC_ERR_STATE, "no geometry grid (dsmc_set_mesh)");
  const size_t total = h->greach ? h->ggrid.tri_ids.size() : 0;
  const size_t n = std::min<size_t>(cap, total);
  if (out && n) CK(h, cudaMemcpy(out, h->greach, n * sizeof(float2), cudaMemcpyDeviceToHost), "read reach");
  if (n_entries) *n_entries = total;
  return DSMC_OK;
}

int dsmc_get_cell_slabs(dsmc_handle* h, float* out, uint64_t cap, uint64_t* n_cells) {
  if (!h) return DSMC_ERR_ARG;
  if (!h->has_geom) return fail(h, DSMC_ERR_STATE, "no geometry grid (dsmc_set_mesh)");
  const auto& g = h->ggrid;
  const size_t total = h->gslab ? (size_t)g.dim[0] * g.dim[1] * g.dim[2] : 0;
  const size_t n = std::min<size_t>(cap, total);
  if (out && n) CK(h, cudaMemcpy(out, h->gslab, n * sizeof(float4), cudaMemcpyDeviceToHost), "read slabs");
  if (n_cells) *n_cells = total;
  return DSMC_OK;
}

int dsmc_read_raw_mesh(const char* path, float* verts, uint32_t* nverts, uint32_t* tris,
                       uint32_t* ntris, float* face_normals) {
  if (!path || !nverts || !ntris) return DSMC_ERR_ARG;
  std::vector<float> v, fn;
  std::vector<uint32_t> t;
  int st = dsmcb::read_raw_mesh(path, v, t, fn);
  if (st) return st;
  *nverts = (uint32_t)(v.size() / 3);
  *ntris = (uint32_t)(t.size() / 3);
  if (verts) std::memcpy(verts, v.data(), v.size() * 4);
  if (tris) std::memcpy(tris, t.data(), t.size() * 4);
  if (face_normals) {
    if (fn.size() == t.size()) std::memcpy(face_normals, fn.data(), fn.size() * 4);
    else {
      std::vector<float> n;
      dsmcb::face_normals(v, t, n);
      std::memcpy(face_normals, n.data(), n.size() * 4);
    }
  }
  return DSMC_OK;
}

int dsmc_mesh_icosphere(int level, float radius, const float center[3], float* verts,
                        uint32_t* nverts, uint32_t* tris, uint32_t* ntris) {
  if (level < 0 || level > 8 || !(radius > 0) || !center || !nverts || !ntris) return DSMC_ERR_ARG;
  std::vector<float> v;
  std::vector<uint32_t> t;
  dsmcb::mesh_icosphere(level, radius, center, v, t);
  *nverts = (uint32_t)(v.size() / 3);
  *ntris = (uint32_t)(t.size() / 3);
  if (verts) std::memcpy(verts, v.data(), v.size() * 4);
  if (tris) std::memcpy(tris, t.data(), t.size() * 4);
  return DSMC_OK;
}

int dsmc_mesh_capsule(float nose_radius, float cone_half_angle_deg, float length,
                      const float nose_center[3], uint32_t ntarget, uint64_t seed, float* verts,
                      uint32_t* nverts, uint32_t* tris, uint32_t* ntris) {
  if (!(nose_radius > 0) || !(cone_half_angle_deg > 0) || cone_half_angle_deg >= 90 ||
      !(length > nose_radius) || !nose_center || !nverts || !ntris)
    return DSMC_ERR_ARG;
  std::vector<float> v;
  std::vector<uint32_t> t;
  dsmcb::mesh_capsule(nose_radius, cone_half_angle_deg, length, nose_center, ntarget, seed, v, t);
  *nverts = (uint32_t)(v.size() / 3);
  *ntris = (uint32_t)(t.size() / 3);
  if (verts) std::memcpy(verts, v.data(), v.size() * 4);
  if (tris) std::memcpy(tris, t.data(), t.size() * 4);
  return DSMC_OK;
}

// Cells whose corners touch a flagged geometry cell get no particles
// (IsGeometryInCell, kernels/dsmc_kernel.cu:478-546).
static bool geometry_in_cell(const dsmcb::GeomGrid& g, const float cmin[3], const float cs[3]) {
  auto flagged = [&](float x, float y, float z) {
    if (x < g.bbox[0] || y < g.bbox[1] || z < g.bbox[2] || x > g.bbox[3] || y > g.bbox[4] ||
        z > g.bbox[5])
      return false;
    auto cvt = [](float f) -> uint32_t { return f > 0.f ? (f >= 4294967296.0f ? 0xffffffffu : (uint32_t)f) : 0u; };
    uint32_t ix = std::min(cvt((x - g.bbox[0]) / g.cell[0]), g.dim[0] - 1);
    uint32_t iy = std::min(cvt((y - g.bbox[1]) / g.cell[1]), g.dim[1] - 1);
    uint32_t iz = std::min(cvt((z - g.bbox[2]) / g.cell[2]), g.dim[2] - 1);
    return g.flags[iz * g.dim[0] * g.dim[1] + iy * g.dim[0] + ix] != 0;
  };
  float x0 = cmin[0], y0 = cmin[1], z0 = cmin[2];
  float x1 = x0 + cs[0], y1 = y0 + cs[1], z1 = z0 + cs[2];
  return flagged(x0, y0, z0) || flagged(x1, y0, z0) || flagged(x1, y1, z0) ||
         flagged(x1, y1, z1) || flagged(x0, y1, z0) || flagged(x0, y1, z1) ||
         flagged(x0, y0, z1) || flagged(x1, y0, z1);
}

namespace {

// Scratch of the extension fills inside the sampling accumulators (40 bytes
// per cell, reset after the fill): per-cell Maxwellian state, an outside
// point, the outside fraction and the free-stream share of a two-stream fill.
float4* fill_state(dsmc_handle* h) { return reinterpret_cast<float4*>(h->acc); }
float4* fill_point(dsmc_handle* h) { return reinterpret_cast<float4*>(h->acc) + h->cells; }
float* fill_frac(dsmc_handle* h) { return reinterpret_cast<float*>(fill_point(h) + h->cells); }
float* fill_mix(dsmc_handle* h) { return fill_frac(h) + h->cells; }
static_assert(2 * sizeof(float4) + 2 * sizeof(float) <= 5 * sizeof(double),
              "fill scratch must fit the accumulators");

// Fraction of every cell outside the mesh (all ones without one).
int outside_fractions(dsmc_handle* h, std::vector<float>& frac) {
  frac.assign(h->cells, 1.f);
  if (!(h->has_geom && h->cfg.geometry)) return DSMC_OK;
  CK(h, dsmcb::launch_outside_fraction(h->grid, base_params(h, h->cfg.dt).geom, h->cells,
                                       fill_frac(h), fill_point(h), h->stream), "outside fraction");
  CK(h, cudaMemcpyAsync(frac.data(), fill_frac(h), h->cells * sizeof(float), cudaMemcpyDeviceToHost,
                        h->stream), "outside fraction");
  CK(h, cudaStreamSynchronize(h->stream), "outside fraction");
  return DSMC_OK;
}

// Uploads the per-cell slots and counts, fills, resets the accumulators and
// indexes the new state.
int finish_fill(dsmc_handle* h, dsmcb::InitParams& ip, const std::vector<uint32_t>& slot,
                const std::vector<uint32_t>& count, uint64_t n, uint32_t* n_out) {
  if (n > h->capacity) return fail(h, DSMC_ERR_CAPACITY, "initial particles exceed capacity");
  CK(h, cudaMemcpyAsync(h->start, slot.data(), (h->cells + 1) * 4, cudaMemcpyHostToDevice, h->stream),
     "init upload");
  CK(h, cudaMemcpyAsync(h->count, count.data(), (h->cells + 1) * 4, cudaMemcpyHostToDevice, h->stream),
     "init upload");
  ip.grid = h->grid;
  ip.cells = h->cells;
  ip.cell_slot = h->start;
  ip.cell_count = h->count;
  ip.out = soa_of(h->A);
  CK(h, dsmcb::launch_init_fill(ip, h->stream), "init fill");
  CK(h, cudaMemsetAsync(h->acc, 0, 5 * (size_t)h->cells * sizeof(double), h->stream), "reset samples");
  int st = reindex(h, (uint32_t)n);
  if (st) return st;
  Meta m{};
  st = read_meta(h, m);
  if (st) return st;
  m.samples = 0;
  CK(h, cudaMemcpy(&h->meta->samples, &m.samples, 4, cudaMemcpyHostToDevice), "meta");
  if (n_out) *n_out = (uint32_t)n;
  return DSMC_OK;
}

double unit_draw(uint64_t& mix) { return (double)(splitmix64(mix) >> 11) / 9007199254740992.0; }

}  // namespace

int dsmc_init_state(dsmc_handle* h, const float stream_vel[3], uint32_t* n_out) {
  if (!h) return DSMC_ERR_ARG;
  const dsmc_config& c = h->cfg;
  std::vector<uint32_t> slot(h->cells + 1), count(h->cells + 1, 0u);
  uint64_t n = 0;
  const bool geo = h->has_geom && c.geometry;
  const bool reference = c.init_kind == DSMC_INIT_REFERENCE;
  dsmcb::InitParams ip{};
  uint64_t mix = c.seed ^ 0x5DEECE66Dull;
  if (reference) {
    // InitSystemState / GenerateInitialVelocities (kernels/dsmc_kernel.cu:394-427):
    // ppc = floor(n V_c / F_N) particles in every cell the mesh does not touch
    for (uint32_t cell = 0; cell < h->cells; cell++) {
      uint32_t cx = cell % c.grid_dim[0], cy = (cell / c.grid_dim[0]) % c.grid_dim[1],
               cz = cell / (c.grid_dim[0] * c.grid_dim[1]);
      float cmin[3] = {c.grid_min[0] + cx * h->cell_size[0], c.grid_min[1] + cy * h->cell_size[1],
                       c.grid_min[2] + cz * h->cell_size[2]};
      if (geo && geometry_in_cell(h->ggrid, cmin, h->cell_size)) {
        slot[cell] = 0xffffffffu;
        continue;
      }
      slot[cell] = (uint32_t)n;
      count[cell] = h->ppc;
      n += h->ppc;
    }
    ip.ppc = h->ppc;
  } else {
    // the Maxwellian and bimodal starts: n V_c / F_N particles times the part
    // of the cell outside the body, rounded stochastically from the seed;
    // positions inside the body are drawn again
    std::vector<float> frac;
    int st = outside_fractions(h, frac);
    if (st) return st;
    const double ppc_f = c.part_per_cell ? (double)c.part_per_cell
                                         : (double)c.density * h->cell_volume / c.fnum;
    uint32_t kmax = 0;
    for (uint32_t cell = 0; cell < h->cells; cell++) {
      const double expect = ppc_f * frac[cell];
      const double fl = std::floor(expect);
      const uint32_t k = (uint32_t)fl + (unit_draw(mix) < expect - fl ? 1u : 0u);
      slot[cell] = (uint32_t)n;
      count[cell] = k;
      kmax = std::max(kmax, k);
      n += k;
    }
    ip.ppc = kmax;
    ip.reject_inside = geo;
    if (geo) {
      ip.geom = base_params(h, c.dt).geom;
      ip.cell_point = fill_point(h);
    }
  }
  ip.kind = c.init_kind;
  ip.vstd = std::sqrt(1.3806e-23f * c.temp / c.gas_mass);
  ip.vstd2 = std::sqrt(1.3806e-23f * (c.init_temp2 > 0 ? c.init_temp2 : c.temp) / c.gas_mass);
  ip.vmp = std::sqrt(2 * 1.3806e-23f * c.temp / c.gas_mass);
  const float* sv = stream_vel ? stream_vel : c.stream_vel;
  ip.stream = make_float3(sv[0], sv[1], sv[2]);
  ip.seed = make_uint2((uint32_t)c.seed, (uint32_t)(c.seed >> 32));
  return finish_fill(h, ip, slot, count, n, n_out);
}

namespace {

// Free-stream share alpha of a cell with mean velocity u and temperature T
// seen as a mixture of the free stream (U, T_inf) and a Maxwellian at the
// wall temperature T_w with drift u_b: the mixture's mean and energy match
// the cell's when
//   alpha e_inf + (1 - alpha) e_w + |u - alpha U|^2 / (1 - alpha) = 3kT/m + |u|^2
// (e = 3kT/m + |drift|^2 of a component), solved by bisection on
// [0, 0.98]; 0 where the cell is colder than the wall or no root lies there.
double two_stream_share(const double u[3], double T, const double U[3], double T_inf, double T_w,
                        double kb_m) {
  const double e_inf = 3.0 * kb_m * T_inf + U[0] * U[0] + U[1] * U[1] + U[2] * U[2];
  const double e_w = 3.0 * kb_m * T_w;
  const double rhs = 3.0 * kb_m * T + u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
  auto f = [&](double a) {
    const double d0 = u[0] - a * U[0], d1 = u[1] - a * U[1], d2 = u[2] - a * U[2];
    return a * e_inf + (1.0 - a) * e_w + (d0 * d0 + d1 * d1 + d2 * d2) / (1.0 - a) - rhs;
  };
  double lo = 0.0, hi = 0.98;
  if (!(f(lo) < 0.0 && f(hi) > 0.0)) return 0.0;
  for (int it = 0; it < 60; it++) {
    const double mid = 0.5 * (lo + hi);
    (f(mid) > 0.0 ? hi : lo) = mid;
  }
  return 0.5 * (lo + hi);
}

// dsmc_init_from_fields and its two-stream form (weight > 0).
int seed_from_fields(dsmc_handle* h, const float* fields5, float weight, uint32_t* n_out) {
  if (!h || !fields5) return fail(h, DSMC_ERR_ARG, "null argument");
  const dsmc_config& c = h->cfg;
  if (!(weight >= 0.f && weight <= 1.f)) return fail(h, DSMC_ERR_ARG, "two-stream weight outside [0, 1]");
  const bool two = weight > 0.f;
  if (two && !(c.wall_temp > 0.f)) return fail(h, DSMC_ERR_ARG, "two-stream fill needs a wall temperature");
  std::vector<float> frac;
  int st = outside_fractions(h, frac);
  if (st) return st;
  std::vector<uint32_t> slot(h->cells + 1), count(h->cells + 1, 0u);
  std::vector<float4> state(h->cells);
  std::vector<float2> maxrem(h->cells);
  std::vector<float> share(two ? h->cells : 0);
  const double U[3] = {c.stream_vel[0], c.stream_vel[1], c.stream_vel[2]};
  const bool geo = h->has_geom && c.geometry;
  const float kb_m = 1.3806e-23f / c.gas_mass;
  uint64_t mix = c.seed ^ 0x2545F4914F6CDD1Dull;
  uint64_t n = 0;
  uint32_t kmax = 0;
  for (uint32_t cell = 0; cell < h->cells; cell++) {
    const float* f = fields5 + 5 * (size_t)cell;
    // n is averaged over the whole cell volume (as dsmc_read_fields gives
    // it), so a cell the body cuts receives its n V_c / F_N particles in the
    // part outside the body; a cell the body covers stays empty
    const double expect = (std::isfinite(f[0]) && f[0] > 0.f && frac[cell] > 0.f)
                              ? (double)f[0] * h->cell_volume / c.fnum : 0.0;
    const double fl = std::floor(expect);
    const uint32_t k = (uint32_t)fl + (unit_draw(mix) < expect - fl ? 1u : 0u);
    slot[cell] = (uint32_t)n;
    count[cell] = k;
    kmax = std::max(kmax, k);
    n += k;
    const float T = (std::isfinite(f[4]) && f[4] > 0.f) ? f[4] : c.temp;
    state[cell] = make_float4(std::isfinite(f[1]) ? f[1] : 0.f, std::isfinite(f[2]) ? f[2] : 0.f,
                              std::isfinite(f[3]) ? f[3] : 0.f, std::sqrt(kb_m * T));
    if (two) {
      // the share alpha from the free stream, the rest a Maxwellian whose
      // drift and temperature keep the cell's mean and energy (the wall
      // temperature itself at weight 1)
      const double u[3] = {state[cell].x, state[cell].y, state[cell].z};
      const double a = weight * two_stream_share(u, T, U, c.temp, c.wall_temp, kb_m);
      share[cell] = (float)a;
      if (a > 0.0) {
        double ub[3], ub2 = 0.0, uu = 0.0, UU = 0.0;
        for (int q = 0; q < 3; q++) {
          ub[q] = (u[q] - a * U[q]) / (1.0 - a);
          ub2 += ub[q] * ub[q];
          uu += u[q] * u[q];
          UU += U[q] * U[q];
        }
        const double e = (3.0 * kb_m * T + uu - a * (3.0 * kb_m * c.temp + UU)) / (1.0 - a) - ub2;
        state[cell] = make_float4((float)ub[0], (float)ub[1], (float)ub[2],
                                  (float)std::sqrt(std::max(e / 3.0, 0.0)));
      }
    }
    // (sigma g)max scaled to the cell's temperature like the initial value
    // (InitSimulationProperties, kernels/dsmc_kernel.cu:329-331)
    maxrem[cell] = make_float2(h->max_rel_vel * std::sqrt(std::max(T, c.temp) / c.temp),
                               (float)unit_draw(mix));
  }
  CK(h, cudaMemcpyAsync(fill_state(h), state.data(), h->cells * sizeof(float4), cudaMemcpyHostToDevice,
                        h->stream), "seed upload");
  CK(h, cudaMemcpyAsync(h->maxrem, maxrem.data(), h->cells * sizeof(float2), cudaMemcpyHostToDevice,
                        h->stream), "seed upload");
  if (two)
    CK(h, cudaMemcpyAsync(fill_mix(h), share.data(), h->cells * sizeof(float), cudaMemcpyHostToDevice,
                          h->stream), "seed upload");
  dsmcb::InitParams ip{};
  ip.ppc = kmax;
  ip.kind = DSMC_INIT_MAXWELL;
  ip.seed = make_uint2((uint32_t)c.seed, (uint32_t)(c.seed >> 32));
  ip.cell_state = fill_state(h);
  if (two) {
    ip.cell_mix = fill_mix(h);
    ip.stream = make_float3(c.stream_vel[0], c.stream_vel[1], c.stream_vel[2]);
    ip.vstd = std::sqrt(kb_m * c.temp);
  }
  ip.reject_inside = geo;
  if (geo) {
    ip.geom = base_params(h, c.dt).geom;
    ip.cell_point = fill_point(h);
  }
  return finish_fill(h, ip, slot, count, n, n_out);
}

}  // namespace

int dsmc_init_from_fields(dsmc_handle* h, const float* fields5, uint32_t* n_out) {
  return seed_from_fields(h, fields5, 0.f, n_out);
}

int dsmc_init_from_fields_two_stream(dsmc_handle* h, const float* fields5, float weight, uint32_t* n_out) {
  return seed_from_fields(h, fields5, weight, n_out);
}

int dsmc_upload_state(dsmc_handle* h, const float* pos, const float* vel, uint32_t n, int soa) {
  if (!h || (n && (!pos || (!vel && !soa)))) return fail(h, DSMC_ERR_ARG, "null state");
  if (n > h->capacity) return fail(h, DSMC_ERR_CAPACITY, "state exceeds particle capacity");
  if (soa) {
    for (int k = 0; k < 6; k++)
      CK(h, cudaMemcpyAsync(h->A[k], pos + (size_t)k * n, (size_t)n * 4, cudaMemcpyHostToDevice,
                            h->stream), "upload");
  } else {
    std::vector<float> t((size_t)n * 6);
    for (uint32_t i = 0; i < n; i++)
      for (int k = 0; k < 3; k++) {
        t[(size_t)k * n + i] = pos[4 * (size_t)i + k];
        t[(size_t)(3 + k) * n + i] = vel[4 * (size_t)i + k];
      }
    for (int k = 0; k < 6; k++)
      CK(h, cudaMemcpyAsync(h->A[k], t.data() + (size_t)k * n, (size_t)n * 4,
                            cudaMemcpyHostToDevice, h->stream), "upload");
    CK(h, cudaStreamSynchronize(h->stream), "upload sync");
  }
  return reindex(h, n);
}

int dsmc_download_state(dsmc_handle* h, float* pos, float* vel, uint32_t* n_io, int soa) {
  if (!h || !n_io) return fail(h, DSMC_ERR_ARG, "null argument");
  Meta m{};
  int st = read_meta(h, m);
  if (st) return st;
  uint32_t n = h->has_state ? m.n_alive + m.n_pending : 0;
  uint32_t cap = *n_io;
  *n_io = n;
  if (!pos) return DSMC_OK;
  if (cap < n) return fail(h, DSMC_ERR_ARG, "output buffer too small");
  if (soa) {
    for (int k = 0; k < 6; k++)
      CK(h, cudaMemcpy(pos + (size_t)k * n, h->A[k], (size_t)n * 4, cudaMemcpyDeviceToHost),
         "download");
  } else {
    std::vector<float> t((size_t)n * 6);
    for (int k = 0; k < 6; k++)
      CK(h, cudaMemcpy(t.data() + (size_t)k * n, h->A[k], (size_t)n * 4, cudaMemcpyDeviceToHost),
         "download");
    for (uint32_t i = 0; i < n; i++) {
      for (int k = 0; k < 3; k++) {
        pos[4 * (size_t)i + k] = t[(size_t)k * n + i];
        if (vel) vel[4 * (size_t)i + k] = t[(size_t)(3 + k) * n + i];
      }
      pos[4 * (size_t)i + 3] = 1.f;
      if (vel) vel[4 * (size_t)i + 3] = 0.f;
    }
  }
  return DSMC_OK;
}

int dsmc_read_keys(dsmc_handle* h, uint32_t* keys, uint32_t* n_io) {
  if (!h || !n_io) return fail(h, DSMC_ERR_ARG, "null argument");
  Meta m{};
  int st = read_meta(h, m);
  if (st) return st;
  const uint32_t n = h->has_state ? m.n_alive + m.n_pending : 0;
  const uint32_t cap = *n_io;
  *n_io = n;
  if (!keys) return DSMC_OK;
  if (cap < n) return fail(h, DSMC_ERR_ARG, "output buffer too small");
  CK(h, cudaMemcpy(keys, h->keys, (size_t)n * 4, cudaMemcpyDeviceToHost), "download keys");
  return DSMC_OK;
}

int dsmc_set_cell_state(dsmc_handle* h, const float* maxrem, const uint32_t* seeds) {
  if (!h) return DSMC_ERR_ARG;
  if (maxrem)
    CK(h, cudaMemcpy(h->maxrem, maxrem, h->cells * sizeof(float2), cudaMemcpyHostToDevice), "upload");
  if (seeds)
    CK(h, cudaMemcpy(h->seeds, seeds, h->cells * sizeof(uint4), cudaMemcpyHostToDevice), "upload");
  return DSMC_OK;
}

int dsmc_get_cell_state(dsmc_handle* h, float* maxrem, uint32_t* seeds) {
  if (!h) return DSMC_ERR_ARG;
  CK(h, cudaStreamSynchronize(h->stream), "sync");
  if (maxrem)
    CK(h, cudaMemcpy(maxrem, h->maxrem, h->cells * sizeof(float2), cudaMemcpyDeviceToHost), "download");
  if (seeds)
    CK(h, cudaMemcpy(seeds, h->seeds, h->cells * sizeof(uint4), cudaMemcpyDeviceToHost), "download");
  return DSMC_OK;
}

// InitGPUTwisters + InitMersenneTwisters (kernels/mtwister.cu:46-68,
// kernels/dsmc_kernel.cu:548-569) and InitMaximums (:1104-1120) for the
// handle's cells; the -mt collisions (ComputeBirdCollisionsDev, :1002-1089)
// from then on.
int dsmc_set_twisters(dsmc_handle* h, const uint32_t* cfg4, const uint32_t* state21,
                      int init_maximums) {
  if (!h || !cfg4) return DSMC_ERR_ARG;
  if (h->cfg.rng != DSMC_RNG_TAUS)
    return fail(h, DSMC_ERR_CONFIG, "the -mt collisions replace the reference RNG mode (rng taus)");
  if (state21)
    for (uint32_t c = 0; c < h->cells; c++)
      if (state21[21 * (size_t)c] >= 19u)
        return fail(h, DSMC_ERR_ARG, "twister state: iState must be below 19");
  if (!h->mt_state) {
    CK(h, cudaMalloc(&h->mt_state, (size_t)h->cells * 21 * sizeof(uint32_t)), "twister states");
    CK(h, cudaMalloc(&h->mt_cfg, (size_t)h->cells * sizeof(uint4)), "twister parameters");
  }
  CK(h, cudaMemcpyAsync(h->mt_cfg, cfg4, (size_t)h->cells * sizeof(uint4), cudaMemcpyHostToDevice,
                        h->stream), "twister parameters");
  if (init_maximums) {
    // the reference's order (include/gpu_dsmc.inl:363-367): InitBirdData's
    // InitMaximums draws from the twister states before InitMersenneTwisters
    // initialises them, i.e. from zeroed states, so every remainder is
    // (0 + 1) / 2^32
    CK(h, cudaMemsetAsync(h->mt_state, 0, (size_t)h->cells * 21 * sizeof(uint32_t), h->stream),
       "twister states");
    CK(h, dsmcb::launch_mt_maximums(h->mt_cfg, h->mt_state, h->maxrem, h->max_rel_vel, h->cells,
                                    h->stream), "InitMaximums");
  }
  if (state21)
    CK(h, cudaMemcpyAsync(h->mt_state, state21, (size_t)h->cells * 21 * sizeof(uint32_t),
                          cudaMemcpyHostToDevice, h->stream), "twister states");
  else
    CK(h, dsmcb::launch_mt_init(h->mt_cfg, h->mt_state, h->cells, h->stream), "twister init");
  CK(h, cudaStreamSynchronize(h->stream), "twisters");
  if (!dsmcb::cell_kernel_is_warp(h->variant)) apply_variant(h, 5);
  h->mt_on = true;
  drop_graph(h);
  return DSMC_OK;
}

int dsmc_read_twisters(const char* path, uint32_t seed, uint32_t count, uint32_t* cfg4) {
  if (!path || (count && !cfg4)) return DSMC_ERR_ARG;
  std::ifstream f(path, std::ios::binary);
  if (!f) return DSMC_ERR_IO;
  f.read(reinterpret_cast<char*>(cfg4), (std::streamsize)count * 16);
  if (!f) return DSMC_ERR_IO;
  uint64_t s = seed;
  for (uint32_t i = 0; i < count; i++) {
    s = (s * 279470273ull) % 4294967291ull;
    cfg4[4 * (size_t)i + 3] = (uint32_t)s;
  }
  return DSMC_OK;
}

int dsmc_get_twisters(dsmc_handle* h, uint32_t* state21) {
  if (!h || !state21) return DSMC_ERR_ARG;
  if (!h->mt_on) return fail(h, DSMC_ERR_STATE, "no twisters set (dsmc_set_twisters)");
  CK(h, cudaStreamSynchronize(h->stream), "sync");
  CK(h, cudaMemcpy(state21, h->mt_state, (size_t)h->cells * 21 * sizeof(uint32_t),
                   cudaMemcpyDeviceToHost), "twister states");
  return DSMC_OK;
}

int dsmc_step(dsmc_handle* h, float dt, int nsteps) {
  if (!h || nsteps < 0) return DSMC_ERR_ARG;
  if (!h->has_state) return fail(h, DSMC_ERR_STATE, "dsmc_step before dsmc_init_state/upload");
  CK(h, ensure_side(h), "side stream");
  for (int i = 0; i < nsteps; i++) {
    cudaError_t e = enqueue_step(h, dt);
    if (e) return cuda_fail(h, e, "step launch");
    h->step++;
    h->sim_time += dt;
  }
  return DSMC_OK;
}

int dsmc_step_graph(dsmc_handle* h, float dt, int nsteps) {
  if (!h || nsteps < 0) return DSMC_ERR_ARG;
  if (!h->has_state) return fail(h, DSMC_ERR_STATE, "dsmc_step before dsmc_init_state/upload");
  CK(h, ensure_side(h), "side stream");
  const uint32_t want_mask = h->profiling ? h->prof_mask : 0u;
  if (!h->graph_exec || h->graph_dt != dt || h->graph_prof_mask != want_mask) {
    drop_graph(h);
    while (h->cap_ev.size() < 2 * kCapPairs) {
      cudaEvent_t ev = nullptr;
      CK(h, cudaEventCreate(&ev), "graph event create");
      h->cap_ev.push_back(ev);
    }
    cudaStream_t cap = nullptr;
    CK(h, cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "graph stream");
    cudaStream_t saved = h->stream;
    h->capturing = true;  // profiled kernels get event-record nodes
    h->stream = cap;
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (!e) e = enqueue_step(h, dt);
    cudaError_t e2 = cudaStreamEndCapture(cap, &h->graph);
    h->stream = saved;
    h->capturing = false;
    cudaStreamDestroy(cap);
    if (e || e2) return cuda_fail(h, e ? e : e2, "graph capture");
    // the event-record nodes, matched to their pairs by placeholder event
    h->gev_node.assign(2 * h->cap_slot.size(), nullptr);
    if (!h->cap_slot.empty()) {
      size_t nn = 0;
      CK(h, cudaGraphGetNodes(h->graph, nullptr, &nn), "graph nodes");
      std::vector<cudaGraphNode_t> nodes(nn);
      CK(h, cudaGraphGetNodes(h->graph, nodes.data(), &nn), "graph nodes");
      for (cudaGraphNode_t nd : nodes) {
        cudaGraphNodeType ty;
        CK(h, cudaGraphNodeGetType(nd, &ty), "graph node type");
        if (ty != cudaGraphNodeTypeEventRecord) continue;
        cudaEvent_t ev = nullptr;
        CK(h, cudaGraphEventRecordNodeGetEvent(nd, &ev), "graph event node");
        for (size_t k = 0; k < h->gev_node.size(); k++)
          if (h->cap_ev[k] == ev) h->gev_node[k] = nd;
      }
      for (cudaGraphNode_t nd : h->gev_node)
        if (!nd) return fail(h, DSMC_ERR_CUDA, "graph capture: an event-record node is missing");
    }
    CK(h, cudaGraphInstantiate(&h->graph_exec, h->graph, 0), "graph instantiate");
    h->graph_dt = dt;
    h->graph_prof_mask = want_mask;
  }
  for (int i = 0; i < nsteps; i++) {
    // fresh events for this replay's profiled kernels
    for (size_t k = 0; k < h->cap_slot.size(); k++) {
      if (h->ev_used == kProfPairs) prof_flush(h);
      const size_t j = h->ev_used++;
      h->ev_kernel[j] = h->cap_slot[k];
      CK(h, cudaGraphExecEventRecordNodeSetEvent(h->graph_exec, h->gev_node[2 * k], h->ev[2 * j]),
         "graph event");
      CK(h, cudaGraphExecEventRecordNodeSetEvent(h->graph_exec, h->gev_node[2 * k + 1],
                                                 h->ev[2 * j + 1]),
         "graph event");
    }
    CK(h, cudaGraphLaunch(h->graph_exec, h->stream), "graph launch");
    h->step++;
    h->sim_time += dt;
  }
  return DSMC_OK;
}

int dsmc_set_kernel_variant(dsmc_handle* h, int variant) {
  if (!h || variant < 0 || variant >= dsmcb::cell_kernel_variants()) return DSMC_ERR_ARG;
  if (h->mt_on && !dsmcb::cell_kernel_is_warp(variant))
    return fail(h, DSMC_ERR_CONFIG, "the -mt collisions run with the split kernels (variants 4 and up)");
  apply_variant(h, variant);
  return DSMC_OK;
}

int dsmc_kernel_variant_count(void) { return dsmcb::cell_kernel_variants(); }

int dsmc_get_kernel_variant(dsmc_handle* h, int* variant, int* chunk_capacity) {
  if (!h) return DSMC_ERR_ARG;
  if (variant) *variant = h->variant;
  if (chunk_capacity) *chunk_capacity = dsmcb::cell_kernel_chunk_capacity(h->variant);
  return DSMC_OK;
}

constexpr int kFirstTunedVariant = 4;

int dsmc_autotune(dsmc_handle* h, float dt, int steps, int* best, float* ms_per_step) {
  if (!h || steps < 1) return DSMC_ERR_ARG;
  if (!h->has_state) return fail(h, DSMC_ERR_STATE, "autotune needs a particle state");
  const int nv = dsmcb::cell_kernel_variants();
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CK(h, cudaEventCreate(&e0), "event");
  cudaError_t ce = cudaEventCreate(&e1);
  if (ce) {
    cudaEventDestroy(e0);
    return cuda_fail(h, ce, "event");
  }
  int st = DSMC_OK, pick = h->variant;
  float best_ms = 0.f;
  // the split variants only: the fused CTA-wide kernel (variants 0-3) takes
  // two to three times as long on every workload measured, and stays
  // selectable by dsmc_set_kernel_variant
  const int v0 = kFirstTunedVariant;
  if (ms_per_step)
    for (int v = 0; v < v0; v++) ms_per_step[v] = 0.f;
  for (int v = v0; v < nv && st == DSMC_OK; v++) {
    apply_variant(h, v);
    st = dsmc_step_graph(h, dt, 2);  // capture + warm-up
    if (st) break;
    ce = cudaEventRecord(e0, h->stream);
    if (!ce) st = dsmc_step_graph(h, dt, steps);
    if (!ce && !st) ce = cudaEventRecord(e1, h->stream);
    if (!ce && !st) ce = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (!ce && !st) ce = cudaEventElapsedTime(&ms, e0, e1);
    if (ce) st = cuda_fail(h, ce, "autotune timing");
    if (st) break;
    ms /= (float)steps;
    if (ms_per_step) ms_per_step[v] = ms;
    if (v == v0 || ms < best_ms) {
      best_ms = ms;
      pick = v;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  apply_variant(h, pick);
  if (best) *best = pick;
  if (st) return st;
  return check_device_flags(h);
}

int dsmc_sample(dsmc_handle* h) {
  if (!h) return DSMC_ERR_ARG;
  if (!h->has_state) return fail(h, DSMC_ERR_STATE, "no particle state");
  if (h->step == 0) return fail(h, DSMC_ERR_STATE, "sampling needs the cell order of a step");
  CK(h, dsmcb::launch_sample_cells(h->A[3], h->A[4], h->A[5], h->start, h->cells, h->acc, h->cells,
                                   1, h->stream), "sample");
  // one more sampling pass
  static const uint32_t one = 1;
  (void)one;
  Meta m{};
  int st = read_meta(h, m);
  if (st) return st;
  m.samples += 1;
  CK(h, cudaMemcpy(&h->meta->samples, &m.samples, 4, cudaMemcpyHostToDevice), "meta");
  return DSMC_OK;
}

int dsmc_reset_samples(dsmc_handle* h) {
  if (!h) return DSMC_ERR_ARG;
  CK(h, cudaMemsetAsync(h->acc, 0, 5 * (size_t)h->cells * sizeof(double), h->stream), "memset");
  CK(h, cudaMemsetAsync(&h->meta->samples, 0, 4, h->stream), "memset");
  CK(h, cudaStreamSynchronize(h->stream), "sync");
  return DSMC_OK;
}

// The per-cell sums (fields == 0) or fields cell-major into host memory:
// formed on the device into a buffer kept for the purpose, one copy out.
static int read_cell_major(dsmc_handle* h, int fields, double* out, uint32_t* nsamples) {
  Meta m{};
  int st = read_meta(h, m);
  if (st) return st;
  if (nsamples) *nsamples = m.samples;
  if (!out) return DSMC_OK;
  if (!h->cellbuf) CK(h, dalloc(&h->cellbuf, 5 * (size_t)h->cells), "cell buffer alloc");
  CK(h, dsmcb::launch_cell_fields(h->acc, h->cells, (double)h->cfg.fnum, (double)h->cell_volume,
                                  m.samples, (double)h->cfg.gas_mass, fields, h->cellbuf, h->stream),
     "cell fields");
  CK(h, cudaMemcpyAsync(out, h->cellbuf, 5 * (size_t)h->cells * sizeof(double),
                        cudaMemcpyDeviceToHost, h->stream), "download");
  CK(h, cudaStreamSynchronize(h->stream), "download sync");
  return DSMC_OK;
}

int dsmc_read_cell_sums(dsmc_handle* h, double* sums5, uint32_t* nsamples) {
  if (!h) return DSMC_ERR_ARG;
  return read_cell_major(h, 0, sums5, nsamples);
}

int dsmc_read_fields(dsmc_handle* h, double* fields5) {
  if (!h || !fields5) return DSMC_ERR_ARG;
  return read_cell_major(h, 1, fields5, nullptr);
}

int dsmc_get_totals(dsmc_handle* h, double totals[3]) {
  if (!h || !totals) return DSMC_ERR_ARG;
  Meta m{};
  int st = read_meta(h, m);
  if (st) return st;
  totals[0] = (double)m.selections;
  totals[1] = (double)m.collisions;
  totals[2] = m.sum_g;
  return DSMC_OK;
}

int dsmc_totals_async(dsmc_handle* h, void* out) {
  if (!h || !out) return DSMC_ERR_ARG;
  static_assert(offsetof(Meta, collisions) == offsetof(Meta, selections) + 8 &&
                    offsetof(Meta, sum_g) == offsetof(Meta, selections) + 16,
                "the running totals are 24 contiguous bytes of Meta");
  CK(h, cudaMemcpyAsync(out, &h->meta->selections, 24, cudaMemcpyDeviceToHost, h->stream),
     "totals copy");
  return DSMC_OK;
}

// ProcessAndOutputStatistics, kernels/dsmc_base.cu:104-163.
int dsmc_dump_statistics(dsmc_handle* h, const char* path) {
  if (!h || !path) return DSMC_ERR_ARG;
  double tot[3];
  int st = dsmc_get_totals(h, tot);
  if (st) return st;
  std::vector<double> f(5 * (size_t)h->cells), s(5 * (size_t)h->cells);
  uint32_t ns = 0;
  if ((st = dsmc_read_cell_sums(h, s.data(), &ns))) return st;
  if ((st = dsmc_read_fields(h, f.data()))) return st;
  FILE* out = std::fopen(path, "w");
  if (!out) return fail(h, DSMC_ERR_IO, std::string("cannot write ") + path);
  std::fprintf(out, "Selections: %g\nCollisions: %g\nMean separation: %g\nCollision ratio: %g\n",
               tot[0], tot[1], tot[1] > 0 ? tot[2] / tot[1] : 0.0, tot[0] > 0 ? tot[1] / tot[0] : 0.0);
  std::fprintf(out, "Simulation time: %g Running time: 0\n", h->sim_time);
  std::fprintf(out, "Cell N  ||  SampNum  ||  Dens  ||          Velocity          ||  Temperature\n");
  double tavg = 0, navg = 0;
  for (uint32_t c = 0; c < h->cells; c++) {
    const double* o = &f[5 * (size_t)c];
    tavg += o[4];
    navg += o[0];
    std::fprintf(out, "%u  ||  %u  ||  %g  ||  %g,%g,%g  ||  %g\n", c, (uint32_t)s[5 * (size_t)c], o[0],
                 o[1], o[2], o[3], o[4]);
  }
  tavg /= h->cells;
  navg /= h->cells;
  const dsmc_config& c = h->cfg;
  double gv = (double)(c.grid_max[0] - c.grid_min[0]) * (c.grid_max[1] - c.grid_min[1]) *
              (c.grid_max[2] - c.grid_min[2]);
  double n2d2 = (double)c.density * c.gas_diam * c.gas_diam * c.density;
  double tcoll = 2.0 * h->sim_time * n2d2 * gv * M_PI * std::pow(tavg / c.gas_tref, 0.25) *
                 std::sqrt(1.3806e-23 * c.gas_tref / (M_PI * c.gas_mass)) / c.fnum;
  std::fprintf(out, "\n\nExpected collisions: %g Ratio: %g\n", tcoll, tot[1] > 0 ? tcoll / tot[1] : 0.0);
  std::fprintf(out, "Average temperature: %g Reference temperature is: %g\nAverage density: %g Reference density: %g\n\n\n",
               tavg, c.temp, navg, c.density);
  std::fclose(out);
  return DSMC_OK;
}

// Snapshot: magic, version, config, counters, particles (SoA), per-cell state.
static const char kSnapMagic[8] = {'D', 'S', 'M', 'C', 'B', '2', '0', '0'};

int dsmc_snapshot(dsmc_handle* h, const char* path) {
  if (!h || !path) return DSMC_ERR_ARG;
  Meta m{};
  int st = read_meta(h, m);
  if (st) return st;
  uint32_t n = h->has_state ? m.n_alive + m.n_pending : 0;
  std::vector<float> part((size_t)n * 6);
  for (int k = 0; k < 6; k++)
    CK(h, cudaMemcpy(part.data() + (size_t)k * n, h->A[k], (size_t)n * 4, cudaMemcpyDeviceToHost), "snapshot");
  std::vector<float2> mr(h->cells);
  std::vector<uint4> sd(h->cells);
  std::vector<double> acc(5 * (size_t)h->cells);
  std::vector<float> rem(6);
  CK(h, cudaMemcpy(mr.data(), h->maxrem, h->cells * sizeof(float2), cudaMemcpyDeviceToHost), "snapshot");
  CK(h, cudaMemcpy(sd.data(), h->seeds, h->cells * sizeof(uint4), cudaMemcpyDeviceToHost), "snapshot");
  CK(h, cudaMemcpy(acc.data(), h->acc, acc.size() * 8, cudaMemcpyDeviceToHost), "snapshot");
  CK(h, cudaMemcpy(rem.data(), h->inj_rem, 6 * 4, cudaMemcpyDeviceToHost), "snapshot");
  std::ofstream f(path, std::ios::binary);
  if (!f) return fail(h, DSMC_ERR_IO, std::string("cannot write ") + path);
  uint32_t ver = 1;
  f.write(kSnapMagic, 8);
  f.write((const char*)&ver, 4);
  f.write((const char*)&h->cfg, sizeof(dsmc_config));
  f.write((const char*)&h->cells, 4);
  f.write((const char*)&n, 4);
  f.write((const char*)&h->step, 8);
  f.write((const char*)&h->sim_time, 8);
  f.write((const char*)&m, sizeof(Meta));
  f.write((const char*)part.data(), part.size() * 4);
  f.write((const char*)mr.data(), mr.size() * sizeof(float2));
  f.write((const char*)sd.data(), sd.size() * sizeof(uint4));
  f.write((const char*)acc.data(), acc.size() * 8);
  f.write((const char*)rem.data(), rem.size() * 4);
  if (!f) return fail(h, DSMC_ERR_IO, "snapshot write failed");
  return DSMC_OK;
}

int dsmc_restore(dsmc_handle* h, const char* path) {
  if (!h || !path) return DSMC_ERR_ARG;
  std::ifstream f(path, std::ios::binary);
  if (!f) return fail(h, DSMC_ERR_IO, std::string("cannot read ") + path);
  char mg[8];
  uint32_t ver = 0, cells = 0, n = 0;
  dsmc_config cfg;
  f.read(mg, 8);
  f.read((char*)&ver, 4);
  if (!f || std::memcmp(mg, kSnapMagic, 8) != 0 || ver != 1)
    return fail(h, DSMC_ERR_IO, "not a dsmc_b200 snapshot");
  f.read((char*)&cfg, sizeof(cfg));
  f.read((char*)&cells, 4);
  f.read((char*)&n, 4);
  if (cells != h->cells) return fail(h, DSMC_ERR_CONFIG, "snapshot cell count differs from the handle's");
  if (n > h->capacity) return fail(h, DSMC_ERR_CAPACITY, "snapshot particles exceed capacity");
  uint64_t step = 0;
  double t = 0;
  Meta m{};
  f.read((char*)&step, 8);
  f.read((char*)&t, 8);
  f.read((char*)&m, sizeof(Meta));
  std::vector<float> part((size_t)n * 6);
  std::vector<float2> mr(cells);
  std::vector<uint4> sd(cells);
  std::vector<double> acc(5 * (size_t)cells);
  std::vector<float> rem(6);
  f.read((char*)part.data(), part.size() * 4);
  f.read((char*)mr.data(), mr.size() * sizeof(float2));
  f.read((char*)sd.data(), sd.size() * sizeof(uint4));
  f.read((char*)acc.data(), acc.size() * 8);
  f.read((char*)rem.data(), rem.size() * 4);
  if (!f) return fail(h, DSMC_ERR_IO, "truncated snapshot");
  int st = dsmc_upload_state(h, part.data(), nullptr, n, 1);
  if (st) return st;
  CK(h, cudaMemcpy(h->maxrem, mr.data(), cells * sizeof(float2), cudaMemcpyHostToDevice), "restore");
  CK(h, cudaMemcpy(h->seeds, sd.data(), cells * sizeof(uint4), cudaMemcpyHostToDevice), "restore");
  CK(h, cudaMemcpy(h->acc, acc.data(), acc.size() * 8, cudaMemcpyHostToDevice), "restore");
  CK(h, cudaMemcpy(h->inj_rem, rem.data(), 6 * 4, cudaMemcpyHostToDevice), "restore");
  Meta cur{};
  CK(h, cudaMemcpy(&cur, h->meta, sizeof(Meta), cudaMemcpyDeviceToHost), "restore");
  cur.step = m.step;
  cur.selections = m.selections;
  cur.collisions = m.collisions;
  cur.sum_g = m.sum_g;
  cur.samples = m.samples;
  cur.injected = m.injected;
  cur.removed = m.removed;
  CK(h, cudaMemcpy(h->meta, &cur, sizeof(Meta), cudaMemcpyHostToDevice), "restore");
  h->step = step;
  h->sim_time = t;
  return DSMC_OK;
}

// ------------------------------------------------------------ stage API ----

static GridGeom grid_of(const dsmc_grid* g) {
  GridGeom r;
  r.gmin = make_float3(g->gmin[0], g->gmin[1], g->gmin[2]);
  r.gmax = make_float3(g->gmax[0], g->gmax[1], g->gmax[2]);
  r.cell = make_float3(g->cell[0], g->cell[1], g->cell[2]);
  r.dim = make_uint3(g->dim[0], g->dim[1], g->dim[2]);
  return r;
}

int dsmc_stage_cell_index(const dsmc_grid* g, const float* x, const float* y, const float* z,
                          uint32_t n, uint32_t* keys, uint32_t* idx, void* stream) {
  if (!g || (n && (!x || !y || !z || !keys))) return DSMC_ERR_ARG;
  cudaError_t e = dsmcb::launch_cell_ids(grid_of(g), x, y, z, n, keys, idx, (cudaStream_t)stream);
  return e ? DSMC_ERR_CUDA : DSMC_OK;
}

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

int dsmc_stage_sort_workspace(uint32_t n, uint32_t nkeys, size_t* bytes) {
  if (!bytes || nkeys == 0) return DSMC_ERR_ARG;
  uint32_t tiles = (nkeys + dsmcb::kScanTile - 1) / dsmcb::kScanTile;
  if (tiles > (uint32_t)dsmcb::kMaxScanTiles) return DSMC_ERR_ARG;
  *bytes = align256(4ull * (nkeys + 1)) * 2 + align256(4ull * tiles) + align256(4ull * n) * 3 +
           align256(sizeof(Meta));
  return DSMC_OK;
}

int dsmc_stage_sort(uint32_t* keys, uint32_t* vals, uint32_t n, uint32_t nkeys,
                    uint32_t* cell_start, void* workspace, size_t workspace_bytes, void* stream) {
  size_t need = 0;
  if (dsmc_stage_sort_workspace(n, nkeys, &need)) return DSMC_ERR_ARG;
  if (n && (!keys || !vals)) return DSMC_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  bool own = false;
  if (!workspace) {
    if (cudaMallocAsync(&workspace, need, s) != cudaSuccess) return DSMC_ERR_OOM;
    own = true;
  } else if (workspace_bytes < need) {
    return DSMC_ERR_ARG;
  }
  char* w = (char*)workspace;
  uint32_t tiles = (nkeys + dsmcb::kScanTile - 1) / dsmcb::kScanTile;
  uint32_t* count = (uint32_t*)w; w += align256(4ull * (nkeys + 1));
  uint32_t* start = (uint32_t*)w; w += align256(4ull * (nkeys + 1));
  uint32_t* tsum = (uint32_t*)w; w += align256(4ull * tiles);
  uint32_t* ticket = (uint32_t*)w; w += align256(4ull * n);
  uint32_t* tval = (uint32_t*)w; w += align256(4ull * n);
  uint32_t* tpos = (uint32_t*)w; w += align256(4ull * n);
  Meta* meta = (Meta*)w;
  cudaError_t e = cudaMemsetAsync(count, 0, 4ull * (nkeys + 1), s);
  if (!e) e = cudaMemsetAsync(tsum, 0, 4ull * tiles, s);
  if (!e) e = cudaMemsetAsync(meta, 0, sizeof(Meta), s);
  if (!e && n) e = dsmcb::launch_count_keys(keys, n, nkeys, ticket, count, tsum, tiles, s);
  if (!e) e = dsmcb::launch_scan(count, nullptr, start, nkeys, tsum, tiles, meta, 0, s);
  if (!e && n) e = dsmcb::launch_scatter_kv(keys, vals, ticket, start, n, nkeys, tval, tpos, s);
  if (!e && n) e = dsmcb::launch_segment_fixup(start, nkeys, tval, tpos, keys, vals, s);
  if (!e && cell_start) e = cudaMemcpyAsync(cell_start, start, 4ull * (nkeys + 1), cudaMemcpyDeviceToDevice, s);
  if (own) cudaFreeAsync(workspace, s);
  return e ? DSMC_ERR_CUDA : DSMC_OK;
}

int dsmc_stage_bounds_reorder(const uint32_t* sorted_keys, const uint32_t* sorted_idx, uint32_t n,
                              uint32_t ncells, uint32_t* cell_start_end, const float* const src[6],
                              float* const dst[6], void* stream) {
  if (n && (!sorted_keys || !cell_start_end)) return DSMC_ERR_ARG;
  if ((src || dst) && (!src || !dst || !sorted_idx)) return DSMC_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaMemsetAsync(cell_start_end, 0, 8ull * ncells, s);
  if (!e && n) e = dsmcb::launch_bounds_reorder(sorted_keys, sorted_idx, n, ncells, cell_start_end, src, dst, s);
  return e ? DSMC_ERR_CUDA : DSMC_OK;
}

int dsmc_stage_collide(const dsmc_collide_params* cp, float* u, float* v, float* w,
                       const uint32_t* cell_start, float* maxrem, uint32_t* seeds, float* stat4,
                       void* stream) {
  if (!cp || !u || !v || !w || !cell_start || !maxrem) return DSMC_ERR_ARG;
  if (cp->rng == DSMC_RNG_TAUS && !seeds) return DSMC_ERR_ARG;
  // the bulk copies of the kernel start on 16-byte boundaries of each array
  for (const void* a : {(const void*)u, (const void*)v, (const void*)w, (const void*)cell_start,
                        (const void*)maxrem, (const void*)seeds})
    if ((uintptr_t)a & 15u) return DSMC_ERR_ARG;
  dsmcb::StepParams p{};
  p.cells = cp->ncells;
  p.cell_volume = cp->cell_volume;
  p.cross_section = cp->cross_section;
  p.fnum = cp->fnum;
  p.avg_conc = cp->avg_conc;
  p.dt = cp->dt;
  p.ntc_coef = (float)(0.5 * (double)cp->fnum * cp->dt / (double)cp->cell_volume);
  p.hard_sphere = std::fabs(cp->omega - 0.5f) < 1e-9f;
  p.vhs_exp = 2.f * cp->omega - 1.f;
  p.vhs_gref = cp->vhs_gref;
  set_vhs_fast(p, cp->cross_section, cp->omega, cp->vhs_gref);
  p.ntc_local = cp->ntc_local;
  p.rng_kind = cp->rng;
  p.seed = make_uint2((uint32_t)cp->seed, (uint32_t)(cp->seed >> 32));
  p.in = SoA{u, v, w, u, v, w};
  p.out = p.in;
  p.start = cell_start;
  p.maxrem = (float2*)maxrem;
  p.seeds = (uint4*)seeds;
  p.stat4 = (float4*)stat4;
  p.meta = nullptr;
  p.flags = dsmcb::kDoCollide | dsmcb::kVelOnly;
  p.cells_per_tile = 256;
  p.n_tiles = (cp->ncells + 255) / 256;
  p.step_override = cp->step ? cp->step : 1u;
  p.cell_variant = 0;
  cudaError_t e = dsmcb::launch_cell(p, (cudaStream_t)stream);
  return e ? DSMC_ERR_CUDA : DSMC_OK;
}

int dsmc_stage_move(dsmc_handle* h, const dsmc_move_params* mp, float* x, float* y, float* z,
                    float* u, float* v, float* w, uint32_t n, void* stream) {
  if (!mp || (n && (!x || !y || !z || !u || !v || !w))) return DSMC_ERR_ARG;
  dsmcb::StepParams p{};
  if (h) p = base_params(h, mp->dt);
  p.grid = grid_of(&mp->grid);
  p.dt = mp->dt;
  p.periodic = mp->periodic;
  p.face_mode = mp->face_mode;
  for (int i = 0; i < 6; i++) {
    p.face_kind[i] = mp->face_kind[i];
    p.face_vstd[i] = mp->face_vstd[i];
  }
  p.seed = make_uint2((uint32_t)mp->seed, (uint32_t)(mp->seed >> 32));
  if (!h) p.has_geom = 0;
  p.out = SoA{x, y, z, u, v, w};
  cudaError_t e = dsmcb::launch_move(p, n, mp->step ? mp->step : 1u, (cudaStream_t)stream);
  return e ? DSMC_ERR_CUDA : DSMC_OK;
}

int dsmc_clearance_at(dsmc_handle* h, const float* xyz, uint32_t n, float* out, void* stream) {
  if (!h || (n && (!xyz || !out))) return DSMC_ERR_ARG;
  if (!h->has_geom) return fail(h, DSMC_ERR_STATE, "no geometry");
  dsmcb::StepParams p = base_params(h, h->cfg.dt);
  cudaError_t e = dsmcb::launch_clearance_at(p.geom, xyz, n, out, (cudaStream_t)stream);
  return e ? cuda_fail(h, e, "clearance lookup") : DSMC_OK;
}

int dsmc_stage_sample(const float* u, const float* v, const float* w, const uint32_t* cell_start,
                      uint32_t ncells, double* sums5, void* stream) {
  if (!u || !v || !w || !cell_start || !sums5) return DSMC_ERR_ARG;
  cudaError_t e = dsmcb::launch_sample_cells(u, v, w, cell_start, ncells, sums5, 1, 5,
                                             (cudaStream_t)stream);
  return e ? DSMC_ERR_CUDA : DSMC_OK;
}

// ------------------------------------------------------------- batches ----

// Several handles advanced by one CUDA graph per timestep: a fork from the
// batch stream to one stream per member, each member's step on its branch,
// and a join back (no counterpart in the reference, which has one solver per
// process).
struct dsmc_batch {
  std::vector<dsmc_handle*> members;
  std::vector<float> dt;
  std::vector<uint64_t> gen;
  cudaStream_t stream = nullptr;
  bool own_stream = true;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // the batched launches' device tables (written before each capture): the
  // members' parameters, their sort arrays, the inflow faces, and per stage
  // the members' first blocks
  dsmcb::StepParams* d_params = nullptr;
  dsmcb::SortArgs* d_sort = nullptr;
  dsmcb::InjectParams* d_inj = nullptr;
  uint32_t* d_block0 = nullptr;
  size_t cap_members = 0, cap_inj = 0;
  std::string err;
};

namespace {

int batch_fail(dsmc_batch* b, int code, const std::string& msg) {
  b->err = msg;
  return code;
}

void batch_drop_graph(dsmc_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
}

void batch_free(dsmc_batch* b) {
  batch_drop_graph(b);
  cudaFree(b->d_params);
  cudaFree(b->d_sort);
  cudaFree(b->d_inj);
  cudaFree(b->d_block0);
  if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

bool batch_graph_current(const dsmc_batch* b, const std::vector<float>& dt) {
  if (!b->exec || dt != b->dt) return false;
  for (size_t i = 0; i < b->members.size(); i++)
    if (b->members[i]->gen != b->gen[i]) return false;
  return true;
}

// Block offsets of a stage: member i gets blocks[i] (at least 1) blocks.
void offsets(const std::vector<uint32_t>& blocks, std::vector<uint32_t>& out) {
  out.push_back(0);
  for (uint32_t k : blocks) out.push_back(out.back() + std::max(k, 1u));
}

// Shares of `wave` blocks by weight, at least one block each.
std::vector<uint32_t> shares(const std::vector<double>& w, uint32_t wave) {
  double total = 0.0;
  for (double x : w) total += x;
  std::vector<uint32_t> out(w.size(), 1u);
  for (size_t i = 0; i < w.size(); i++)
    if (total > 0.0) out[i] = std::max(1u, (uint32_t)std::lround((double)wave * w[i] / total));
  return out;
}

// The batch's step: each stage of the split step launched once for all
// members, member i running its own parameters in a share of the grid
// (dsmcb::BatchOf), in the stage order of a member stepped alone (scan,
// scatter, order, inflow injection, NTC, flight, mesh, sampling).  Shares
// follow the members' particle counts at capture time (cells for the scan and
// the sampling), so that every stage fills the GPU once with the whole
// ensemble's work instead of once per member.
int batch_capture(dsmc_batch* b, const std::vector<float>& dt) {
  batch_drop_graph(b);
  const size_t n = b->members.size();
  cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e) return batch_fail(b, DSMC_ERR_CUDA, std::string("batch sync: ") + cudaGetErrorString(e));
  std::vector<dsmcb::StepParams> P(n);
  std::vector<dsmcb::SortArgs> A(n);
  std::vector<dsmcb::InjectParams> I;
  std::vector<double> np(n), nc(n);
  uint32_t max_tiles = 0;
  for (size_t i = 0; i < n; i++) {
    dsmc_handle* h = b->members[i];
    if (h->mt_on) return batch_fail(b, DSMC_ERR_STATE, "the -mt collisions cannot run in a batch");
    Meta m{};
    const int st = read_meta(h, m);
    if (st) return batch_fail(b, st, h->err);
    np[i] = (double)m.n_alive + (double)m.n_pending + 1.0;
    nc[i] = (double)h->cells;
    // every member runs the split kernels with the order kernel's
    // (128 particles, 4 warps, 5 CTAs) shape and tiles of 32 cells, whatever
    // shape it uses stepped alone
    P[i] = step_params(h, dt[i], true);
    P[i].cell_variant = 5;
    P[i].cells_per_tile = (int)dsmcb::cell_kernel_w_tile();
    P[i].n_tiles = (h->cells + dsmcb::cell_kernel_w_tile() - 1) / dsmcb::cell_kernel_w_tile();
    A[i] = dsmcb::SortArgs{h->count, h->cursor, h->start, h->tile_sum, h->orig, h->keys,
                           h->meta, h->cells, h->n_scan_tiles, h->capacity};
    for (const auto& in : h->inflows) I.push_back(inject_params(h, in, dt[i], P[i].seed));
    max_tiles = std::max(max_tiles, h->n_scan_tiles);
  }
  const size_t flight_smem = (size_t)max_tiles * 4u;
  uint32_t wave[5];
  e = dsmcb::cell_batch_waves(wave, flight_smem);
  if (e) return batch_fail(b, DSMC_ERR_CUDA, std::string("batch shapes: ") + cudaGetErrorString(e));
  // per stage: scan, scatter, order, NTC, flight, mesh, sampling; then the
  // inflow plan (one block per face) and fill
  std::vector<std::vector<uint32_t>> blocks(9);
  for (size_t i = 0; i < n; i++) blocks[0].push_back(b->members[i]->n_scan_tiles);
  // the order kernel's and the NTC kernel's work per tile of 32 cells has a
  // floor (a tile's chunk costs about as much with few particles as with
  // eight per cell): weigh their shares by cells as well as particles
  std::vector<double> wcell(n);
  for (size_t i = 0; i < n; i++) wcell[i] = np[i] + 8.0 * nc[i];
  blocks[1] = shares(np, (uint32_t)dsmcb::num_sms() * 4u);
  blocks[2] = shares(wcell, wave[0]);
  for (size_t i = 0; i < n; i++)  // the order kernel needs no more warps than tiles
    blocks[2][i] = std::min(blocks[2][i], std::max(1u, (P[i].n_tiles + 3u) / 4u));
  blocks[3] = shares(wcell, wave[1]);
  blocks[4] = shares(np, wave[2]);
  blocks[5] = shares(np, wave[3]);
  blocks[6] = shares(nc, wave[4]);
  blocks[7].assign(I.size(), 1u);
  blocks[8].assign(I.size(), 4u);
  std::vector<uint32_t> off;
  std::vector<size_t> at(9);
  std::vector<uint32_t> total(9);
  for (int k = 0; k < 9; k++) {
    at[k] = off.size();
    offsets(blocks[k], off);
    total[k] = off.back();
  }
  // device tables (grown as needed)
  if (n > b->cap_members) {
    cudaFree(b->d_params);
    cudaFree(b->d_sort);
    b->d_params = nullptr;
    b->d_sort = nullptr;
    b->cap_members = 0;
    e = cudaMalloc(&b->d_params, n * sizeof(dsmcb::StepParams));
    if (!e) e = cudaMalloc(&b->d_sort, n * sizeof(dsmcb::SortArgs));
    if (e) return batch_fail(b, DSMC_ERR_OOM, "batch tables");
    b->cap_members = n;
  }
  if (I.size() > b->cap_inj) {
    cudaFree(b->d_inj);
    b->d_inj = nullptr;
    b->cap_inj = 0;
    e = cudaMalloc(&b->d_inj, I.size() * sizeof(dsmcb::InjectParams));
    if (e) return batch_fail(b, DSMC_ERR_OOM, "batch tables");
    b->cap_inj = I.size();
  }
  cudaFree(b->d_block0);
  b->d_block0 = nullptr;
  e = cudaMalloc(&b->d_block0, off.size() * sizeof(uint32_t));
  if (!e) e = cudaMemcpy(b->d_params, P.data(), n * sizeof(dsmcb::StepParams), cudaMemcpyHostToDevice);
  if (!e) e = cudaMemcpy(b->d_sort, A.data(), n * sizeof(dsmcb::SortArgs), cudaMemcpyHostToDevice);
  if (!e && !I.empty())
    e = cudaMemcpy(b->d_inj, I.data(), I.size() * sizeof(dsmcb::InjectParams), cudaMemcpyHostToDevice);
  if (!e) e = cudaMemcpy(b->d_block0, off.data(), off.size() * sizeof(uint32_t), cudaMemcpyHostToDevice);
  if (e) return batch_fail(b, DSMC_ERR_CUDA, std::string("batch tables: ") + cudaGetErrorString(e));
  const uint32_t nm = (uint32_t)n, ni = (uint32_t)I.size();
  auto sv = [&](int k) { return dsmcb::BatchOf<dsmcb::SortArgs>{b->d_sort, b->d_block0 + at[k], nm}; };
  auto pv = [&](int k) { return dsmcb::BatchOf<dsmcb::StepParams>{b->d_params, b->d_block0 + at[k], nm}; };
  auto iv = [&](int k) { return dsmcb::BatchOf<dsmcb::InjectParams>{b->d_inj, b->d_block0 + at[k], ni}; };
  e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
  if (!e) e = dsmcb::launch_scan_b(sv(0), total[0], b->stream);
  if (!e) e = dsmcb::launch_scatter_b(sv(1), total[1], b->stream);
  bool coop_mesh = true;
  for (size_t i = 0; i < n; i++)
    if (P[i].has_geom && !P[i].geom.nearest) coop_mesh = false;
  if (!e) e = dsmcb::launch_cell_stage_b(0, pv(2), total[2], flight_smem, coop_mesh, b->stream);
  if (!e && ni) e = dsmcb::launch_inject_b(iv(7), total[7], iv(8), total[8], flight_smem, b->stream);
  for (int st = 1; st < 5 && !e; st++)
    e = dsmcb::launch_cell_stage_b(st, pv(2 + st), total[2 + st], flight_smem, coop_mesh, b->stream);
  cudaError_t e2 = cudaStreamEndCapture(b->stream, &b->graph);
  if (e || e2) {
    batch_drop_graph(b);
    return batch_fail(b, DSMC_ERR_CUDA,
                      std::string("batch graph capture: ") + cudaGetErrorString(e ? e : e2));
  }
  e = cudaGraphInstantiate(&b->exec, b->graph, 0);
  if (e) {
    batch_drop_graph(b);
    return batch_fail(b, DSMC_ERR_CUDA, std::string("batch graph instantiate: ") + cudaGetErrorString(e));
  }
  b->dt = dt;
  for (size_t i = 0; i < n; i++) b->gen[i] = b->members[i]->gen;
  return DSMC_OK;
}

}  // namespace

int dsmc_batch_create(dsmc_handle* const* members, uint32_t n, dsmc_batch** out) {
  if (!members || !n || !out) return DSMC_ERR_ARG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return DSMC_ERR_CUDA;
  dsmc_batch* b = new dsmc_batch();
  for (uint32_t i = 0; i < n; i++) {
    if (!members[i] || members[i]->device != dev) {
      delete b;
      g_create_error = "batch members must be handles created on the current device";
      return DSMC_ERR_ARG;
    }
    for (uint32_t j = 0; j < i; j++)
      if (members[j] == members[i]) {
        delete b;
        g_create_error = "a handle appears twice in the batch";
        return DSMC_ERR_ARG;
      }
    b->members.push_back(members[i]);
  }
  b->gen.assign(n, 0);
  const cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e) {
    g_create_error = std::string("batch streams: ") + cudaGetErrorString(e);
    batch_free(b);
    return DSMC_ERR_CUDA;
  }
  *out = b;
  return DSMC_OK;
}

int dsmc_batch_destroy(dsmc_batch* b) {
  if (!b) return DSMC_ERR_ARG;
  if (b->stream) cudaStreamSynchronize(b->stream);
  batch_free(b);
  return DSMC_OK;
}

const char* dsmc_batch_last_error(const dsmc_batch* b) { return b ? b->err.c_str() : ""; }

int dsmc_batch_set_stream(dsmc_batch* b, void* stream) {
  if (!b) return DSMC_ERR_ARG;
  if (b->own_stream && b->stream) {
    cudaStreamSynchronize(b->stream);
    cudaStreamDestroy(b->stream);
  }
  if (stream) {
    b->stream = (cudaStream_t)stream;
    b->own_stream = false;
  } else {
    b->own_stream = true;
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
      return batch_fail(b, DSMC_ERR_CUDA, "batch stream");
  }
  batch_drop_graph(b);
  return DSMC_OK;
}

int dsmc_batch_step(dsmc_batch* b, const float* dt, int nsteps) {
  if (!b || nsteps < 0) return DSMC_ERR_ARG;
  const size_t n = b->members.size();
  std::vector<float> d(n);
  for (size_t i = 0; i < n; i++) {
    dsmc_handle* h = b->members[i];
    if (!h->has_state) return batch_fail(b, DSMC_ERR_STATE, "a member has no particle state");
    d[i] = dt ? dt[i] : h->cfg.dt;
  }
  if (!batch_graph_current(b, d)) {
    const int st = batch_capture(b, d);
    if (st) return st;
  }
  for (int k = 0; k < nsteps; k++) {
    const cudaError_t e = cudaGraphLaunch(b->exec, b->stream);
    if (e) return batch_fail(b, DSMC_ERR_CUDA, std::string("batch graph launch: ") + cudaGetErrorString(e));
    for (size_t i = 0; i < n; i++) {
      b->members[i]->step++;
      b->members[i]->sim_time += d[i];
    }
  }
  return DSMC_OK;
}

int dsmc_batch_sync(dsmc_batch* b) {
  if (!b) return DSMC_ERR_ARG;
  const cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e) return batch_fail(b, DSMC_ERR_CUDA, std::string("batch sync: ") + cudaGetErrorString(e));
  for (dsmc_handle* h : b->members) {
    const int st = check_device_flags(h);
    if (st) return batch_fail(b, st, h->err);
  }
  return DSMC_OK;
}

int dsmc_batch_autotune(dsmc_batch* b, const float* dt, int steps, int* variants) {
  if (!b || steps < 1) return DSMC_ERR_ARG;
  int st = dsmc_batch_sync(b);
  if (st) return st;
  for (size_t i = 0; i < b->members.size(); i++) {
    dsmc_handle* h = b->members[i];
    int best = 0;
    st = dsmc_autotune(h, dt ? dt[i] : h->cfg.dt, steps, &best, nullptr);
    if (st) return batch_fail(b, st, h->err);
    if (variants) variants[i] = best;
  }
  return DSMC_OK;
}

}  // extern "C"
