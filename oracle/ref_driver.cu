// Headless driver for the reference's own GPU kernels.
//
// TEST INFRASTRUCTURE ONLY.  This translation unit compiles the reference's
// kernels/dsmc_kernel.cu unchanged (it is #included from the reference tree by
// oracle/Makefile) and exposes its stage wrappers through a plain C ABI so the
// tests can drive them stage by stage on the same inputs as the product
// library.  Nothing in the product links or loads this file's output.
//
// What the driver replaces in the reference and why:
//  * include/gpu_dsmc.inl drives the stages but pulls in OpenGL interop, so the
//    stage order of RunBenchmarkSimulationStep (include/gpu_dsmc.inl:220-274)
//    is re-issued here (ref_step).
//  * InitBirdData (kernels/dsmc_kernel.cu:1122-1155) seeds the per-cell
//    HybridTaus states from /dev/urandom and runs InitMaximums on the
//    Mersenne-Twister state, which only holds 65536 entries.  The driver
//    allocates the same per-cell buffers itself and lets the caller upload
//    seeds and (sigma*g)max / remainder, so runs are reproducible and any cell
//    count works.
//  * Model::CreateGrid (src/model.cpp:733-769) needs the GL-linked Model class;
//    ref_build_grid re-issues its binning loop over the reference's own
//    reg_grid_t (src/reggrid.cpp) and AABB_t::tri_overlaps (src/aabb.cpp,
//    include/tritest.h).
#include "dsmc_kernel.cu"

#include <cstring>
#include <vector>

// Draws from the reference's HybridTausRngInt / HybridTausRng
// (kernels/mtwister.cu:135-153): state i produces `draws` integers, then
// `draws` floats.
__global__ void RefTausDrawsDev(uint4* states, uint n, uint draws, uint* ints, float* floats) {
  uint i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint4 s = states[i];
  for (uint k = 0; k < draws; k++) ints[i * draws + k] = HybridTausRngInt(&s);
  for (uint k = 0; k < draws; k++) floats[i * draws + k] = HybridTausRng(&s);
  states[i] = s;
}

extern "C" {

int ref_taus_draws(unsigned* states_dev, unsigned n, unsigned draws, unsigned* ints_dev,
                   float* floats_dev) {
  RefTausDrawsDev<<<(n + 127) / 128, 128>>>((uint4*)states_dev, n, draws, ints_dev, floats_dev);
  cudaError_t e = cudaDeviceSynchronize();
  return e == cudaSuccess ? 0 : (int)e;
}

struct ref_config {
  float gmin[3];
  float gmax[3];
  int dim[3];
  float density, fnum, temp;
  float mass, diam, tref;
  char periodic;
};

static settings_t g_ref_settings;
static uint* g_ref_geom_hashes = 0;
static bool g_ref_has_geom = false;

static int ref_status(void) {
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaGetLastError();
  return e == cudaSuccess ? 0 : (int)e;
}

// settings_t as kernels/dsmc.cu:322-330 and src/sim_settings.cpp:74-103 fill it.
int ref_init(const ref_config* c) {
  settings_t s;
  s.benchmark = true;
  s.boundaries.reset(vec3_t(c->gmin[0], c->gmin[1], c->gmin[2]),
                     vec3_t(c->gmax[0], c->gmax[1], c->gmax[2]));
  s.grid_dim = vec3i_t(c->dim[0], c->dim[1], c->dim[2]);
  s.cell_size.reset(s.boundaries.get_xsize() / s.grid_dim.x,
                    s.boundaries.get_ysize() / s.grid_dim.y,
                    s.boundaries.get_zsize() / s.grid_dim.z);
  s.density = c->density;
  s.fnum = c->fnum;
  s.temp = c->temp;
  s.gas.molmass = c->mass;
  s.gas.diameter = c->diam;
  s.gas.Tref = c->tref;
  s.periodicCondition = c->periodic;
  float cell_volume = s.cell_size.x * s.cell_size.y * s.cell_size.z;
  uint ppc = s.density * cell_volume / s.fnum;
  s.partPerCell = ppc;
  s.numParticles = ppc * s.getCellsCount();
  g_ref_settings = s;

  InitSimulationProperties(s);

  const uint cells = s.getCellsCount();
  if (maximums) cudaFree(maximums);
  if (devStatistics) cudaFree(devStatistics);
  if (devCellStatistics) cudaFree(devCellStatistics);
  if (devSeeds) cudaFree(devSeeds);
  cudaMalloc(&maximums, cells * sizeof(float2));
  cudaMalloc(&devStatistics, cells * sizeof(float4));
  cudaMalloc(&devCellStatistics, cells * sizeof(dsmc::statistics_t));
  cudaMalloc(&devSeeds, cells * sizeof(uint4));
  cudaMemset(maximums, 0, cells * sizeof(float2));
  cudaMemset(devStatistics, 0, cells * sizeof(float4));
  cudaMemset(devCellStatistics, 0, cells * sizeof(dsmc::statistics_t));
  cudaMemset(devSeeds, 0, cells * sizeof(uint4));
  return ref_status();
}

// Host-side values the reference derives in InitSimulationProperties.
int ref_derived(unsigned* part_per_cell, float* cell_volume, float* cross_section,
                float* max_rel_vel, float cell_size[3]) {
  const settings_t& s = g_ref_settings;
  *part_per_cell = s.partPerCell;
  *cell_volume = s.cell_size.x * s.cell_size.y * s.cell_size.z;
  double cs = DSMC_PI * s.gas.diameter * s.gas.diameter;
  *cross_section = (float)cs;
  double rv = s.gas.diameter * s.gas.diameter * DSMC_PI * sqrtf(s.temp / 300.0) * 300;
  *max_rel_vel = (float)rv;
  cell_size[0] = s.cell_size.x;
  cell_size[1] = s.cell_size.y;
  cell_size[2] = s.cell_size.z;
  return 0;
}

// settings_t::readFromFile (src/sim_settings.cpp:46-132) on `path`, with the
// gas file opened relative to the working directory as the reference does.
// f: grid min (3), max (3), density, fnum, temp, stream velocity (3), gas
// mass, diameter, T_ref, cell size (3); i: grid dims (3), periodic character.
// Host code only: no device work.
static void ref_settings_out(const settings_t& s, float* f, int* i) {
  const float v[18] = {s.boundaries.min.x, s.boundaries.min.y, s.boundaries.min.z,
                       s.boundaries.max.x, s.boundaries.max.y, s.boundaries.max.z,
                       s.density, s.fnum, s.temp,
                       s.streamVelocity.x, s.streamVelocity.y, s.streamVelocity.z,
                       s.gas.molmass, s.gas.diameter, s.gas.Tref,
                       s.cell_size.x, s.cell_size.y, s.cell_size.z};
  std::memcpy(f, v, sizeof(v));
  i[0] = s.grid_dim.x;
  i[1] = s.grid_dim.y;
  i[2] = s.grid_dim.z;
  i[3] = s.periodicCondition;
}

int ref_read_settings(const char* path, float f[18], int i[4]) {
  settings_t s;
  s.readFromFile(path);
  ref_settings_out(s, f, i);
  return 0;
}

// settings_t() then settings_t::readFromCmdLine (src/sim_settings.cpp:34-44,
// 134-186) on argv.  f: the 18 values of ref_read_settings, then dt and the
// run time; i: grid dims, periodic character, then benchmark, geometry, mt,
// cpu.  Host code only.
int ref_read_cmdline(int argc, char** argv, float f[20], int i[8]) {
  settings_t s;
  s.readFromCmdLine(argc, argv);
  ref_settings_out(s, f, i);
  f[18] = s.dt;
  f[19] = s.maxRunTime;
  i[4] = s.benchmark;
  i[5] = s.geometry;
  i[6] = s.mt;
  i[7] = s.cpu;
  return 0;
}

// The -mt twisters as GPUDSMCSolver::Init sets them up
// (include/gpu_dsmc.inl:346-368): InitGPUTwisters on the parameter file at
// `path` with `seed` (kernels/mtwister.cu:46-68), then InitMersenneTwisters
// (kernels/dsmc_kernel.cu:548-569).
int ref_mt_init(const char* path, unsigned seed) {
  InitGPUTwisters(path, seed);
  InitMersenneTwisters();
  return ref_status();
}

// The first `count` twisters: parameters (matrix_a, mask_b, mask_c, seed)
// and states (iState, mti1, mt[19]), either pointer may be null.
int ref_mt_get(unsigned count, unsigned* cfg4, unsigned* state21) {
  if (count > MT_RNG_COUNT) return -1;
  if (cfg4) cudaMemcpyFromSymbol(cfg4, ds_MT, count * sizeof(mt_struct_stripped));
  if (state21) cudaMemcpyFromSymbol(state21, ds_mtState, count * sizeof(mt_state));
  return ref_status();
}

// ComputeBird with mt = true: ComputeBirdCollisionsDev
// (kernels/dsmc_kernel.cu:1002-1089), cell c drawing from twister c.
int ref_collide_mt(float4* vel, const uint2* cse, uint avg_conc, float dt) {
  ComputeBird(vel, cse, 0, avg_conc, dt, true);
  return ref_status();
}

int ref_set_cell_state(const float* maxrem, const unsigned* seeds) {
  const uint cells = g_ref_settings.getCellsCount();
  if (maxrem) cudaMemcpy(maximums, maxrem, cells * sizeof(float2), cudaMemcpyHostToDevice);
  if (seeds) cudaMemcpy(devSeeds, seeds, cells * sizeof(uint4), cudaMemcpyHostToDevice);
  return ref_status();
}

int ref_get_cell_state(float* maxrem, unsigned* seeds, float* coll_stats, float* cell_stats) {
  const uint cells = g_ref_settings.getCellsCount();
  if (maxrem) cudaMemcpy(maxrem, maximums, cells * sizeof(float2), cudaMemcpyDeviceToHost);
  if (seeds) cudaMemcpy(seeds, devSeeds, cells * sizeof(uint4), cudaMemcpyDeviceToHost);
  if (coll_stats) cudaMemcpy(coll_stats, devStatistics, cells * sizeof(float4), cudaMemcpyDeviceToHost);
  if (cell_stats)
    cudaMemcpy(cell_stats, devCellStatistics, cells * sizeof(dsmc::statistics_t),
               cudaMemcpyDeviceToHost);
  return ref_status();
}

int ref_clear_stats(void) {
  const uint cells = g_ref_settings.getCellsCount();
  cudaMemset(devStatistics, 0, cells * sizeof(float4));
  cudaMemset(devCellStatistics, 0, cells * sizeof(dsmc::statistics_t));
  return ref_status();
}

// Re-issues the binning loop of Model::CreateGrid (src/model.cpp:733-769) over
// the reference's reg_grid_t and AABB_t.  Outputs: per geometry cell the
// triangle count, the flattened triangle ids (in bin order), and the
// "has geometry" flag after encloseGrid.  Returns the number of bin entries.
long ref_build_grid(const float* verts, unsigned nverts, const unsigned* tris, unsigned ntris,
                    const int dim[3], float out_bbox[6], float out_cell[3], unsigned* out_count,
                    unsigned* out_tri_ids, long cap, unsigned char* out_flag) {
  std::vector<vec3_t> v(nverts);
  for (unsigned i = 0; i < nverts; i++) v[i] = vec3_t(verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]);
  bbox_t bb;
  bb.min.reset(100000, 100000, 100000);
  bb.max.reset(-100000, -100000, -100000);
  for (unsigned i = 0; i < nverts; i++) {  // Model::surface_t::CalcBBox, src/model.cpp:150-174
    if (v[i].x < bb.min.x) bb.min.x = v[i].x;
    if (v[i].y < bb.min.y) bb.min.y = v[i].y;
    if (v[i].z < bb.min.z) bb.min.z = v[i].z;
    if (v[i].x > bb.max.x) bb.max.x = v[i].x;
    if (v[i].y > bb.max.y) bb.max.y = v[i].y;
    if (v[i].z > bb.max.z) bb.max.z = v[i].z;
  }
  reg_grid_t grid;
  grid.reset(bb, vec3i_t(dim[0], dim[1], dim[2]));
  std::vector<std::vector<unsigned> > bins(grid.cellCount());
  vec3i_t gi;
  for (gi.x = 0; gi.x < grid.dim.x; gi.x++)
    for (gi.y = 0; gi.y < grid.dim.y; gi.y++)
      for (gi.z = 0; gi.z < grid.dim.z; gi.z++) {
        AABB_t aabb = grid.getAABB(gi);
        uint idx = grid.getCellIdx(gi);
        for (uint t = 0; t < ntris; t++) {
          if (aabb.tri_overlaps(v[tris[3 * t]], v[tris[3 * t + 1]], v[tris[3 * t + 2]])) {
            bins[idx].push_back(t);
            grid[idx].second = true;
          }
        }
      }
  grid.encloseGrid();
  long total = 0;
  for (uint c = 0; c < grid.cellCount(); c++) {
    out_count[c] = (unsigned)bins[c].size();
    out_flag[c] = grid[c].second ? 1 : 0;
    for (size_t k = 0; k < bins[c].size(); k++) {
      if (total < cap) out_tri_ids[total] = bins[c][k];
      total++;
    }
  }
  out_bbox[0] = grid.gridSize.min.x; out_bbox[1] = grid.gridSize.min.y; out_bbox[2] = grid.gridSize.min.z;
  out_bbox[3] = grid.gridSize.max.x; out_bbox[4] = grid.gridSize.max.y; out_bbox[5] = grid.gridSize.max.z;
  out_cell[0] = grid.cellSize.x; out_cell[1] = grid.cellSize.y; out_cell[2] = grid.cellSize.z;
  return total;
}

// The reference's tri/box test on one triangle (for oracle pinning).
int ref_tri_box_overlap(const float center[3], const float half[3], const float tri[9]) {
  AABB_t a(vec3_t(center[0], center[1], center[2]), vec3_t(half[0], half[1], half[2]));
  return a.tri_overlaps(vec3_t(tri[0], tri[1], tri[2]), vec3_t(tri[3], tri[4], tri[5]),
                        vec3_t(tri[6], tri[7], tri[8])) ? 1 : 0;
}

// Uploads a geometry grid the way SetModel -> InitRegularGrid does
// (kernels/dsmc_base.cu:49-55, kernels/dsmc_kernel.cu:350-376).  The grid is
// given as bbox, cell size, dims, per-cell triangle lists (CSR over triangle
// ids into tris), per-cell flags, and per-triangle face normals.
int ref_set_geometry(const float bbox[6], const float cell[3], const int dim[3],
                     const unsigned* cell_count, const unsigned* tri_ids,
                     const unsigned char* flags, const float* verts, unsigned nverts,
                     const unsigned* tris, const float* face_normals) {
  reg_grid_t grid;
  grid.gridSize.min.reset(bbox[0], bbox[1], bbox[2]);
  grid.gridSize.max.reset(bbox[3], bbox[4], bbox[5]);
  grid.cellSize.reset(cell[0], cell[1], cell[2]);
  grid.dim = vec3i_t(dim[0], dim[1], dim[2]);
  grid.nodes.resize(grid.cellCount());
  grid.normals.resize(grid.cellCount());
  size_t off = 0;
  for (uint c = 0; c < grid.cellCount(); c++) {
    grid.nodes[c].second = flags[c] != 0;
    for (uint k = 0; k < cell_count[c]; k++) {
      unsigned t = tri_ids[off + k];
      grid.nodes[c].first.push_back(tris[3 * t]);
      grid.nodes[c].first.push_back(tris[3 * t + 1]);
      grid.nodes[c].first.push_back(tris[3 * t + 2]);
      grid.normals[c].push_back(vec3_t(face_normals[3 * t], face_normals[3 * t + 1], face_normals[3 * t + 2]));
    }
    off += cell_count[c];
  }
  if (g_ref_has_geom) {
    DeinitRegularGrid();
    if (g_ref_geom_hashes) cudaFree(g_ref_geom_hashes);
  }
  g_ref_geom_hashes = InitRegularGrid(grid, verts, nverts);
  g_ref_has_geom = true;
  return ref_status();
}

// ---- stage wrappers (device pointers, float4 AoS as in include/particles.h) ----

int ref_cell_ids(float4* pos, uint* hashes, uint* idx, uint n) {
  CalculateCellIDs(pos, hashes, idx, n);
  return ref_status();
}

int ref_sort(uint* hashes, uint* idx, uint n) {
  SortParticlesIndices(hashes, idx, n);
  return ref_status();
}

int ref_bounds(uint2* cse, float4* sorted_pos, float4* sorted_vel, uint* hashes, uint* idx,
               float4* old_pos, float4* old_vel, uint n) {
  cudaMemset(cse, 0, g_ref_settings.getCellsCount() * sizeof(uint2));
  FindCellBoundaries(cse, sorted_pos, sorted_vel, 0, hashes, idx, old_pos, old_vel, 0, n, false);
  return ref_status();
}

int ref_collide(float4* vel, const uint2* cse, uint avg_conc, float dt) {
  ComputeBird(vel, cse, 0, avg_conc, dt, false);
  return ref_status();
}

int ref_move(float4* pos, float4* vel, float dt, uint n, int geometry, char bc) {
  if (geometry)
    IntegrateAndProcessCollisions(pos, vel, 0, dt, g_ref_geom_hashes, n, false, bc);
  else
    Integrate(pos, vel, 0, dt, n, false, bc);
  return ref_status();
}

int ref_sample(const float4* vel, const uint2* cse) {
  SampleCellStatistics(vel, cse, 0, false);
  return ref_status();
}

int ref_get_statistics(float out[4]) {
  float4 s = GetStatistics();
  out[0] = s.x; out[1] = s.y; out[2] = s.z; out[3] = s.w;
  return ref_status();
}

// One RunBenchmarkSimulationStep (include/gpu_dsmc.inl:220-274): the caller
// passes the ping-pong buffers already swapped (old_* hold the state to sort).
int ref_step(float4* pos, float4* old_pos, float4* vel, float4* old_vel, uint* hashes,
             uint* idx, uint2* cse, uint n, float dt, int collide, int geometry, int sample) {
  CalculateCellIDs(old_pos, hashes, idx, n);
  SortParticlesIndices(hashes, idx, n);
  cudaMemset(cse, 0, g_ref_settings.getCellsCount() * sizeof(uint2));
  FindCellBoundaries(cse, pos, vel, 0, hashes, idx, old_pos, old_vel, 0, n, false);
  if (collide) ComputeBird(vel, cse, idx, g_ref_settings.partPerCell, dt, false);
  if (geometry)
    IntegrateAndProcessCollisions(pos, vel, 0, dt, g_ref_geom_hashes, n, false,
                                  g_ref_settings.periodicCondition);
  else
    Integrate(pos, vel, 0, dt, n, false, g_ref_settings.periodicCondition);
  if (sample) SampleCellStatistics(vel, cse, idx, false);
  return ref_status();
}

// DoBenchmark's loop of RunBenchmarkSimulationStep (include/gpu_dsmc.inl:220-274)
// for `steps` steps, for timing the reference's kernels: before each step the
// ping-pong buffers are swapped as particles.swap_* do, and every 100th step
// ends with SampleCellStatistics.  pos[k]/vel[k] (k = 0, 1) are the two
// buffers and `cur` the one that holds the state at the start; *cur_out is
// the one that holds it at the end.  *ms is the device time of the loop from
// CUDA events on the default stream, with one synchronisation at the end.
int ref_run_steps(float4* pos0, float4* pos1, float4* vel0, float4* vel1, uint* hashes, uint* idx,
                  uint2* cse, uint n, float dt, int collide, int geometry, int steps, int cur,
                  int* cur_out, float* ms) {
  float4* pos[2] = {pos0, pos1};
  float4* vel[2] = {vel0, vel1};
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  cudaEventRecord(t0, 0);
  for (int s = 1; s <= steps; ++s) {
    const int old = cur;
    cur = 1 - cur;
    CalculateCellIDs(pos[old], hashes, idx, n);
    SortParticlesIndices(hashes, idx, n);
    cudaMemset(cse, 0, g_ref_settings.getCellsCount() * sizeof(uint2));
    FindCellBoundaries(cse, pos[cur], vel[cur], 0, hashes, idx, pos[old], vel[old], 0, n, false);
    if (collide) ComputeBird(vel[cur], cse, idx, g_ref_settings.partPerCell, dt, false);
    if (geometry)
      IntegrateAndProcessCollisions(pos[cur], vel[cur], 0, dt, g_ref_geom_hashes, n, false,
                                    g_ref_settings.periodicCondition);
    else
      Integrate(pos[cur], vel[cur], 0, dt, n, false, g_ref_settings.periodicCondition);
    if (s % 100 == 0) SampleCellStatistics(vel[cur], cse, idx, false);
  }
  cudaEventRecord(t1, 0);
  cudaEventSynchronize(t1);
  cudaEventElapsedTime(ms, t0, t1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  *cur_out = cur;
  return ref_status();
}

}  // extern "C"
