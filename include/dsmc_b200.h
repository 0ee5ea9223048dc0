/* dsmc_b200 - B200-native DSMC timestep behind a plain C ABI.
 *
 * Drop-in boundary for the GPU solver path of denglide/CudaDsmc.  Every entry
 * point names the reference interface it replaces (file:line in that
 * project).  Conventions, compared with the reference:
 *   - state lives in a handle (the reference keeps it in module-level statics,
 *     kernels/dsmc_kernel.cu:117-137), so several solvers can coexist;
 *   - work is ordered on the handle's CUDA stream (dsmc_set_stream);
 *   - no exceptions cross the ABI: every call returns DSMC_OK or an error
 *     code and dsmc_last_error() describes the last failure (the reference
 *     polls cudaGetLastError and throws std::runtime_error,
 *     kernels/dsmc_kernel.cu:2053-2072);
 *   - particle state is structure-of-arrays FP32 (x, y, z, u, v, w) on the
 *     device; the host-side upload/download calls also accept the reference's
 *     float4 AoS layout.
 */
#ifndef DSMC_B200_H
#define DSMC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DSMC_B200_ABI_VERSION 1

/* Status codes. */
enum {
  DSMC_OK = 0,
  DSMC_ERR_ARG = 1,      /* invalid argument */
  DSMC_ERR_CONFIG = 2,   /* unreadable or inconsistent configuration */
  DSMC_ERR_CUDA = 3,     /* a CUDA call failed */
  DSMC_ERR_OOM = 4,      /* device allocation failed */
  DSMC_ERR_STATE = 5,    /* call out of order (e.g. step before init) */
  DSMC_ERR_CAPACITY = 6, /* particle count exceeded the handle's capacity */
  DSMC_ERR_IO = 7,       /* file could not be read */
  DSMC_ERR_DEVICE = 8    /* a kernel reported an error flag */
};

/* Boundary kinds of the six domain faces (extension; the reference only has
 * its four boundary functors, kernels/dsmc_kernel.cu:1316-1555). */
enum {
  DSMC_FACE_SPECULAR = 0,
  DSMC_FACE_DIFFUSE = 1,
  DSMC_FACE_OUTFLOW = 2,
  DSMC_FACE_PERIODIC = 3,
  DSMC_FACE_INFLOW = 4 /* outflow face that also injects free-stream particles */
};

enum { DSMC_RNG_TAUS = 0, DSMC_RNG_PHILOX = 1 };
enum { DSMC_INIT_REFERENCE = 0, DSMC_INIT_MAXWELL = 1, DSMC_INIT_BIMODAL = 2 };

/* Simulation settings: settings_t (include/sim_settings.h:32-69) plus the
 * extensions this library adds.  dsmc_config_default() gives the reference
 * defaults (include/dsmc.h, src/sim_settings.cpp:35-44). */
typedef struct dsmc_config {
  /* --- reference settings_t --- */
  float grid_min[3];
  float grid_max[3];
  int grid_dim[3];
  float density;        /* number density, m^-3 */
  float fnum;           /* real molecules per simulator particle */
  float temp;           /* free-stream temperature, K */
  float stream_vel[3];  /* m/s */
  char periodic;        /* 'x','y','z' or 'n' (reference boundary functors) */
  float gas_mass;       /* kg */
  float gas_diam;       /* m, at gas_tref */
  float gas_tref;       /* K */
  float dt;             /* s */
  int geometry;         /* 1: collide with the mesh set by dsmc_set_mesh */
  int benchmark;
  /* --- extensions --- */
  float gas_omega;      /* VHS viscosity exponent; 0.5 = hard sphere (reference) */
  int ntc_local;        /* 0: NTC uses the initial particles per cell (reference,
                           include/gpu_dsmc.inl:250); 1: uses N_c - 1 (Bird) */
  int rng;              /* DSMC_RNG_TAUS (reference per-cell HybridTaus) or DSMC_RNG_PHILOX */
  uint64_t seed;
  int face_mode;        /* 0: reference functors from `periodic`; 1: face_kind[] */
  int face_kind[6];     /* -x,+x,-y,+y,-z,+z */
  float face_temp[6];   /* wall temperature of diffuse faces, K */
  int wall_diffuse;     /* mesh wall: 0 specular (reference), 1 diffuse */
  float wall_temp;      /* K */
  int init_kind;        /* DSMC_INIT_* */
  float init_temp2;     /* second temperature of the bimodal start, K */
  int sample_every;     /* sampling interval in steps (reference: 100) */
  float capacity_factor;/* particle buffer capacity / initial count (>= 1) */
  uint32_t part_per_cell; /* 0: derive as the reference does, kernels/dsmc.cu:324-330 */
  int geom_nearest;     /* mesh hits: 0 = the reference's first listed triangle of the start
                           and end grid cells (kernels/dsmc_kernel.cu:1256-1314,1621-1639);
                           1 = nearest triangle along the whole path */
} dsmc_config;

typedef struct dsmc_handle dsmc_handle;

/* Fills the reference defaults (settings_t::settings_t). */
int dsmc_config_default(dsmc_config* cfg);

/* settings_t::readFromFile (src/sim_settings.cpp:46-132): <grid><min/max/dim>,
 * <density>, <fnum>, <temp>, <streamvel>, <periodic>, <gas file=...>name</gas>,
 * plus the extension tags <omega>, <wall kind= T=>, <face ...>, <rng>, <seed>,
 * <sample every=>.  The gas file is looked up relative to the working
 * directory first (as the reference does), then to the XML file's directory. */
int dsmc_config_read_xml(const char* path, dsmc_config* cfg);

/* settings_t::readFromCmdLine (src/sim_settings.cpp:134-186): -f, -benchmark,
 * -no-geometry, -density, -dt, -run-for.  -mt is rejected here: the -mt
 * collisions need the twister file, which the caller loads with
 * dsmc_read_twisters and hands to dsmc_set_twisters (dsmc_bench does this). */
int dsmc_config_from_args(int argc, const char* const* argv, dsmc_config* cfg, float* run_for);

/* CreateSolver(SolverGPU) + DSMCSolver::Init (kernels/dsmc_base.cu:43-47,
 * 221-233; include/gpu_dsmc.inl:341-378): allocates the particle and per-cell
 * buffers on the current device. */
int dsmc_create(const dsmc_config* cfg, dsmc_handle** out);
int dsmc_destroy(dsmc_handle* h);
const char* dsmc_last_error(const dsmc_handle* h);
const char* dsmc_status_string(int status);

/* Orders all of the handle's work on this stream (a cudaStream_t; NULL = legacy default). */
int dsmc_set_stream(dsmc_handle* h, void* stream);
/* Synchronises the stream and reports device-side error flags. */
int dsmc_sync(dsmc_handle* h);

/* Derived quantities (settings_t/main, kernels/dsmc.cu:324-330; InitSimulationProperties,
 * kernels/dsmc_kernel.cu:309-348). */
typedef struct dsmc_info {
  uint32_t part_per_cell;
  uint32_t cells;
  uint32_t capacity;
  uint32_t num_particles;
  float cell_size[3];
  float cell_volume;
  float cross_section;
  float max_rel_vel;
  uint64_t step;
  uint32_t samples;
  double sim_time;
  uint64_t particle_steps; /* sum over steps of the particles in cells */
  uint32_t injected;       /* particles injected by inflow faces (total) */
  uint32_t removed;        /* particles removed through outflow faces (total) */
  uint32_t giant_cells;    /* cells processed outside the shared-memory tiles (total) */
  uint32_t mesh_flights;   /* flights of the last step tested against the mesh (split variants) */
} dsmc_info;
int dsmc_get_info(dsmc_handle* h, dsmc_info* info);

/* Per-kernel timing with CUDA events recorded around every launch of
 * dsmc_step and dsmc_step_graph on the handle's stream (no equivalent in the
 * reference, which times the whole loop only, kernels/dsmc.cu:440-449).  A
 * graph is captured with event-record nodes around the profiled kernels,
 * retargeted at fresh events before each replay, and captured again when the
 * profiled set changes.  dsmc_profile(h, 1)
 * starts a window, dsmc_profile_read returns per kernel the summed
 * milliseconds and launch counts since then (kernels: 0 scan, 1 scatter,
 * 2 cell, 3 inflow injection) and closes the window. */
int dsmc_profile(dsmc_handle* h, int enable);
int dsmc_profile_read(dsmc_handle* h, double ms[4], uint32_t launches[4]);
/* The same window kernel by kernel (n slots, at most 8 used): 0 scan,
 * 1 scatter, 2 the fused cell kernel or, with a split variant
 * (dsmc_set_kernel_variant >= 4), its order kernel (gather, stable order,
 * pair counts), 3 inflow injection, 4 flight, 5 flights that may reach the
 * body, 6 sampling, 7 NTC selections.  dsmc_profile_read reports slots 2 and
 * 4-7 summed as "cell".  No counterpart in the reference. */
int dsmc_profile_read_kernels(dsmc_handle* h, int n, double* ms, uint32_t* launches);
/* Restricts the open window's events to the slots whose bits are set in
 * `slots` (bit k = slot k above); dsmc_profile(h, 1) times all of them.  An
 * event pair around a kernel costs the GPU a few microseconds, so a timed run
 * keeps them to the kernel it reports on.  No counterpart in the reference. */
int dsmc_profile_mask(dsmc_handle* h, uint32_t slots);

/* DSMCSolver::SetModel -> Model::CreateGrid + InitRegularGrid
 * (kernels/dsmc_base.cu:49-55, src/model.cpp:733-769,
 * kernels/dsmc_kernel.cu:350-376): bins the triangle mesh into a uniform grid
 * of grid_dim cells over the mesh's bounding box and uploads it.  tris holds
 * 3 vertex ids per triangle; face normals are computed as
 * normalize(cross(v1-v0, v2-v0)) unless normals (3 floats per triangle) is
 * given. */
int dsmc_set_mesh(dsmc_handle* h, const float* verts, uint32_t nverts, const uint32_t* tris,
                  uint32_t ntris, const float* normals, const int grid_dim[3]);

/* Uploads a prebuilt geometry grid as the reference stores it in .raw files
 * and reg_grid_t (include/reggrid.h:32-56): bbox, cell size, dims, per-cell
 * triangle count, triangle ids in bin order, per-cell flag (after the
 * enclose fill). */
int dsmc_set_geometry_grid(dsmc_handle* h, const float bbox[6], const float cell[3],
                           const int dim[3], const uint32_t* cell_count, const uint32_t* tri_ids,
                           const uint8_t* flags, const float* verts, uint32_t nverts,
                           const uint32_t* tris, uint32_t ntris, const float* normals);

/* The geometry-grid builder on the host (the same binning as dsmc_set_mesh
 * computes on the device).
 * Returns the number of bin entries through *n_entries (tri_ids holds at most
 * cap of them). */
int dsmc_build_geometry_grid(const float* verts, uint32_t nverts, const uint32_t* tris,
                             uint32_t ntris, const int grid_dim[3], float bbox[6], float cell[3],
                             uint32_t* cell_count, uint32_t* tri_ids, uint64_t cap,
                             uint8_t* flags, uint64_t* n_entries);

/* The handle's geometry grid as dsmc_set_mesh built it on the device (or as
 * dsmc_set_geometry_grid received it): bbox, cell size, dims, per-cell
 * triangle count, triangle ids in bin order, per-cell flag, and with planes
 * != NULL each entry's plane (unit normal x, y, z and offset; 4 floats per
 * entry) read from the device.  Any output may be NULL; tri_ids and planes
 * hold at most cap entries; *n_entries gets the entry count. */
int dsmc_get_geometry_grid(dsmc_handle* h, float bbox[6], float cell[3], int dim[3],
                           uint32_t* cell_count, uint32_t* tri_ids, float* planes, uint64_t cap,
                           uint8_t* flags, uint64_t* n_entries);

/* Model::LoadRaw (src/model.cpp:348-401): reads the reference's .raw mesh
 * (vertices, indices, face normals).  With verts == NULL only the counts are
 * returned. */
int dsmc_read_raw_mesh(const char* path, float* verts, uint32_t* nverts, uint32_t* tris,
                       uint32_t* ntris, float* face_normals);

/* Triangulated test bodies: an icosphere (subdivision level, 20*4^level
 * triangles) and a blunt capsule (spherical nose + cone + flat base, ~ntarget
 * triangles, seeded jitter of the azimuthal start).  With verts == NULL only
 * the counts are returned. */
int dsmc_mesh_icosphere(int level, float radius, const float center[3], float* verts,
                        uint32_t* nverts, uint32_t* tris, uint32_t* ntris);
int dsmc_mesh_capsule(float nose_radius, float cone_half_angle_deg, float length,
                      const float nose_center[3], uint32_t ntarget, uint64_t seed, float* verts,
                      uint32_t* nverts, uint32_t* tris, uint32_t* ntris);

/* GPUDSMCSolver::InitSystemState (include/gpu_dsmc.inl:68-92): fills the
 * domain with part_per_cell particles per cell (skipping cells flagged as
 * geometry) and runs a zero-length move.  Returns the particle count. */
int dsmc_init_state(dsmc_handle* h, const float stream_vel[3], uint32_t* n_out);

/* Seeds the particle population from per-cell fields instead of the
 * free-stream fill (extension; the reference only has the uniform fill,
 * kernels/dsmc_kernel.cu:394-427): fields5 holds per cell (x fastest) the
 * number density n [m^-3], the mean velocity (u, v, w) [m/s] and the
 * temperature T [K].  n is the density averaged over the whole cell volume,
 * the convention of dsmc_read_fields, so that fields sampled from a run seed
 * each cell with the particle count it had: each cell receives n V_c / F_N
 * particles (rounded stochastically from the seed) drawn from the Maxwellian
 * at (u, v, w, T), in a cell the mesh cuts all of them in the part outside
 * the body; a cell none of whose 4 x 4 x 4 sub-cell centres lies outside the
 * mesh counts as covered and stays empty, as in dsmc_init_state; non-finite or
 * non-positive n gives an empty cell, a non-finite or non-positive T the
 * configured temperature.  Resets the sampling accumulators. */
int dsmc_init_from_fields(dsmc_handle* h, const float* fields5, uint32_t* n_out);

/* dsmc_init_from_fields with each cell's Maxwellian replaced by a two-stream
 * mixture (extension): a share alpha of the cell's particles is drawn from
 * the free stream (the configured stream velocity and temperature), the
 * rest from a Maxwellian whose drift and temperature keep the cell's mean
 * velocity and energy.  alpha is weight times the share at which that rest
 * has the wall temperature (the configured wall_temp, which must be
 * positive), found per cell by bisection on [0, 0.98]; 0 where the cell is
 * colder than the wall or no such share exists.  In rarefied flow a cell
 * holds free-stream molecules beside molecules re-emitted by the wall, and a
 * single Maxwellian with their mean and temperature relaxes to that only
 * over a transit of the domain.  weight in [0, 1] (0: dsmc_init_from_fields
 * itself); particle counts as dsmc_init_from_fields. */
int dsmc_init_from_fields_two_stream(dsmc_handle* h, const float* fields5, float weight, uint32_t* n_out);

/* Host <-> device particle state.  soa != 0: six arrays of n floats
 * (x,y,z,u,v,w) back to back; soa == 0: pos4 and vel4 float4 AoS as the
 * reference's particles_state_t.  Upload resets the cell order. */
int dsmc_upload_state(dsmc_handle* h, const float* pos, const float* vel, uint32_t n, int soa);
int dsmc_download_state(dsmc_handle* h, float* pos, float* vel, uint32_t* n, int soa);
/* The cell key of every particle slot that dsmc_download_state returns, in
 * the same order: the cell the particle sits in for the next step's sort, or
 * 0xffffffff for a particle that left the domain (outflow) or was found
 * inside the body.  The reference keeps its keys (gridHashes,
 * include/gpu_dsmc.inl:352-359) internal; this exposes them for parity
 * checks. */
int dsmc_read_keys(dsmc_handle* h, uint32_t* keys, uint32_t* n);
/* The -mt collisions (ComputeBirdCollisionsDev, kernels/dsmc_kernel.cu:1002-1089):
 * cell c draws its NTC pairs and angles from Mersenne Twister c, the variant of
 * kernels/mtwister.cu:30-117.  cfg4: per cell (matrix_a, mask_b, mask_c, seed),
 * as dsmc_read_twisters returns them; state21: per cell (iState, mti1, mt[19]),
 * or NULL to initialise each twister from its seed (InitTwisterFast,
 * kernels/mtwister.cu:108-117).  init_maximums: also set (sigma g)max and the
 * remainders as the reference's start does: InitMaximums (kernels/dsmc_kernel.cu:
 * 1104-1120) runs before the twisters are initialised (include/gpu_dsmc.inl:363-367)
 * and draws from zeroed states, so every remainder is (0 + 1) / 2^32.
 * Needs the reference RNG mode (rng taus) and the split kernels (variants 4
 * and up; a fused variant is replaced by 5).  The twisters are not part of
 * snapshots. */
int dsmc_set_twisters(dsmc_handle* h, const uint32_t* cfg4, const uint32_t* state21,
                      int init_maximums);
int dsmc_get_twisters(dsmc_handle* h, uint32_t* state21);
/* InitGPUTwisters' host part (kernels/mtwister.cu:46-68): the first `count`
 * 16-byte records of a twister parameter file (data/MersenneTwister.dat), each
 * seed replaced by the next value of the chain seed <- seed * 279470273 mod
 * 4294967291 started from `seed` (SEED = 999 in the reference). */
int dsmc_read_twisters(const char* path, uint32_t seed, uint32_t count, uint32_t* cfg4);
/* Per-cell collision state: (sigma*g)max and remainder (float2 per cell,
 * kernels/dsmc_kernel.cu:131) and HybridTaus seeds (uint4 per cell, :124). */
int dsmc_set_cell_state(dsmc_handle* h, const float* maxrem, const uint32_t* seeds);
int dsmc_get_cell_state(dsmc_handle* h, float* maxrem, uint32_t* seeds);

/* RunSimulationStep / DoBenchmark (include/gpu_dsmc.inl:128-274,
 * kernels/dsmc_base.cu:64-84): nsteps timesteps of length dt, sampling every
 * sample_every steps.  Asynchronous on the handle's stream. */
int dsmc_step(dsmc_handle* h, float dt, int nsteps);
/* Same as dsmc_step but replays a captured CUDA graph of the step (captured
 * on the first call, and again after a change of dt, variant or profiled
 * kernel set). */
int dsmc_step_graph(dsmc_handle* h, float dt, int nsteps);

/* Launch shape of the step's cell kernel (no counterpart in the reference,
 * whose kernels use fixed block sizes).  Variants 0-3 are a CTA-wide kernel:
 * 0 = 512 threads per CTA and up to 2048 particles per shared-memory chunk,
 * 1 = 256/1024, 2 = 128/512, 3 = 64/256.  Variants 4-7 are split kernels
 * whose warps each work through their own tiles of 32 cells, with chunks of
 * up to 256 (4) or 128 (5-7) particles per warp; 5 is the default.  Results
 * do not
 * depend on the variant, except in the Philox mode for a cell holding more
 * particles than the chunk (it is then collided by one thread instead of one
 * warp, a different but equivalent stream of draws).  Changing it drops the
 * captured graph. */
int dsmc_set_kernel_variant(dsmc_handle* h, int variant);
int dsmc_get_kernel_variant(dsmc_handle* h, int* variant, int* chunk_capacity);
/* Number of cell-kernel variants (valid variants are 0 .. count-1). */
int dsmc_kernel_variant_count(void);
/* Times `steps` graph-replayed timesteps (after 2 warm-up steps) of every
 * split variant (4 .. count-1, count = dsmc_kernel_variant_count()) and keeps
 * the fastest.  These are real timesteps of the run: the simulation advances
 * by (count - 4) * (steps + 2) steps.  ms_per_step (optional) receives count
 * times in milliseconds (0 for the fused variants 0-3, which are not timed).
 * Blocks until done. */
int dsmc_autotune(dsmc_handle* h, float dt, int steps, int* best, float* ms_per_step);

/* Batches (no counterpart in the reference, which runs one solver per
 * process): independent handles of uneven size advanced together, one CUDA
 * graph launch per timestep in which each kernel of the step runs once for
 * all members (each member in a share of the grid that follows its particle
 * count), so that the ensemble fills the GPU like one large instance.
 * Members run the split kernels with the order kernel's (128 particles,
 * 4 warps) shape whatever shape they use alone; the -mt collisions are
 * refused.  Members must live on the current device and appear once; the
 * batch does not own them (destroy the batch first).  Batch work is ordered
 * on the batch stream, not on the members' streams: call dsmc_batch_sync
 * before using a member on its own.  The graph is captured on the first step
 * and again whenever a dt or a member's launch set changes (mesh, stream).
 * Results equal stepping each member alone with that shape. */
typedef struct dsmc_batch dsmc_batch;
int dsmc_batch_create(dsmc_handle* const* members, uint32_t n, dsmc_batch** out);
int dsmc_batch_destroy(dsmc_batch* b);
const char* dsmc_batch_last_error(const dsmc_batch* b);
/* Orders the batch's launches on this stream (NULL: a stream of its own). */
int dsmc_batch_set_stream(dsmc_batch* b, void* stream);
/* nsteps timesteps of every member; dt holds one step length per member
 * (NULL: each member's configured dt).  Asynchronous on the batch stream. */
int dsmc_batch_step(dsmc_batch* b, const float* dt, int nsteps);
/* Synchronises the batch stream and reports the members' device error flags. */
int dsmc_batch_sync(dsmc_batch* b);
/* dsmc_autotune for every member, for the shape it uses when stepped alone
 * (each advances by (count - 4) * (steps + 2) steps); variants (optional)
 * receives the chosen variant per member. */
int dsmc_batch_autotune(dsmc_batch* b, const float* dt, int steps, int* variants);

/* SampleCellStatistics (kernels/dsmc_kernel.cu:892-910): adds the current
 * velocities to the FP64 per-cell accumulators now. */
int dsmc_sample(dsmc_handle* h);
int dsmc_reset_samples(dsmc_handle* h);

/* Per-cell FP64 accumulators: 5 doubles per cell (count, sum u, sum v, sum w,
 * sum |v|^2) and the number of sampling passes. */
int dsmc_read_cell_sums(dsmc_handle* h, double* sums5, uint32_t* nsamples);
/* ProcessAndOutputStatistics' per-cell fields (kernels/dsmc_base.cu:104-163):
 * n = fnum N/(V samples), u = sum v / N, T = m (sum|v|^2/N - |u|^2)/(3k);
 * 5 doubles per cell (n, ux, uy, uz, T). */
int dsmc_read_fields(dsmc_handle* h, double* fields5);
/* GetStatistics (kernels/dsmc_kernel.cu:840-854): selections, collisions,
 * sum of relative speeds of collisions (all steps so far). */
int dsmc_get_totals(dsmc_handle* h, double totals[3]);
/* The same totals without waiting: enqueues on the handle's stream a copy of
 * 24 bytes into `out` (selections and collisions as uint64, the sum of
 * relative speeds as double), valid once the stream has passed this point
 * (an event recorded after the call, or dsmc_sync).  `out` should be pinned
 * host memory for the copy to stay asynchronous.  No counterpart in the
 * reference, which reads its statistics synchronously; it lets a host read
 * every step's totals while the next step runs. */
int dsmc_totals_async(dsmc_handle* h, void* out);
/* DSMCSolver::DumpStatistics (kernels/dsmc_base.cu:165-174) as text. */
int dsmc_dump_statistics(dsmc_handle* h, const char* path);

/* Binary snapshot of the whole handle state (particles, per-cell state,
 * accumulators, counters) and its restore. */
int dsmc_snapshot(dsmc_handle* h, const char* path);
int dsmc_restore(dsmc_handle* h, const char* path);

/* ---------------------------------------------------------------------
 * Stage API: the individual stages of one timestep on caller-owned device
 * pointers, ordered on `stream` (cudaStream_t).  These run the same device
 * code as dsmc_step.  Cell grids are described by dsmc_grid.
 * ------------------------------------------------------------------- */
typedef struct dsmc_grid {
  float gmin[3];
  float gmax[3];
  float cell[3];
  uint32_t dim[3];
} dsmc_grid;

/* CalculateCellIDs (kernels/dsmc_kernel.cu:1712-1732): keys[i] = cell id of
 * (x[i],y[i],z[i]), idx[i] = i. */
int dsmc_stage_cell_index(const dsmc_grid* g, const float* x, const float* y, const float* z,
                          uint32_t n, uint32_t* keys, uint32_t* idx, void* stream);

/* SortParticlesIndices (kernels/dsmc_kernel.cu:2033-2051): stable sort of
 * (keys, vals) by key, keys < nkeys; also writes the exclusive cell starts
 * (nkeys+1 entries) when cell_start != NULL.  workspace may be NULL (the call
 * then allocates on the stream); dsmc_stage_sort_workspace gives its size. */
int dsmc_stage_sort_workspace(uint32_t n, uint32_t nkeys, size_t* bytes);
int dsmc_stage_sort(uint32_t* keys, uint32_t* vals, uint32_t n, uint32_t nkeys,
                    uint32_t* cell_start, void* workspace, size_t workspace_bytes, void* stream);

/* dsmc_stage_sort without any allocation (no counterpart in the reference):
 * for callers that may not allocate device memory while they run, such as
 * code recording work into a memory-constrained pool or running next to a
 * caching allocator that owns the device.  The scratch is a fixed static
 * device array of about 13.6 MB, reserved on each device when the library's
 * kernels are loaded there; this call never calls cudaMalloc, cudaFree or an
 * allocating library function.
 * Limits: n <= DSMC_SORT_STATIC_MAX_N and nkeys <= DSMC_SORT_STATIC_MAX_KEYS;
 * larger sizes return DSMC_ERR_CAPACITY before any device work.
 * The scratch address is looked up once per device on the first call there;
 * make that first call outside any stream capture.  The address is kept for
 * the life of the process: after a reset of the device (cudaDeviceReset, or
 * a reset of its primary context) the array may sit elsewhere, so a process
 * that resets a device must not call this entry point on it again.  Every call zeroes the
 * scratch counters it needs on `stream` itself, so nothing has to be cleared
 * beforehand.  All calls on one device share the scratch: calls that may
 * overlap (different streams or host threads without ordering between them)
 * race and corrupt each other's results; order them on one stream. */
#define DSMC_SORT_STATIC_MAX_N 1048576u
#define DSMC_SORT_STATIC_MAX_KEYS 131072u
int dsmc_stage_sort_static(uint32_t* keys, uint32_t* vals, uint32_t n, uint32_t nkeys,
                           uint32_t* cell_start, void* stream);

/* FindCellBoundaries (kernels/dsmc_kernel.cu:1734-1808): cell start/end
 * (uint2 per cell, (0,0) for empty cells) from sorted keys, and the gather of
 * the six state arrays into sorted order (src -> dst). */
int dsmc_stage_bounds_reorder(const uint32_t* sorted_keys, const uint32_t* sorted_idx, uint32_t n,
                              uint32_t ncells, uint32_t* cell_start_end, const float* const src[6],
                              float* const dst[6], void* stream);

/* Collision constants for the collide stage (gpu_sim_settings_t fields,
 * kernels/dsmc_kernel.cu:79-101). */
typedef struct dsmc_collide_params {
  uint32_t ncells;
  float cell_volume;
  float cross_section;
  float fnum;
  float avg_conc;
  float dt;
  float omega;
  float vhs_gref;
  int ntc_local;
  int rng;
  uint64_t seed;
  uint32_t step;
} dsmc_collide_params;

/* ComputeBirdCollisionsNoMTDev (kernels/dsmc_kernel.cu:912-1102): NTC
 * collisions in every cell of the sorted velocity arrays (u,v,w in place),
 * cells given by cell_start (ncells+1 exclusive starts).  maxrem (float2 per
 * cell) and seeds (uint4 per cell, HybridTaus) are updated; stat4 (float4 per
 * cell: selections, collisions, sum g) is accumulated when non-NULL. */
int dsmc_stage_collide(const dsmc_collide_params* p, float* u, float* v, float* w,
                       const uint32_t* cell_start, float* maxrem, uint32_t* seeds, float* stat4,
                       void* stream);

/* Move constants: the simulation grid and the boundary treatment. */
typedef struct dsmc_move_params {
  dsmc_grid grid;
  float dt;
  char periodic;
  int face_mode;
  int face_kind[6];
  float face_vstd[6];
  uint64_t seed;
  uint32_t step;
} dsmc_move_params;

/* The lower bound of the distance to the body that decides which flights
 * the step tests against the mesh (no counterpart in the reference, which
 * tests every flight starting or ending in a cell with triangles): out[i] for
 * the point xyz[3i..3i+2] (device pointers), -1 outside the geometry grid.
 * The table is built with the mesh (dsmc_set_mesh). */
int dsmc_clearance_at(dsmc_handle* h, const float* xyz, uint32_t n, float* out, void* stream);

/* Per bin entry of the geometry grid (the order of dsmc_get_geometry_grid's
 * tri_ids), the reach of the entry's triangle as two floats (r, k): a
 * particle re-emitted or reflected from the triangle whose remaining path is
 * shorter than r and whose direction makes more than k with the triangle's
 * normal (the sine of its elevation) cannot cross a listed triangle, so the
 * nearest-hit traversal stops without a second walk of the grid.  Triangles
 * near it that rise above its plane either cap r (by a lower bound of their
 * distance) or, when their rise is bounded by a slope below 1/2 of the
 * distance from the triangle, raise k to that slope.  r = 0 where no path
 * qualifies.  At most cap pairs into out (host memory, 2 floats each);
 * *n_entries gets the entry count, and 0 when the table is off (a body more
 * than 2 m from the origin, where the 1 um set-off from the wall nears the
 * coordinates' rounding). */
int dsmc_get_entry_reach(dsmc_handle* h, float* out, uint64_t cap, uint64_t* n_entries);

/* Per cell of the geometry grid (cell-major, x fastest), the slab that holds
 * every vertex of the cell's listed triangles, as 4 floats (m.x, m.y, m.z,
 * e): |m . v - e| <= 1 for each such vertex v (m the triangles' mean normal
 * over the slab's half thickness); (0, 0, 0, 0) for an empty cell or one
 * whose normals disagree.  The mesh step skips a cell whose slab a path
 * stays outside.  At most cap cells into out (host memory); *n_cells gets
 * the cell count. */
int dsmc_get_cell_slabs(dsmc_handle* h, float* out, uint64_t cap, uint64_t* n_cells);

/* IntegrateDev / ProcessCollisionsDev (kernels/dsmc_kernel.cu:1557-1699):
 * free flight, mesh collisions (with the handle's geometry when h != NULL and
 * it has one) and the boundary functor, in place on the six arrays. */
int dsmc_stage_move(dsmc_handle* h, const dsmc_move_params* p, float* x, float* y, float* z,
                    float* u, float* v, float* w, uint32_t n, void* stream);

/* SampleCellStatisticsDev (kernels/dsmc_kernel.cu:856-910) in FP64: adds
 * count, sums of u,v,w and |v|^2 per cell into sums5 (5 doubles per cell). */
int dsmc_stage_sample(const float* u, const float* v, const float* w, const uint32_t* cell_start,
                      uint32_t ncells, double* sums5, void* stream);

/* --- Warm-start surrogate kernels (no counterpart in the reference) ---
 * Device pointers, asynchronous on `stream`.  BF16 operands, FP32
 * accumulation; the GEMM runs on the tensor cores (tcgen05.mma, its
 * accumulator in tensor memory), 128 x 128 tiles.  dsmc_gemm_bf16: c = A B (+ bias) (+ beta c) for an m x n
 * result; a_trans = 1 reads A stored k x m, b_trans = 1 reads B stored n x k
 * (row-major, leading dimensions lda/ldb/ldc/ldcb in elements).  act = 1
 * applies GELU: c keeps the pre-activation, c_bf16 (optional) receives the
 * activation in BF16.  Requires k, lda, ldb multiples of 8, 16-byte aligned
 * A and B, m a multiple of 8 when a_trans, n a multiple of 8 unless b_trans.
 * split_k > 1 splits the reduction and adds into c with atomics (c zeroed by
 * the caller; no bias, act or c_bf16). */
int dsmc_gemm_bf16(int m, int n, int k, const void* a, int lda, int a_trans, const void* b, int ldb,
                   int b_trans, float* c, int ldc, float beta, const float* bias, int act, void* c_bf16,
                   int ldcb, int split_k, void* stream);
/* Synchronises `stream` and reports whether a dsmc_gemm_bf16 launch since
 * the last check gave up waiting on its tensor-core work (DSMC_ERR_DEVICE;
 * its output is then incomplete); clears the flag. */
int dsmc_gemm_check(void* stream);
/* dz = dh * GELU'(z), in FP32 and/or BF16. */
int dsmc_gelu_backward(const float* z, const float* dh, float* dz, void* dz_bf16, size_t n,
                       void* stream);
/* out[col] = sum over rows of x[row * ld + col]. */
int dsmc_colsum(const float* x, int rows, int cols, int ld, float* out, void* stream);
/* Masked mean-square error: for every finite BF16 target t, loss += (y - t)^2,
 * count += 1 and dy = scale * 2 (y - t); NaN targets give dy = 0. */
int dsmc_mse_grad(const float* y, const void* t_bf16, size_t n, float scale, void* dy_bf16, float* dy,
                  double* loss, unsigned long long* count, void* stream);
/* Adam step t (>= 1) with decoupled weight decay; refreshes w_bf16 if given. */
int dsmc_adam_step(float* w, const float* g, float* m, float* v, void* w_bf16, size_t n, float lr,
                   float b1, float b2, float eps, int t, float weight_decay, void* stream);
int dsmc_to_bf16(const float* x, void* y, size_t n, void* stream);

#ifdef __cplusplus
}
#endif
#endif
