/* CPU restatement of the reference's DSMC timestep (denglide/CudaDsmc).
 *
 * TEST INFRASTRUCTURE ONLY: this library is the checker for the product's
 * CUDA kernels and the timed CPU baseline.  The product never links it.
 *
 * Layout follows the reference: particle positions and velocities are float4
 * AoS (include/particles.h:34-74), cellStartEnd is uint2 per cell, the
 * collision statistics are float4 per cell and (sigma*g)max/remainder is
 * float2 per cell (kernels/dsmc_kernel.cu:117-133).
 */
#ifndef DSMC_ORACLE_H
#define DSMC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Step constants: gpu_sim_settings_t (kernels/dsmc_kernel.cu:79-101) plus the
 * extensions the product adds (VHS exponent, wall model). */
typedef struct {
  float gmin[3];
  float gmax[3];
  float cell[3];
  uint32_t dim[3];
  uint32_t cells;
  float cell_volume;
  float cross_section; /* pi*d^2 (float), InitSimulationProperties :323-325 */
  float fnum;
  char periodic;       /* 'x','y','z' or anything else = closed box */
  /* VHS: sigma(g) = cross_section * (vhs_gref / g)^(2*omega-1); omega = 0.5
   * reproduces the reference's hard sphere exactly. */
  float omega;
  float vhs_gref;
} orc_sim;

/* Geometry grid: collision_grid_t (kernels/dsmc_kernel.cu:109-115) and the
 * CSR upload of UploadIndices (:223-274). */
typedef struct {
  float bmin[3];
  float bmax[3];
  float cell[3];
  uint32_t dim[3];
  const uint32_t* flags;     /* per geometry cell, "has geometry" */
  const uint32_t* start_end; /* 2 per geometry cell (0xffffffff,0xffffffff = empty) */
  const uint32_t* tri_vidx;  /* 3 vertex ids per bin entry */
  const float* verts;        /* 3 floats per vertex */
  const float* normals;      /* 3 floats per bin entry */
} orc_geom;

/* HybridTaus generator (kernels/mtwister.cu:118-153). */
uint32_t orc_taus_int(uint32_t s[4]);
float orc_taus_float(uint32_t s[4]);

/* Mersenne Twister variant of the -mt path (kernels/mtwister.cu:40-117):
 * cfg = one 16-byte twister record (matrix_a, mask_b, mask_c, seed), st = 21
 * words (iState, mti1, mt[19]). */
uint32_t orc_mt_lcg(uint32_t a);
void orc_mt_seed_chain(uint32_t seed, uint32_t* cfg, uint32_t n);
void orc_mt_init(const uint32_t cfg[4], uint32_t st[21]);
uint32_t orc_mt_int(uint32_t st[21], const uint32_t cfg[4]);
float orc_mt_float(uint32_t st[21], const uint32_t cfg[4]);

/* Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11). */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

void orc_cell_ids(const orc_sim* s, const float* pos4, uint32_t n, uint32_t* keys, uint32_t* idx);
void orc_sort(uint32_t* keys, uint32_t* vals, uint32_t n, uint32_t nkeys);
void orc_bounds_reorder(const orc_sim* s, uint32_t n, const uint32_t* keys, const uint32_t* idx,
                        const float* opos4, const float* ovel4, float* spos4, float* svel4,
                        uint32_t* cse);
void orc_collide(const orc_sim* s, float* vel4, const uint32_t* cse, float* maxrem, float* stat4,
                 uint32_t* seeds, float avg_conc, float dt);
/* ComputeBirdCollisionsDev (the -mt collisions, kernels/dsmc_kernel.cu:1002-1089):
 * twister c per cell, 21 state words and 4 parameter words each. */
void orc_collide_mt(const orc_sim* s, float* vel4, const uint32_t* cse, float* maxrem, float* stat4,
                    uint32_t* mt_state, const uint32_t* mt_cfg, float avg_conc, float dt);
/* InitMaximums (kernels/dsmc_kernel.cu:1104-1120). */
void orc_init_maximums_mt(uint32_t cells, float max_rel_vel, uint32_t* mt_state,
                          const uint32_t* mt_cfg, float* maxrem);
void orc_move(const orc_sim* s, const orc_geom* g, float* pos4, float* vel4, uint32_t n, float dt);
void orc_sample(const orc_sim* s, const float* vel4, const uint32_t* cse, float* cell_stats7);
void orc_sample_f64(const orc_sim* s, const float* vel4, const uint32_t* cse, double* acc5);

/* One reference timestep (include/gpu_dsmc.inl:220-274) on ping-pong buffers:
 * old_* hold the state to be sorted; pos4/vel4 receive the sorted, collided,
 * moved state. */
void orc_step(const orc_sim* s, const orc_geom* g, float* pos4, float* old_pos4, float* vel4,
              float* old_vel4, uint32_t* keys, uint32_t* idx, uint32_t* cse, uint32_t n,
              float dt, float avg_conc, float* maxrem, float* stat4, uint32_t* seeds,
              int collide, int sample, float* cell_stats7);

/* Akenine-Moller triangle/box overlap (separating-axis test). */
int orc_tri_box_overlap(const float center[3], const float half[3], const float tri[9]);

/* Geometry grid build: Model::CreateGrid + reg_grid_t::encloseGrid
 * (src/model.cpp:733-769, src/reggrid.cpp:27-93).  Returns the number of bin
 * entries (tri_ids holds at most cap of them). */
long orc_build_grid(const float* verts, uint32_t nverts, const uint32_t* tris, uint32_t ntris,
                    const int dim[3], float bbox[6], float cell[3], uint32_t* count,
                    uint32_t* tri_ids, long cap, uint8_t* flags);

/* ---- The extension mode (fast_oracle.c): Philox streams, VHS, warp-collided
 * dense cells, nearest wall crossings with diffuse walls, per-face
 * boundaries, inflow.  No counterpart in the reference. */
typedef struct {
  uint32_t key[2];     /* Philox key: the run's 64-bit seed, low word first */
  uint32_t step;       /* timestep counter (Philox counter word 2) */
  float ntc_coef;      /* 0.5 F_N dt / V_c, rounded to float */
  float avg_conc;      /* particles per cell of the reference NTC (ntc_local = 0) */
  int ntc_local;       /* 1: N_c - 1 */
  int hard_sphere;
  float cross_section; /* hard sphere: sigma g = g cross_section */
  float vhs_k, vhs_c1; /* VHS: sigma g = vhs_k 2^(vhs_c1 log2 g) */
  uint32_t heavy_min;  /* pair count from which a cell is collided by a warp */
  uint32_t warp_cap;   /* cells holding more particles are collided by one lane */
  float tie_rel;       /* relative margin of an acceptance flagged as a near tie */
} orc_fast;

/* NTC collisions of every cell in the sorted SoA velocities (in place).
 * cell_info (optional): per cell the pair count, the collisions, the path
 * (0 none, 1 lane, 2 warp, 3 lane for a cell above warp_cap) and the near
 * ties; sum_g_out (optional): sum of the colliding pairs' relative speeds. */
void orc_collide_fast(const orc_fast* f, float* u, float* v, float* w, const uint32_t* start,
                      uint32_t ncells, float* maxrem, uint32_t* cell_info, double* sum_g_out);

typedef struct {
  float gmin[3];
  float gmax[3];
  float cell[3];
  uint32_t dim[3];
  int face_kind[6];    /* -x,+x,-y,+y,-z,+z: 0 specular, 1 diffuse, 2 outflow, 3 periodic, 4 inflow */
  float face_vstd[6];  /* sqrt(k T_face / m) */
  float dt;
  uint32_t key[2];
  uint32_t step;
  uint32_t ntris;      /* 0: no body */
  const float* tri;    /* 9 floats per triangle: the three vertices */
  const float* plane;  /* 4 floats per triangle: unit normal, offset (orc_tri_planes) */
  int wall_diffuse;
  float wall_vstd;
  float amb_rel;       /* relative margin of a crossing flagged as ambiguous */
} orc_fast_move;

/* Flights of n particles (SoA, in place); gidx0 + i is particle i's wall
 * stream.  live[i] = 0: the particle left the domain or was inside the body;
 * amb[i] = 1: a crossing within the margin (see fast_oracle.c). */
void orc_move_fast(const orc_fast_move* m, float* x, float* y, float* z, float* u, float* v,
                   float* w, uint32_t n, uint32_t gidx0, uint8_t* live, uint8_t* amb);
void orc_tri_planes(const float* tri9, uint32_t ntris, float* plane4);

typedef struct {
  int face;
  float number_flux;   /* simulator particles per unit area per second */
  float area;
  float stream[3];
  float vstd;
} orc_inflow;

/* The injection count of one step (k_inject_plan), remainder updated. */
uint32_t orc_inject_plan(const orc_inflow* in, float dt, float* remainder, uint32_t max_k);
/* One step's injection through an inflow face: returns the count k (at most
 * max_k) and writes the particles to x..w[0, k). */
uint32_t orc_inject_fast(const orc_inflow* in, const float gmin[3], const float gmax[3], float dt,
                         const uint32_t key[2], uint32_t step, float* remainder, uint32_t max_k,
                         float* x, float* y, float* z, float* u, float* v, float* w, uint8_t* amb,
                         float tie_rel);

int orc_set_threads(int n);
int orc_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
