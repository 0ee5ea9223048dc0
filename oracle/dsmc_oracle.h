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

int orc_set_threads(int n);
int orc_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
