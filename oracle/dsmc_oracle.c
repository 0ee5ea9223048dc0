/* CPU restatement of the reference's DSMC timestep (denglide/CudaDsmc).
 *
 * TEST INFRASTRUCTURE ONLY.  The product (cudadsmc_b200/libdsmc_b200.so)
 * never links, loads or calls this file.  It serves as
 *   - the checker the parity tests compare the CUDA kernels against, and
 *   - the timed CPU baseline (OpenMP over all host threads).
 *
 * Each function cites the reference lines it restates.  Floating point
 * follows the reference's device arithmetic: FP32 everywhere except where the
 * reference promotes to double (the NTC pair count, the HybridTaus scaling,
 * the periodic wrap and the triangle-test determinant threshold).  The build
 * uses -ffp-contract=off; the multiply-adds that nvcc contracts in the
 * reference build are written as fmaf() at the places noted.  CUDA's fast
 * __cosf/__sinf intrinsics are replaced by libm cosf/sinf, so post-collision
 * velocities agree with the GPU within a stated tolerance, not bit for bit.
 */
#include "dsmc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_PI_F 3.14159265358979f /* DSMC_PI, include/dsmc.h:26 */
#define ORC_BOUNCE_DELTA 0.001     /* double, kernels/dsmc_kernel.cu:53 */
#define ORC_COLLISION_LIMIT 10u    /* kernels/dsmc_kernel.cu:1250 */
#define ORC_EPS 0.0001f            /* kernels/dsmc_kernel.cu:1251 */
#define ORC_MODEL_WIDTH 0.0001f    /* kernels/dsmc_kernel.cu:1253 */
#define ORC_TRI_EPSILON 0.000001   /* double, kernels/tri_intersect.cu:1 */
#define ORC_NONE 0xffffffffu

static int g_threads = 0;

int orc_set_threads(int n) {
  g_threads = n;
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#endif
  return 0;
}

int orc_get_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* float -> uint conversion with the device's round-toward-zero saturating
 * semantics (cvt.rzi.u32.f32: NaN and negatives give 0). */
static inline uint32_t f2u_sat(float f) {
  if (!(f > 0.0f)) return 0u;
  if (f >= 4294967296.0f) return 0xffffffffu;
  return (uint32_t)f;
}

static inline uint32_t umin32(uint32_t a, uint32_t b) { return a < b ? a : b; }

/* x*x + y*y + z*z as the reference's device build evaluates it. */
static inline float len2f(float x, float y, float z) { return fmaf(z, z, fmaf(x, x, y * y)); }

/* ---------------------------------------------------------------- RNG ---- */

/* TausStep / LCGStep / HybridTausRng(Int), kernels/mtwister.cu:118-153. */
static inline uint32_t taus_step(uint32_t* z, int s1, int s2, int s3, uint32_t m) {
  uint32_t b = (((*z) << s1) ^ (*z)) >> s2;
  *z = (((*z) & m) << s3) ^ b;
  return *z;
}

uint32_t orc_taus_int(uint32_t s[4]) {
  uint32_t a = taus_step(&s[0], 13, 19, 12, 4294967294u);
  uint32_t b = taus_step(&s[1], 2, 25, 4, 4294967288u);
  uint32_t c = taus_step(&s[2], 3, 11, 17, 4294967280u);
  s[3] = s[3] * 1664525u + 1013904223u;
  return a ^ b ^ c ^ s[3];
}

float orc_taus_float(uint32_t s[4]) {
  /* double product, rounded to float on return (kernels/mtwister.cu:135-143). */
  return (float)(2.3283064365387e-10 * (double)orc_taus_int(s));
}

/* Mersenne Twister variant of the reference's -mt path and of its initial
 * fill (kernels/mtwister.cu, parameters include/MersenneTwister.h:31-40:
 * 19-word state, middle word 9, one lower bit, tempering shifts 12/7/15/18).
 * A twister's parameters are one 16-byte record of data/MersenneTwister.dat
 * (matrix_a, mask_b, mask_c, seed); its state is
 *   st[0] = iState, st[1] = mti1, st[2 .. 20] = mt[0 .. 18]
 * as in mt_state (kernels/mtwister.cu:30-35). */
#define ORC_MT_NN 19
#define ORC_MT_MM 9

/* lcg_rand, kernels/mtwister.cu:40-44 (unsigned long is 64 bits here). */
uint32_t orc_mt_lcg(uint32_t a) { return (uint32_t)(((uint64_t)a * 279470273ull) % 4294967291ull); }

/* The seed chain of InitGPUTwisters (kernels/mtwister.cu:46-68): twister i
 * gets the (i+1)-th value of lcg_rand from `seed`, in cfg[4*i+3]. */
void orc_mt_seed_chain(uint32_t seed, uint32_t* cfg, uint32_t n) {
  for (uint32_t i = 0; i < n; i++) {
    seed = orc_mt_lcg(seed);
    cfg[4 * i + 3] = seed;
  }
}

/* InitTwisterFast, kernels/mtwister.cu:108-117. */
void orc_mt_init(const uint32_t cfg[4], uint32_t st[21]) {
  uint32_t* mt = st + 2;
  mt[0] = cfg[3];
  for (int i = 1; i < ORC_MT_NN; i++) mt[i] = 1812433253u * (mt[i - 1] ^ (mt[i - 1] >> 30)) + (uint32_t)i;
  st[0] = 0;
  st[1] = mt[0];
}

/* GetRandomIntegerFast, kernels/mtwister.cu:70-101: one word of the ring
 * advanced per draw, then tempered. */
uint32_t orc_mt_int(uint32_t st[21], const uint32_t cfg[4]) {
  uint32_t* mt = st + 2;
  int i1 = (int)st[0] + 1, im = (int)st[0] + ORC_MT_MM;
  if (i1 >= ORC_MT_NN) i1 -= ORC_MT_NN;
  if (im >= ORC_MT_NN) im -= ORC_MT_NN;
  const uint32_t mti = st[1];
  st[1] = mt[i1];
  uint32_t x = (mti & 0xFFFFFFFEu) | (st[1] & 0x1u);
  x = mt[im] ^ (x >> 1) ^ ((x & 1u) ? cfg[0] : 0u);
  mt[st[0]] = x;
  st[0] = (uint32_t)i1;
  x ^= x >> 12;
  x ^= (x << 7) & cfg[1];
  x ^= (x << 15) & cfg[2];
  x ^= x >> 18;
  return x;
}

/* GetRandomFloatFast, kernels/mtwister.cu:103-106: float arithmetic. */
float orc_mt_float(uint32_t st[21], const uint32_t cfg[4]) {
  return ((float)orc_mt_int(st, cfg) + 1.0f) / 4294967296.0f;
}

/* The random source of one cell's collisions: HybridTaus (default) or the
 * cell's twister (-mt). */
typedef struct {
  uint32_t* taus;
  uint32_t* mt;
  const uint32_t* cfg;
} orc_cell_rng;

static inline uint32_t cell_rng_int(orc_cell_rng* r) {
  return r->mt ? orc_mt_int(r->mt, r->cfg) : orc_taus_int(r->taus);
}

static inline float cell_rng_float(orc_cell_rng* r) {
  return r->mt ? orc_mt_float(r->mt, r->cfg) : orc_taus_float(r->taus);
}

/* Philox-4x32 with 10 rounds: each round multiplies words 0 and 2 by the
 * published constants, mixes high halves with words 1,3 and the key, and the
 * key advances by the Weyl increments between rounds. */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; r++) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    c0 = hi1 ^ c1 ^ k0;
    c1 = lo1;
    c2 = hi0 ^ c3 ^ k1;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* ---------------------------------------------------------- cell index ---- */

/* GetCellID3D, kernels/dsmc_kernel.cu:1701-1710. */
static inline uint32_t cell_id3d(const orc_sim* s, const float* p) {
  uint32_t x = f2u_sat((p[0] - s->gmin[0]) / s->cell[0]);
  uint32_t y = f2u_sat((p[1] - s->gmin[1]) / s->cell[1]);
  uint32_t z = f2u_sat((p[2] - s->gmin[2]) / s->cell[2]);
  return umin32(z, s->dim[2] - 1) * s->dim[0] * s->dim[1] + umin32(y, s->dim[1] - 1) * s->dim[0] +
         umin32(x, s->dim[0] - 1);
}

/* CalculateCellIDsDev, kernels/dsmc_kernel.cu:1712-1724. */
void orc_cell_ids(const orc_sim* s, const float* pos4, uint32_t n, uint32_t* keys, uint32_t* idx) {
  long i;
#pragma omp parallel for schedule(static)
  for (i = 0; i < (long)n; i++) {
    keys[i] = cell_id3d(s, pos4 + 4 * i);
    idx[i] = (uint32_t)i;
  }
}

/* ---------------------------------------------------------------- sort ---- */

/* Stable sort of (key, value) pairs by key: the result thrust::sort_by_key
 * gives at kernels/dsmc_kernel.cu:2033-2051.  Counting sort; with several
 * threads each owns a contiguous chunk and its own histogram, which keeps the
 * order of equal keys. */
void orc_sort(uint32_t* keys, uint32_t* vals, uint32_t n, uint32_t nkeys) {
  if (n == 0) return;
  int nt = 1;
#ifdef _OPENMP
  nt = omp_get_max_threads();
  if (nt > 32) nt = 32;
  if ((size_t)n < (size_t)nt * 4096) nt = 1;
#endif
  uint32_t* hist = (uint32_t*)calloc((size_t)nt * nkeys, sizeof(uint32_t));
  uint32_t* k2 = (uint32_t*)malloc((size_t)n * sizeof(uint32_t));
  uint32_t* v2 = (uint32_t*)malloc((size_t)n * sizeof(uint32_t));
  const size_t chunk = ((size_t)n + nt - 1) / nt;
#pragma omp parallel num_threads(nt)
  {
    int t = 0;
#ifdef _OPENMP
    t = omp_get_thread_num();
#endif
    size_t b = (size_t)t * chunk, e = b + chunk;
    if (e > n) e = n;
    uint32_t* h = hist + (size_t)t * nkeys;
    for (size_t i = b; i < e; i++) h[keys[i]]++;
#pragma omp barrier
#pragma omp single
    {
      uint32_t run = 0;
      for (uint32_t k = 0; k < nkeys; k++)
        for (int tt = 0; tt < nt; tt++) {
          uint32_t c = hist[(size_t)tt * nkeys + k];
          hist[(size_t)tt * nkeys + k] = run;
          run += c;
        }
    }
    for (size_t i = b; i < e; i++) {
      uint32_t d = h[keys[i]]++;
      k2[d] = keys[i];
      v2[d] = vals[i];
    }
  }
  memcpy(keys, k2, (size_t)n * sizeof(uint32_t));
  memcpy(vals, v2, (size_t)n * sizeof(uint32_t));
  free(k2);
  free(v2);
  free(hist);
}

/* FindCellBoundariesDev with REORDER, kernels/dsmc_kernel.cu:1734-1787, after
 * the cudaMemset of include/gpu_dsmc.inl:104. */
void orc_bounds_reorder(const orc_sim* s, uint32_t n, const uint32_t* keys, const uint32_t* idx,
                        const float* opos4, const float* ovel4, float* spos4, float* svel4,
                        uint32_t* cse) {
  memset(cse, 0, (size_t)s->cells * 2 * sizeof(uint32_t));
  long i;
#pragma omp parallel for schedule(static)
  for (i = 0; i < (long)n; i++) {
    uint32_t h = keys[i];
    if (i == 0 || h != keys[i - 1]) {
      cse[2 * h] = (uint32_t)i;
      if (i > 0) cse[2 * keys[i - 1] + 1] = (uint32_t)i;
    }
    if (i == (long)n - 1) cse[2 * h + 1] = (uint32_t)i + 1;
    if (spos4) memcpy(spos4 + 4 * i, opos4 + 4 * (size_t)idx[i], 16);
    if (svel4) memcpy(svel4 + 4 * i, ovel4 + 4 * (size_t)idx[i], 16);
  }
}

/* ------------------------------------------------------------- collide ---- */

/* ComputeBirdCollisionsNoMTDev, kernels/dsmc_kernel.cu:912-1000 (one cell),
 * and ComputeBirdCollisionsDev (:1002-1089), the same steps with the cell's
 * twister as the random source.  With omega != 0.5 the acceptance uses the
 * VHS cross-section sigma(g) = cross_section * (vhs_gref/g)^(2*omega-1). */
static void collide_cell(const orc_sim* s, float* vel4, uint32_t c, const uint32_t* cse,
                         float* maxrem, float* stat4, orc_cell_rng* rng, float avg_conc, float dt) {
  uint32_t st = cse[2 * c], en = cse[2 * c + 1];
  int part = (int)(en - st);
  if (part < 2) return;
  float stat[4] = {stat4[4 * c], stat4[4 * c + 1], stat4[4 * c + 2], stat4[4 * c + 3]};
  float vmax_x = maxrem[2 * c], vmax_y = maxrem[2 * c + 1];
  /* (0.5*partCount*avgConc*fnum*vmax*dt)/cell_volume + rem, in double (:934). */
  float fpc = (float)((0.5 * (double)part * (double)avg_conc * (double)s->fnum * (double)vmax_x *
                       (double)dt) / (double)s->cell_volume + (double)vmax_y);
  uint32_t pairs = f2u_sat(fpc);
  stat[0] += (float)pairs;
  vmax_y = fpc - (float)pairs;
  const int hard_sphere = (s->omega == 0.5f);
  for (uint32_t i = 0; i < pairs; i++) {
    uint32_t px = st + cell_rng_int(rng) % (uint32_t)part;
    float v1[4];
    memcpy(v1, vel4 + 4 * (size_t)px, 16);
    uint32_t py = st + cell_rng_int(rng) % (uint32_t)part;
    float v2[4];
    memcpy(v2, vel4 + 4 * (size_t)py, 16);
    float mag = sqrtf(len2f(v1[0] - v2[0], v1[1] - v2[1], v1[2] - v2[2]));
    float v;
    if (hard_sphere)
      v = mag * s->cross_section;
    else
      v = mag * (s->cross_section * powf(s->vhs_gref / mag, 2.0f * s->omega - 1.0f));
    if (v / vmax_x > cell_rng_float(rng)) {
      stat[1] += 1.0f;
      stat[2] += mag;
      float b = 2.0f * cell_rng_float(rng) - 1.0f;
      float a = sqrtf(fmaf(-b, b, 1.0f));
      float cc = 2 * ORC_PI_F * cell_rng_float(rng);
      float ax = b * mag / 2.0f;
      float ay = a * mag * cosf(cc) / 2.0f;
      float az = a * mag * sinf(cc) / 2.0f;
      float* o1 = vel4 + 4 * (size_t)px;
      float* o2 = vel4 + 4 * (size_t)py;
      o1[0] = (v1[0] + v2[0]) / 2.0f + ax;
      o1[1] = (v1[1] + v2[1]) / 2.0f + ay;
      o1[2] = (v1[2] + v2[2]) / 2.0f + az;
      o2[0] = (v1[0] + v2[0]) / 2.0f - ax;
      o2[1] = (v1[1] + v2[1]) / 2.0f - ay;
      o2[2] = (v1[2] + v2[2]) / 2.0f - az;
    }
    if (v > vmax_x) vmax_x = v;
  }
  maxrem[2 * c] = vmax_x;
  maxrem[2 * c + 1] = vmax_y;
  memcpy(stat4 + 4 * c, stat, 16);
}

void orc_collide(const orc_sim* s, float* vel4, const uint32_t* cse, float* maxrem, float* stat4,
                 uint32_t* seeds, float avg_conc, float dt) {
  long c;
#pragma omp parallel for schedule(dynamic, 256)
  for (c = 0; c < (long)s->cells; c++) {
    orc_cell_rng r = {seeds + 4 * c, NULL, NULL};
    collide_cell(s, vel4, (uint32_t)c, cse, maxrem, stat4, &r, avg_conc, dt);
  }
}

/* The -mt collisions: cell c draws from twister c (state mt_state[21*c],
 * parameters mt_cfg[4*c]), as ComputeBirdCollisionsDev does
 * (kernels/dsmc_kernel.cu:1002-1089). */
void orc_collide_mt(const orc_sim* s, float* vel4, const uint32_t* cse, float* maxrem, float* stat4,
                    uint32_t* mt_state, const uint32_t* mt_cfg, float avg_conc, float dt) {
  long c;
#pragma omp parallel for schedule(dynamic, 256)
  for (c = 0; c < (long)s->cells; c++) {
    orc_cell_rng r = {NULL, mt_state + 21 * c, mt_cfg + 4 * c};
    collide_cell(s, vel4, (uint32_t)c, cse, maxrem, stat4, &r, avg_conc, dt);
  }
}

/* InitMaximums, kernels/dsmc_kernel.cu:1104-1120: (sigma g)max from the
 * settings and the remainder from one draw of the cell's twister. */
void orc_init_maximums_mt(uint32_t cells, float max_rel_vel, uint32_t* mt_state,
                          const uint32_t* mt_cfg, float* maxrem) {
  for (uint32_t c = 0; c < cells; c++) {
    maxrem[2 * c] = max_rel_vel;
    maxrem[2 * c + 1] = orc_mt_float(mt_state + 21 * (size_t)c, mt_cfg + 4 * (size_t)c);
  }
}

/* ---------------------------------------------------------------- move ---- */

/* GetCollisionCellID(float4), kernels/dsmc_kernel.cu:180-204. */
static inline uint32_t coll_cell_id(const orc_geom* g, const float* p) {
  if (p[0] < g->bmin[0] || p[1] < g->bmin[1] || p[2] < g->bmin[2] || p[0] > g->bmax[0] ||
      p[1] > g->bmax[1] || p[2] > g->bmax[2])
    return ORC_NONE;
  uint32_t x = f2u_sat((p[0] - g->bmin[0]) / g->cell[0]);
  uint32_t y = f2u_sat((p[1] - g->bmin[1]) / g->cell[1]);
  uint32_t z = f2u_sat((p[2] - g->bmin[2]) / g->cell[2]);
  x = umin32(x, g->dim[0] - 1);
  y = umin32(y, g->dim[1] - 1);
  z = umin32(z, g->dim[2] - 1);
  return z * g->dim[0] * g->dim[1] + y * g->dim[0] + x;
}

/* normalize, kernels/vectors.cu:24-31. */
static inline void normalize3(const float* v, float* o) {
  float l = sqrtf(len2f(v[0], v[1], v[2]));
  if (l > 0) {
    o[0] = v[0] / l; o[1] = v[1] / l; o[2] = v[2] / l;
  } else {
    o[0] = v[0]; o[1] = v[1]; o[2] = v[2];
  }
}

static inline float dot3(const float* a, const float* b) {
  return fmaf(a[2], b[2], fmaf(a[0], b[0], a[1] * b[1]));
}

static inline void cross3(const float* a, const float* b, float* d) {
  d[0] = fmaf(a[1], b[2], -(a[2] * b[1]));
  d[1] = fmaf(a[2], b[0], -(a[0] * b[2]));
  d[2] = fmaf(a[0], b[1], -(a[1] * b[0]));
}

/* Moller-Trumbore ray/triangle test, kernels/tri_intersect.cu:14-56. */
static int intersect_tri(const float* orig, const float* dir, const float* v0, const float* v1,
                         const float* v2, float* t, float* u, float* v) {
  float e1[3] = {v1[0] - v0[0], v1[1] - v0[1], v1[2] - v0[2]};
  float e2[3] = {v2[0] - v0[0], v2[1] - v0[1], v2[2] - v0[2]};
  float pvec[3], qvec[3];
  cross3(dir, e2, pvec);
  float det = dot3(e1, pvec);
  if ((double)det > -ORC_TRI_EPSILON && (double)det < ORC_TRI_EPSILON) return 0;
  float inv_det = (float)(1.0 / (double)det);
  float tvec[3] = {orig[0] - v0[0], orig[1] - v0[1], orig[2] - v0[2]};
  *u = dot3(tvec, pvec) * inv_det;
  if (*u < 0.0f || *u > 1.0f) return 0;
  cross3(tvec, e1, qvec);
  *v = dot3(dir, qvec) * inv_det;
  if (*v < 0.0f || *u + *v > 1.0f) return 0;
  *t = dot3(e2, qvec) * inv_det;
  return 1;
}

/* CollideWithGeometry, kernels/dsmc_kernel.cu:1256-1314: first triangle of
 * the cell's list (in list order) hit within the step's path. */
static int collide_geom(const orc_geom* g, float* pos, float* vel, float* old, uint32_t cellid) {
  uint32_t st = g->start_end[2 * cellid], en = g->start_end[2 * cellid + 1];
  float dir[3];
  normalize3(vel, dir);
  float dx = pos[0] - old[0], dy = pos[1] - old[1], dz = pos[2] - old[2];
  float dist = sqrtf(len2f(dx, dy, dz));
  if (dist < ORC_EPS) return 0;
  for (uint32_t i = st; i < en; i++) {
    const uint32_t* id = g->tri_vidx + 3 * (size_t)i;
    const float* a = g->verts + 3 * (size_t)id[0];
    const float* b = g->verts + 3 * (size_t)id[1];
    const float* c = g->verts + 3 * (size_t)id[2];
    float t, u, v;
    if (intersect_tri(old, dir, a, b, c, &t, &u, &v)) {
      if (t >= 0 && t <= dist) {
        float uv = 1 - u - v;
        const float* nrm = g->normals + 3 * (size_t)i;
        float w[3] = {nrm[0] * ORC_MODEL_WIDTH, nrm[1] * ORC_MODEL_WIDTH, nrm[2] * ORC_MODEL_WIDTH};
        float p[3];
        for (int k = 0; k < 3; k++) p[k] = fmaf(c[k], v, fmaf(a[k], uv, b[k] * u));
        /* reflect4, kernels/vectors.cu:101-106 */
        float d = dot3(vel, nrm);
        for (int k = 0; k < 3; k++) vel[k] = fmaf(-(2 * d), nrm[k], vel[k]);
        float p1p[3];
        normalize3(vel, p1p);
        float od = dist - t;
        for (int k = 0; k < 3; k++) pos[k] = fmaf(p1p[k], od, p[k]);
        for (int k = 0; k < 3; k++) old[k] = p[k] + w[k];
        return 1;
      }
    }
  }
  return 0;
}

/* Periodic wrap: gmin + BOUNCE_DELTA + p - gmax evaluated in double. */
static inline float wrap_hi(float gmin, float p, float gmax) {
  return (float)((double)gmin + ORC_BOUNCE_DELTA + (double)p - (double)gmax);
}
static inline float wrap_lo(float gmax, float p, float gmin) {
  return (float)((double)gmax - ORC_BOUNCE_DELTA + (double)p - (double)gmin);
}
static inline float clamp_hi(float gmax) { return (float)((double)gmax - ORC_BOUNCE_DELTA); }
static inline float clamp_lo(float gmin) { return (float)((double)gmin + ORC_BOUNCE_DELTA); }

/* Periodic{X,Y,Z}BoundaryCondition and NoPeriodicBoundaryCondition,
 * kernels/dsmc_kernel.cu:1316-1555, with their order of face checks. */
static void apply_bc(const orc_sim* s, float* p, float* v) {
  const float* mn = s->gmin;
  const float* mx = s->gmax;
  switch (s->periodic) {
    case 'z':
      if (p[2] > mx[2]) p[2] = wrap_hi(mn[2], p[2], mx[2]);
      if (p[1] > mx[1]) { p[1] = clamp_hi(mx[1]); v[1] *= -1; }
      if (p[2] < mn[2]) p[2] = wrap_lo(mx[2], p[2], mn[2]);
      if (p[1] < mn[1]) { p[1] = clamp_lo(mn[1]); v[1] *= -1; }
      if (p[0] < mn[0]) { p[0] = clamp_lo(mn[0]); v[0] *= -1; }
      if (p[0] > mx[0]) { p[0] = clamp_hi(mx[0]); v[0] *= -1; }
      break;
    case 'x':
      if (p[0] > mx[0]) p[0] = wrap_hi(mn[0], p[0], mx[0]);
      if (p[1] > mx[1]) { p[1] = clamp_hi(mx[1]); v[1] *= -1; }
      if (p[0] < mn[0]) p[0] = wrap_lo(mx[0], p[0], mn[0]);
      if (p[1] < mn[1]) { p[1] = clamp_lo(mn[1]); v[1] *= -1; }
      if (p[2] < mn[2]) { p[2] = clamp_lo(mn[2]); v[2] *= -1; }
      if (p[2] > mx[2]) { p[2] = clamp_hi(mx[2]); v[2] *= -1; }
      break;
    case 'y':
      if (p[1] > mx[1]) p[1] = wrap_hi(mn[1], p[1], mx[1]);
      if (p[0] > mx[0]) { p[0] = clamp_hi(mx[0]); v[0] *= -1; }
      if (p[1] < mn[1]) p[1] = wrap_lo(mx[1], p[1], mn[1]);
      if (p[0] < mn[0]) { p[0] = clamp_lo(mn[0]); v[0] *= -1; }
      if (p[2] < mn[2]) { p[2] = clamp_lo(mn[2]); v[2] *= -1; }
      if (p[2] > mx[2]) { p[2] = clamp_hi(mx[2]); v[2] *= -1; }
      break;
    default:
      if (p[1] > mx[1]) { p[1] = clamp_hi(mx[1]); v[1] *= -1; }
      if (p[0] > mx[0]) { p[0] = clamp_hi(mx[0]); v[0] *= -1; }
      if (p[1] < mn[1]) { p[1] = clamp_lo(mn[1]); v[1] *= -1; }
      if (p[0] < mn[0]) { p[0] = clamp_lo(mn[0]); v[0] *= -1; }
      if (p[2] < mn[2]) { p[2] = clamp_lo(mn[2]); v[2] *= -1; }
      if (p[2] > mx[2]) { p[2] = clamp_hi(mx[2]); v[2] *= -1; }
      break;
  }
}

/* IntegrateDev (g == NULL) and ProcessCollisionsDev,
 * kernels/dsmc_kernel.cu:1557-1657. */
static void move_one(const orc_sim* s, const orc_geom* g, float* pos4, float* vel4, float dt) {
  float old[3] = {pos4[0], pos4[1], pos4[2]};
  float vel[3] = {vel4[0], vel4[1], vel4[2]};
  float p[3];
  for (int k = 0; k < 3; k++) p[k] = fmaf(vel[k], dt, old[k]);
  if (g) {
    uint32_t i = 0;
    int coll = 0;
    do {
      uint32_t stc = coll_cell_id(g, old);
      uint32_t enc = coll_cell_id(g, p);
      if (stc != ORC_NONE) {
        if (g->flags[stc] != 0) coll = collide_geom(g, p, vel, old, stc);
      }
      if (!coll && stc != enc && enc != ORC_NONE) {
        if (g->flags[enc] != 0) coll = collide_geom(g, p, vel, old, enc);
      }
    } while (coll && i++ < ORC_COLLISION_LIMIT);
  }
  apply_bc(s, p, vel);
  pos4[0] = p[0]; pos4[1] = p[1]; pos4[2] = p[2];
  vel4[0] = vel[0]; vel4[1] = vel[1]; vel4[2] = vel[2];
}

void orc_move(const orc_sim* s, const orc_geom* g, float* pos4, float* vel4, uint32_t n, float dt) {
  long i;
#pragma omp parallel for schedule(dynamic, 4096)
  for (i = 0; i < (long)n; i++) move_one(s, g, pos4 + 4 * i, vel4 + 4 * i, dt);
}

/* ------------------------------------------------------------- sample ---- */

/* SampleCellStatisticsDev, kernels/dsmc_kernel.cu:856-890 (FP32 statistics_t:
 * numInSample, xyzSum, velMag, padding = 7 floats). */
void orc_sample(const orc_sim* s, const float* vel4, const uint32_t* cse, float* cs7) {
  long c;
#pragma omp parallel for schedule(static)
  for (c = 0; c < (long)s->cells; c++) {
    uint32_t st = cse[2 * c], en = cse[2 * c + 1];
    if (en - st <= 0 || en <= st) continue;
    float* o = cs7 + 7 * c;
    for (uint32_t i = st; i < en; i++) {
      const float* v = vel4 + 4 * (size_t)i;
      o[0] += 1.0f;
      o[1] += v[0];
      o[2] += v[1];
      o[3] += v[2];
      o[4] += len2f(v[0], v[1], v[2]);
    }
  }
}

/* The same sums in FP64 (count, sum u, sum v, sum w, sum |v|^2), the product's
 * sampling accumulators. */
void orc_sample_f64(const orc_sim* s, const float* vel4, const uint32_t* cse, double* acc5) {
  long c;
#pragma omp parallel for schedule(static)
  for (c = 0; c < (long)s->cells; c++) {
    uint32_t st = cse[2 * c], en = cse[2 * c + 1];
    double* o = acc5 + 5 * c;
    for (uint32_t i = st; i < en; i++) {
      const float* v = vel4 + 4 * (size_t)i;
      double x = v[0], y = v[1], z = v[2];
      o[0] += 1.0;
      o[1] += x;
      o[2] += y;
      o[3] += z;
      o[4] += x * x + y * y + z * z;
    }
  }
}

/* --------------------------------------------------------------- step ---- */

void orc_step(const orc_sim* s, const orc_geom* g, float* pos4, float* old_pos4, float* vel4,
              float* old_vel4, uint32_t* keys, uint32_t* idx, uint32_t* cse, uint32_t n,
              float dt, float avg_conc, float* maxrem, float* stat4, uint32_t* seeds,
              int collide, int sample, float* cell_stats7) {
  orc_cell_ids(s, old_pos4, n, keys, idx);
  orc_sort(keys, idx, n, s->cells);
  orc_bounds_reorder(s, n, keys, idx, old_pos4, old_vel4, pos4, vel4, cse);
  if (collide) orc_collide(s, vel4, cse, maxrem, stat4, seeds, avg_conc, dt);
  orc_move(s, g, pos4, vel4, n, dt);
  if (sample) orc_sample(s, vel4, cse, cell_stats7);
}

/* ------------------------------------------------------------ geometry ---- */

/* Separating-axis triangle/box test (Akenine-Moller, "Fast 3D Triangle-Box
 * Overlap Testing", 2001): the box and triangle are disjoint iff their
 * projections are disjoint on one of 13 axes - the 3 box normals, the
 * triangle normal and the 9 cross products of box normals with triangle
 * edges.  All three vertices are projected on every axis. */
int orc_tri_box_overlap(const float center[3], const float half[3], const float tri[9]) {
  float v[3][3];
  for (int i = 0; i < 3; i++)
    for (int k = 0; k < 3; k++) v[i][k] = tri[3 * i + k] - center[k];
  float e[3][3];
  for (int k = 0; k < 3; k++) {
    e[0][k] = v[1][k] - v[0][k];
    e[1][k] = v[2][k] - v[1][k];
    e[2][k] = v[0][k] - v[2][k];
  }
  /* 9 edge axes: axis = unit_j x e_i. */
  for (int i = 0; i < 3; i++) {
    for (int j = 0; j < 3; j++) {
      float a[3] = {0, 0, 0};
      /* unit_j x e = (u_y e_z - u_z e_y, u_z e_x - u_x e_z, u_x e_y - u_y e_x) */
      if (j == 0) { a[1] = -e[i][2]; a[2] = e[i][1]; }
      if (j == 1) { a[0] = e[i][2]; a[2] = -e[i][0]; }
      if (j == 2) { a[0] = -e[i][1]; a[1] = e[i][0]; }
      float p0 = a[0] * v[0][0] + a[1] * v[0][1] + a[2] * v[0][2];
      float p1 = a[0] * v[1][0] + a[1] * v[1][1] + a[2] * v[1][2];
      float p2 = a[0] * v[2][0] + a[1] * v[2][1] + a[2] * v[2][2];
      float mn = p0, mx = p0;
      if (p1 < mn) mn = p1;
      if (p1 > mx) mx = p1;
      if (p2 < mn) mn = p2;
      if (p2 > mx) mx = p2;
      float r = half[0] * fabsf(a[0]) + half[1] * fabsf(a[1]) + half[2] * fabsf(a[2]);
      if (mn > r || mx < -r) return 0;
    }
  }
  /* 3 box normals: the triangle's bounding interval per axis. */
  for (int k = 0; k < 3; k++) {
    float mn = v[0][k], mx = v[0][k];
    for (int i = 1; i < 3; i++) {
      if (v[i][k] < mn) mn = v[i][k];
      if (v[i][k] > mx) mx = v[i][k];
    }
    if (mn > half[k] || mx < -half[k]) return 0;
  }
  /* Triangle plane: box centre (origin) distance vs box projection radius. */
  float nrm[3] = {e[0][1] * e[1][2] - e[0][2] * e[1][1], e[0][2] * e[1][0] - e[0][0] * e[1][2],
                  e[0][0] * e[1][1] - e[0][1] * e[1][0]};
  float dist = nrm[0] * v[0][0] + nrm[1] * v[0][1] + nrm[2] * v[0][2];
  float r = half[0] * fabsf(nrm[0]) + half[1] * fabsf(nrm[1]) + half[2] * fabsf(nrm[2]);
  if (dist > r || dist < -r) return 0;
  return 1;
}

/* Model::CreateGrid (src/model.cpp:733-769) over reg_grid_t::reset/getAABB
 * (src/reggrid.cpp:27-47,81-88) and AABB_t::from_bbox (include/aabb.h:70-78),
 * then encloseGrid (src/reggrid.cpp:49-79). */
long orc_build_grid(const float* verts, uint32_t nverts, const uint32_t* tris, uint32_t ntris,
                    const int dim[3], float bbox[6], float cell[3], uint32_t* count,
                    uint32_t* tri_ids, long cap, uint8_t* flags) {
  float mn[3] = {100000, 100000, 100000}, mx[3] = {-100000, -100000, -100000};
  for (uint32_t i = 0; i < nverts; i++)
    for (int k = 0; k < 3; k++) {
      float x = verts[3 * i + k];
      if (x < mn[k]) mn[k] = x;
      if (x > mx[k]) mx[k] = x;
    }
  const uint32_t dx = (uint32_t)dim[0], dy = (uint32_t)dim[1], dz = (uint32_t)dim[2];
  for (int k = 0; k < 3; k++) {
    cell[k] = (mx[k] - mn[k]) / (float)(uint32_t)dim[k];
    bbox[k] = mn[k];
    bbox[3 + k] = mx[k];
  }
  const uint32_t ncell = dx * dy * dz;
  memset(count, 0, (size_t)ncell * sizeof(uint32_t));
  memset(flags, 0, ncell);
  /* bin per cell, cells visited x-major like the reference; entries stored in
   * cell-index order afterwards */
  uint32_t** bins = (uint32_t**)calloc(ncell, sizeof(uint32_t*));
  uint32_t* caps = (uint32_t*)calloc(ncell, sizeof(uint32_t));
  long xi;
#pragma omp parallel for schedule(dynamic, 1)
  for (xi = 0; xi < (long)dx; xi++) {
    for (uint32_t y = 0; y < dy; y++)
      for (uint32_t z = 0; z < dz; z++) {
        float bmin[3] = {mn[0] + (float)xi * cell[0], mn[1] + (float)y * cell[1],
                         mn[2] + (float)z * cell[2]};
        float center[3], half[3];
        for (int k = 0; k < 3; k++) {
          float bmax = bmin[k] + cell[k];
          half[k] = (bmax - bmin[k]) / 2;
          center[k] = bmin[k] + half[k];
        }
        uint32_t c = dx * dy * z + dx * y + (uint32_t)xi;
        for (uint32_t t = 0; t < ntris; t++) {
          float tri[9];
          for (int q = 0; q < 3; q++)
            for (int k = 0; k < 3; k++) tri[3 * q + k] = verts[3 * (size_t)tris[3 * t + q] + k];
          if (orc_tri_box_overlap(center, half, tri)) {
            if (count[c] == caps[c]) {
              caps[c] = caps[c] ? 2 * caps[c] : 8;
              bins[c] = (uint32_t*)realloc(bins[c], caps[c] * sizeof(uint32_t));
            }
            bins[c][count[c]++] = t;
            flags[c] = 1;
          }
        }
      }
  }
  /* encloseGrid: along z, cells between a flagged cell and the next flagged
   * cell become flagged (interior of the body). */
  for (uint32_t x = 0; x < dx; x++)
    for (uint32_t y = 0; y < dy; y++) {
      int last_full = 0;
      uint32_t last_z = 0;
      for (uint32_t z = 0; z < dz; z++) {
        uint32_t c = dx * dy * z + dx * y + x;
        if (flags[c]) {
          if (!last_full) {
            last_z = z;
            last_full = 1;
          } else {
            while (last_z != z) {
              flags[dx * dy * last_z + dx * y + x] = 1;
              last_z++;
            }
            last_full = 0;
          }
        }
      }
    }
  long total = 0;
  for (uint32_t c = 0; c < ncell; c++) {
    for (uint32_t k = 0; k < count[c]; k++) {
      if (total < cap) tri_ids[total] = bins[c][k];
      total++;
    }
    free(bins[c]);
  }
  free(bins);
  free(caps);
  return total;
}
