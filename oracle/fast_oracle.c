/* CPU restatement of the timestep's extension mode (the mode the capsule
 * workload runs): Philox-4x32-10 random streams, NTC selections of distinct
 * pairs with the VHS cross-section, warp-collided dense cells, the nearest
 * wall crossing of a triangle mesh with diffuse re-emission, per-face domain
 * boundaries and flux-weighted inflow injection.
 *
 * TEST INFRASTRUCTURE ONLY.  The product (cudadsmc_b200/libdsmc_b200.so)
 * never links, loads or calls this file.  It is the checker the GPU parity
 * tests compare the CUDA kernels against.
 *
 * None of this has a counterpart in the reference (denglide/CudaDsmc), whose
 * step is HybridTaus, hard-sphere, first-hit specular and closed-box only.
 * What it shares with the reference is restated from there and cited:
 *   - the NTC pair count and acceptance (ComputeBirdCollisionsNoMTDev,
 *     kernels/dsmc_kernel.cu:912-1000);
 *   - the Moller-Trumbore ray/triangle test (kernels/tri_intersect.cu:14-56),
 *     here with a determinant threshold relative to the triangle's size;
 *   - GetCellID3D (kernels/dsmc_kernel.cu:1701-1710).
 * Published methods: Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11); the
 * VHS model and diffuse reflection with full accommodation, the NTC scheme
 * and the inflow flux of a drifting Maxwellian (Bird, Molecular Gas Dynamics
 * and the Direct Simulation of Gas Flows, 1994, ch. 4, 11, 12).
 *
 * Floating point: the device code of this mode writes every rounding step
 * explicitly (fmaf, single-rounded products and sums, IEEE division and
 * square root), so the restatement below evaluates the same steps and agrees
 * bit for bit, except where the device calls a function with an error bound
 * of its own:
 *   - the base-2 log and exponential of the VHS power law (hardware
 *     approximations, relative error about 1e-6; here log2/exp2 in double);
 *   - logf, sincosf, sincospif and cospif (here libm, and sin/cos of pi x in
 *     double).
 * These differ from the device by an ulp or two.  Every decision that such a
 * value takes (an acceptance test, a rejection step, a wall crossing) is
 * checked here against a relative margin, and the cell or particle is
 * reported as a near tie when it falls inside it: the tests exclude those by
 * that stated cause and require them to be rare.
 */
#include "dsmc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define FO_NONE 0xffffffffu
#define FO_PI 3.14159265358979323846
#define FO_PURPOSE_COLLIDE 0x636f6c6cu
#define FO_PURPOSE_PAIRS 0x70616972u
#define FO_PURPOSE_WALL 0x77616c6cu
#define FO_PURPOSE_INJECT 0x696e6a65u
#define FO_PURPOSE_HEAVY 0x68650000u

/* ------------------------------------------------------------- Philox ---- */

/* A stream: key, counter words 1..3 fixed, the block index in word 0; words
 * handed out four at a time (x, y, z, w of each block). */
typedef struct {
  uint32_t key[2];
  uint32_t c1, c2, c3;
  uint32_t block;
  uint32_t buf[4];
  int used;
} pstream;

static void ps_init(pstream* s, const uint32_t key[2], uint32_t a, uint32_t b, uint32_t c) {
  s->key[0] = key[0];
  s->key[1] = key[1];
  s->c1 = a;
  s->c2 = b;
  s->c3 = c;
  s->block = 0;
  s->used = 4;
}

static uint32_t ps_next(pstream* s) {
  if (s->used == 4) {
    const uint32_t ctr[4] = {s->block, s->c1, s->c2, s->c3};
    orc_philox4x32_10(ctr, s->key, s->buf);
    s->block++;
    s->used = 0;
  }
  return s->buf[s->used++];
}

/* uniform in (0, 1): 24 random bits, offset by half an ulp of 2^-24 */
static float ps_uniform(pstream* s) {
  return ((float)(ps_next(s) >> 8) + 0.5f) * (1.0f / 16777216.0f);
}

/* __umulhi(r, n): the high word of the 64-bit product */
static inline uint32_t umulhi(uint32_t a, uint32_t b) { return (uint32_t)(((uint64_t)a * b) >> 32); }

static inline int near_tie(float a, float b, float rel) {
  float m = fabsf(a) > fabsf(b) ? fabsf(a) : fabsf(b);
  return fabsf(a - b) <= rel * m;
}

/* sin(pi x), cos(pi x) correctly rounded to float (the device's sincospif
 * is within an ulp of these). */
static void sincospi_f(float x, float* s, float* c) {
  const double a = FO_PI * (double)x;
  *s = (float)sin(a);
  *c = (float)cos(a);
}

/* ------------------------------------------------------------ collide ---- */

/* sigma(g) g: hard sphere sigma g; VHS K 2^(c1 log2 g), each step rounded to
 * float as the device rounds it. */
static float sigma_g_fast(const orc_fast* f, float mag) {
  if (f->hard_sphere) return mag * f->cross_section;
  if (!(mag > 0.0f)) return 0.0f;
  const float l = (float)log2((double)mag);
  const float y = f->vhs_c1 * l;
  return f->vhs_k * (float)exp2((double)y);
}

static float rel_speed(const float* v1, const float* v2) {
  const float dx = v1[0] - v2[0], dy = v1[1] - v2[1], dz = v1[2] - v2[2];
  return sqrtf(fmaf(dz, dz, fmaf(dx, dx, dy * dy)));
}

/* Isotropic scattering of a pair (scatter_pair of the device code). */
static void scatter_pair(const float* v1, const float* v2, float mag, float r_cos, float r_phi,
                         float* o1, float* o2) {
  const float b = fmaf(2.0f, r_cos, -1.0f);
  float a = fmaf(-b, b, 1.0f);
  a = sqrtf(a > 0.0f ? a : 0.0f);
  float sn, cn;
  sincospi_f(2.0f * r_phi, &sn, &cn);
  const float h = 0.5f * mag;
  const float ah = a * h;
  const float ang[3] = {b * h, ah * cn, ah * sn};
  for (int k = 0; k < 3; k++) {
    const float cm = 0.5f * (v1[k] + v2[k]);
    o1[k] = cm + ang[k];
    o2[k] = cm - ang[k];
  }
}

typedef struct {
  float* u;
  float* v;
  float* w;
  uint32_t off;
} vel_view;

static void vget(const vel_view* a, uint32_t k, float* o) {
  o[0] = a->u[a->off + k];
  o[1] = a->v[a->off + k];
  o[2] = a->w[a->off + k];
}
static void vset(const vel_view* a, uint32_t k, const float* o) {
  a->u[a->off + k] = o[0];
  a->v[a->off + k] = o[1];
  a->w[a->off + k] = o[2];
}

/* The NTC pair count of a cell (ntc_pairs_fast): M = floor(coef n avg
 * (sigma g)max + remainder), the new remainder the fraction left. */
static uint32_t pairs_fast(const orc_fast* f, uint32_t n, float* vmx, float* rem) {
  const float avg = f->ntc_local ? (float)(n - 1u) : f->avg_conc;
  const float fpc = fmaf((f->ntc_coef * (float)n) * avg, *vmx, *rem);
  const uint32_t M = fpc > 0.0f ? (uint32_t)fpc : 0u;
  *rem = fpc - (float)M;
  return M;
}

/* The selections of one cell by one lane (ntc_select_fast): M pairs of
 * distinct particles drawn from the cell's pair stream, accepted when
 * sigma g > R (sigma g)max with R and the scattering angles from the cell's
 * collision stream, (sigma g)max raised as they come. */
static uint32_t select_lane(const orc_fast* f, uint32_t cell, uint32_t n, const vel_view* acc,
                            uint32_t M, float* vmx, double* sum_g, uint32_t* ties) {
  pstream r, q;
  ps_init(&r, f->key, cell, f->step, FO_PURPOSE_COLLIDE);
  ps_init(&q, f->key, cell, f->step, FO_PURPOSE_PAIRS);
  uint32_t ncol = 0;
  for (uint32_t i = 0; i < M; i++) {
    const uint32_t pi = umulhi(ps_next(&q), n);
    uint32_t pj = pi + 1u + umulhi(ps_next(&q), n - 1u);
    if (pj >= n) pj -= n;
    float v1[3], v2[3];
    vget(acc, pi, v1);
    vget(acc, pj, v2);
    const float mag = rel_speed(v1, v2);
    const float v = sigma_g_fast(f, mag);
    const float rhs = ps_uniform(&r) * *vmx;
    if (!f->hard_sphere && near_tie(v, rhs, f->tie_rel)) (*ties)++;
    if (v > rhs) {
      ncol++;
      *sum_g += mag;
      float o1[3], o2[3];
      const float rc = ps_uniform(&r), rp = ps_uniform(&r);
      scatter_pair(v1, v2, mag, rc, rp, o1, o2);
      vset(acc, pi, o1);
      vset(acc, pj, o2);
    }
    if (v > *vmx) *vmx = v;
  }
  return ncol;
}

/* The selections of one dense cell by a warp of 32 lanes
 * (ntc_select_heavy_warp).  Each lane has its own stream.  A round: the idle
 * lanes, in lane order, draw new pairs while pairs remain to be drawn; every
 * pending pair claims its two particles, the lowest lane winning each claim;
 * lanes that won both of their particles evaluate their pair against the
 * (sigma g)max of the round's start and collide it; the losers keep their
 * pair for the next round.  After the round (sigma g)max takes the largest
 * sigma g the winners saw.  Returns the collisions. */
static uint32_t select_warp(const orc_fast* f, uint32_t cell, uint32_t n, const vel_view* acc,
                            uint32_t M, float* vmx, double* sum_g, uint32_t* ties,
                            uint32_t* claim) {
  pstream rng[32];
  uint32_t pi[32], pj[32];
  int pend[32];
  for (int l = 0; l < 32; l++) {
    ps_init(&rng[l], f->key, cell, f->step, FO_PURPOSE_HEAVY + (uint32_t)l);
    pend[l] = 0;
    pi[l] = pj[l] = 0;
  }
  for (uint32_t k = 0; k < n; k++) claim[k] = FO_NONE;
  uint32_t drawn = 0, done = 0, ncol = 0;
  float vmax = *vmx;
  while (done < M) {
    uint32_t idle = 0;
    for (int l = 0; l < 32; l++) idle += pend[l] ? 0u : 1u;
    const uint32_t want = idle < M - drawn ? idle : M - drawn;
    uint32_t rank = 0;
    for (int l = 0; l < 32; l++) {
      if (pend[l]) continue;
      if (rank < want) {
        pi[l] = umulhi(ps_next(&rng[l]), n);
        uint32_t j = pi[l] + 1u + umulhi(ps_next(&rng[l]), n - 1u);
        if (j >= n) j -= n;
        pj[l] = j;
        pend[l] = 1;
      }
      rank++;
    }
    drawn += want;
    for (int l = 0; l < 32; l++) {
      if (!pend[l]) continue;
      if ((uint32_t)l < claim[pi[l]]) claim[pi[l]] = (uint32_t)l;
      if ((uint32_t)l < claim[pj[l]]) claim[pj[l]] = (uint32_t)l;
    }
    int win[32];
    for (int l = 0; l < 32; l++)
      win[l] = pend[l] && claim[pi[l]] == (uint32_t)l && claim[pj[l]] == (uint32_t)l;
    float mx = 0.0f;
    for (int l = 0; l < 32; l++) {
      if (!win[l]) continue;
      float v1[3], v2[3];
      vget(acc, pi[l], v1);
      vget(acc, pj[l], v2);
      const float mag = rel_speed(v1, v2);
      const float vv = sigma_g_fast(f, mag);
      const float rhs = ps_uniform(&rng[l]) * vmax;
      if (!f->hard_sphere && near_tie(vv, rhs, f->tie_rel)) (*ties)++;
      if (vv > rhs) {
        ncol++;
        *sum_g += mag;
        float o1[3], o2[3];
        const float rc = ps_uniform(&rng[l]), rp = ps_uniform(&rng[l]);
        scatter_pair(v1, v2, mag, rc, rp, o1, o2);
        vset(acc, pi[l], o1);
        vset(acc, pj[l], o2);
      }
      if (vv > mx) mx = vv;
    }
    for (int l = 0; l < 32; l++) {
      if (!pend[l]) continue;
      claim[pi[l]] = FO_NONE;
      claim[pj[l]] = FO_NONE;
    }
    for (int l = 0; l < 32; l++)
      if (win[l]) {
        pend[l] = 0;
        done++;
      }
    if (mx > vmax) vmax = mx;
  }
  *vmx = vmax;
  return ncol;
}

void orc_collide_fast(const orc_fast* f, float* u, float* v, float* w, const uint32_t* start,
                      uint32_t ncells, float* maxrem, uint32_t* cell_info, double* sum_g_out) {
  double sum_g_all = 0.0;
  long c;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : sum_g_all)
  for (c = 0; c < (long)ncells; c++) {
    const uint32_t s = start[c], n = start[c + 1] - start[c];
    uint32_t* info = cell_info ? cell_info + 4 * (size_t)c : NULL;
    if (info) memset(info, 0, 16);
    if (n < 2) continue;
    float vmx = maxrem[2 * c], rem = maxrem[2 * c + 1];
    const uint32_t M = pairs_fast(f, n, &vmx, &rem);
    vel_view acc = {u, v, w, s};
    uint32_t ties = 0, ncol = 0, path = 0;
    double sg = 0.0;
    if (M > 0) {
      if (M >= f->heavy_min && n <= f->warp_cap) {
        uint32_t* claim = (uint32_t*)malloc((size_t)n * sizeof(uint32_t));
        ncol = select_warp(f, (uint32_t)c, n, &acc, M, &vmx, &sg, &ties, claim);
        free(claim);
        path = 2;
      } else {
        ncol = select_lane(f, (uint32_t)c, n, &acc, M, &vmx, &sg, &ties);
        path = n > f->warp_cap ? 3u : 1u;
      }
    }
    maxrem[2 * c] = vmx;
    maxrem[2 * c + 1] = rem;
    sum_g_all += sg;
    if (info) {
      info[0] = M;
      info[1] = ncol;
      info[2] = path;
      info[3] = ties;
    }
  }
  if (sum_g_out) *sum_g_out = sum_g_all;
}

/* --------------------------------------------------------------- move ---- */

static inline float dot_x(const float* a, const float* b) {
  return fmaf(a[2], b[2], fmaf(a[0], b[0], a[1] * b[1]));
}
static inline void cross_x(const float* a, const float* b, float* d) {
  d[0] = fmaf(a[1], b[2], -(a[2] * b[1]));
  d[1] = fmaf(a[2], b[0], -(a[0] * b[2]));
  d[2] = fmaf(a[0], b[1], -(a[1] * b[0]));
}

/* Ray/triangle test with the determinant threshold relative to the
 * triangle's size (intersect_triangle_rel); also returns the barycentric u, v
 * for the near-edge check. */
static int tri_hit(const float* o, const float* d, const float* a, const float* b, const float* c,
                   float* t, float* uo, float* vo) {
  const float e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  const float e2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
  float pv[3], qv[3];
  cross_x(d, e2, pv);
  const float det = dot_x(e1, pv);
  const float scale = dot_x(e1, e1) + dot_x(e2, e2);
  if (fabsf(det) <= 1e-9f * scale) return 0;
  const float inv = 1.0f / det;
  const float tv[3] = {o[0] - a[0], o[1] - a[1], o[2] - a[2]};
  const float u = dot_x(tv, pv) * inv;
  if (u < 0.0f || u > 1.0f) return 0;
  cross_x(tv, e1, qv);
  const float v = dot_x(d, qv) * inv;
  if (v < 0.0f || u + v > 1.0f) return 0;
  *t = dot_x(e2, qv) * inv;
  *uo = u;
  *vo = v;
  return 1;
}

/* The nearest triangle crossed by o + s d, s in [0, dist], over every
 * triangle of the mesh (the device walks the uniform grid's cells along the
 * path and tests the triangles binned there: the same set of crossings).
 * The plane pre-test of the device is applied as it is written there, so the
 * candidate triangles are the same.  *amb: the crossing is within the margin
 * of another crossing, of a triangle edge or of an end of the path. */
static int nearest_hit(const orc_fast_move* m, const float* o, const float* d, float dist,
                       float* t_out, uint32_t* tri_out, int* amb) {
  float best = 3.0e38f, second = 3.0e38f, bu = 0.5f, bv = 0.25f;
  uint32_t bi = FO_NONE;
  for (uint32_t i = 0; i < m->ntris; i++) {
    const float* P = m->plane + 4 * (size_t)i;
    const float s0 = dot_x(P, o) - P[3];
    const float s1 = fmaf(dist, dot_x(P, d), s0);
    const float tol = 1e-7f * (fabsf(P[3]) + 1.0f);
    if ((s0 > tol && s1 > tol) || (s0 < -tol && s1 < -tol)) continue;
    const float* T = m->tri + 9 * (size_t)i;
    float t, u, v;
    if (tri_hit(o, d, T, T + 3, T + 6, &t, &u, &v) && t >= 0.0f && t <= dist) {
      if (t < best) {
        second = best;
        best = t;
        bi = i;
        bu = u;
        bv = v;
      } else if (t < second) {
        second = t;
      }
    }
  }
  if (bi == FO_NONE) return 0;
  const float mg = m->amb_rel * (dist > 1e-30f ? dist : 1e-30f);
  const float em = m->amb_rel * 10.0f;
  if (second - best <= mg || best <= mg || dist - best <= mg || bu <= em || bv <= em ||
      bu + bv >= 1.0f - em)
    *amb = 1;
  *t_out = best;
  *tri_out = bi;
  return 1;
}

/* Diffuse re-emission (diffuse_emit_r): normal speed from the flux-weighted
 * half-range Maxwellian, tangential components Gaussian, about n_out. */
static void diffuse_emit(const float* n, float vstd, pstream* r, float* vel) {
  const float r1 = ps_uniform(r), r2 = ps_uniform(r), r3 = ps_uniform(r);
  const float vn = vstd * sqrtf(-2.0f * logf(r1));
  const float rad = vstd * sqrtf(-2.0f * logf(r2));
  const float ang = 6.2831853f * r3;
  const float s = sinf(ang), c = cosf(ang);
  const float t1 = rad * c, t2 = rad * s;
  const float a[3] = {fabsf(n[0]) < 0.9f ? 1.0f : 0.0f, fabsf(n[0]) < 0.9f ? 0.0f : 1.0f, 0.0f};
  float q[3], e1[3], e2[3];
  cross_x(a, n, q);
  const float ql = sqrtf(dot_x(q, q));
  for (int k = 0; k < 3; k++) e1[k] = ql > 0.0f ? q[k] / ql : q[k];
  cross_x(n, e1, e2);
  for (int k = 0; k < 3; k++) vel[k] = fmaf(t2, e2[k], fmaf(t1, e1[k], vn * n[k]));
}

/* One face axis of the per-face boundaries (face_axis). 0: left the domain. */
static int face_axis(const orc_fast_move* m, int axis, float* pos, float* vel, pstream* r) {
  const float lo = m->gmin[axis], hi = m->gmax[axis];
  float* x = &pos[axis];
  int face = -1;
  float bound = 0.0f;
  if (*x < lo) {
    face = 2 * axis;
    bound = lo;
  } else if (*x > hi) {
    face = 2 * axis + 1;
    bound = hi;
  }
  if (face < 0) return 1;
  const int kind = m->face_kind[face];
  if (kind == 2 || kind == 4) return 0;
  if (kind == 3) {
    *x = (face & 1) ? *x - (hi - lo) : *x + (hi - lo);
    return 1;
  }
  if (kind == 0) {
    *x = fmaf(2.0f, bound, -*x);
    vel[axis] = -vel[axis];
    return 1;
  }
  const float tau = vel[axis] != 0.0f ? (*x - bound) / vel[axis] : 0.0f;
  for (int k = 0; k < 3; k++) pos[k] = fmaf(-vel[k], tau, pos[k]);
  float n_in[3] = {0.0f, 0.0f, 0.0f};
  pos[axis] = bound;
  n_in[axis] = (face & 1) ? -1.0f : 1.0f;
  diffuse_emit(n_in, m->face_vstd[face], r, vel);
  for (int k = 0; k < 3; k++) pos[k] = fmaf(vel[k], tau, pos[k]);
  return 1;
}

static int face_bc(const orc_fast_move* m, float* pos, float* vel, pstream* r) {
  for (int a = 0; a < 3; a++)
    if (!face_axis(m, a, pos, vel, r)) return 0;
  for (int a = 0; a < 3; a++) {
    if (pos[a] < m->gmin[a]) pos[a] = m->gmin[a];
    if (pos[a] > m->gmax[a]) pos[a] = m->gmax[a];
  }
  return 1;
}

/* One particle's flight (move_particle_body, nearest mode, then face_bc):
 * free flight for dt; while the path crosses the body (at most 10 times), the
 * nearest crossing: a face reached from behind removes the particle (it was
 * inside the closed body), otherwise the particle is re-emitted (diffuse) or
 * reflected (specular) at the crossing, set off by 1e-6 m along the normal,
 * and flies the rest of the path length. */
static int move_one(const orc_fast_move* m, const float* mb, float* pos, float* vel, uint32_t gidx,
                    int* amb) {
  float old[3] = {pos[0], pos[1], pos[2]};
  for (int k = 0; k < 3; k++) pos[k] = fmaf(vel[k], m->dt, old[k]);
  pstream r;
  ps_init(&r, m->key, gidx, m->step, FO_PURPOSE_WALL);
  if (m->ntris) {
    for (int b = 0; b < 10; b++) {
      const float seg[3] = {pos[0] - old[0], pos[1] - old[1], pos[2] - old[2]};
      const float dist = sqrtf(fmaf(seg[2], seg[2], fmaf(seg[0], seg[0], seg[1] * seg[1])));
      if (!(dist > 1e-12f)) break;
      /* a path whose box misses the mesh's box (mb, widened by 1e-4 m)
       * crosses no triangle: skip the search (a shortcut of this
       * restatement only) */
      int off = 0;
      for (int k = 0; k < 3; k++) {
        const float lo = old[k] < pos[k] ? old[k] : pos[k];
        const float hi = old[k] < pos[k] ? pos[k] : old[k];
        if (hi < mb[k] - 1e-4f || lo > mb[3 + k] + 1e-4f) off = 1;
      }
      if (off) break;
      const float idist = 1.0f / dist;
      const float d[3] = {seg[0] * idist, seg[1] * idist, seg[2] * idist};
      float t;
      uint32_t ti;
      if (!nearest_hit(m, old, d, dist, &t, &ti, amb)) break;
      const float* n = m->plane + 4 * (size_t)ti;
      if (fmaf(d[2], n[2], fmaf(d[0], n[0], d[1] * n[1])) > 0.0f) return 0;
      float hp[3];
      for (int k = 0; k < 3; k++) hp[k] = fmaf(n[k], 1e-6f, fmaf(d[k], t, old[k]));
      const float rest = dist - t;
      if (m->wall_diffuse) {
        const float speed = sqrtf(fmaf(vel[2], vel[2], fmaf(vel[0], vel[0], vel[1] * vel[1])));
        diffuse_emit(n, m->wall_vstd, &r, vel);
        const float tau = speed > 0.0f ? rest / speed : 0.0f;
        for (int k = 0; k < 3; k++) pos[k] = fmaf(vel[k], tau, hp[k]);
      } else {
        const float vn2 = 2.0f * fmaf(vel[2], n[2], fmaf(vel[0], n[0], vel[1] * n[1]));
        for (int k = 0; k < 3; k++) vel[k] = fmaf(-vn2, n[k], vel[k]);
        const float sp = sqrtf(fmaf(vel[2], vel[2], fmaf(vel[0], vel[0], vel[1] * vel[1])));
        float rr[3];
        for (int k = 0; k < 3; k++) rr[k] = sp > 0.0f ? vel[k] / sp : vel[k];
        for (int k = 0; k < 3; k++) pos[k] = fmaf(rr[k], rest, hp[k]);
      }
      for (int k = 0; k < 3; k++) old[k] = hp[k];
    }
  }
  return face_bc(m, pos, vel, &r);
}

void orc_move_fast(const orc_fast_move* m, float* x, float* y, float* z, float* u, float* v,
                   float* w, uint32_t n, uint32_t gidx0, uint8_t* live, uint8_t* amb) {
  float mb[6] = {3.0e38f, 3.0e38f, 3.0e38f, -3.0e38f, -3.0e38f, -3.0e38f};
  for (size_t q = 0; q < 3 * (size_t)m->ntris; q++) {
    const float* vx = m->tri + 3 * q;
    for (int k = 0; k < 3; k++) {
      if (vx[k] < mb[k]) mb[k] = vx[k];
      if (vx[k] > mb[3 + k]) mb[3 + k] = vx[k];
    }
  }
  long i;
#pragma omp parallel for schedule(dynamic, 256)
  for (i = 0; i < (long)n; i++) {
    float pos[3] = {x[i], y[i], z[i]}, vel[3] = {u[i], v[i], w[i]};
    int a = 0;
    const int l = move_one(m, mb, pos, vel, gidx0 + (uint32_t)i, &a);
    x[i] = pos[0]; y[i] = pos[1]; z[i] = pos[2];
    u[i] = vel[0]; v[i] = vel[1]; w[i] = vel[2];
    if (live) live[i] = (uint8_t)l;
    if (amb) amb[i] = (uint8_t)a;
  }
}

/* Planes of the triangles as the library's mesh upload computes them: the
 * unit normal of (v1 - v0) x (v2 - v0) in double, the offset n . v0, both
 * rounded to float. */
void orc_tri_planes(const float* tri9, uint32_t ntris, float* plane4) {
  for (uint32_t i = 0; i < ntris; i++) {
    const float* a = tri9 + 9 * (size_t)i;
    const float* b = a + 3;
    const float* c = a + 6;
    double e1[3] = {(double)b[0] - a[0], (double)b[1] - a[1], (double)b[2] - a[2]};
    double e2[3] = {(double)c[0] - a[0], (double)c[1] - a[1], (double)c[2] - a[2]};
    double pn[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                    e1[0] * e2[1] - e1[1] * e2[0]};
    double l = sqrt(pn[0] * pn[0] + pn[1] * pn[1] + pn[2] * pn[2]);
    if (l > 0) {
      pn[0] /= l;
      pn[1] /= l;
      pn[2] /= l;
    }
    plane4[4 * (size_t)i] = (float)pn[0];
    plane4[4 * (size_t)i + 1] = (float)pn[1];
    plane4[4 * (size_t)i + 2] = (float)pn[2];
    plane4[4 * (size_t)i + 3] = (float)(pn[0] * a[0] + pn[1] * a[1] + pn[2] * a[2]);
  }
}

/* ------------------------------------------------------------- inflow ---- */

/* Inward normal speed / c_mp of the flux-weighted drifting Maxwellian,
 * f(z) ~ z exp(-(z - s)^2), z > 0, by rejection from the envelope
 * (|y| + max(s, 0)) exp(-y^2), y = z - s (sample_flux_normal). */
static float flux_normal(float s, pstream* r, int* amb, float rel) {
  const float sp = s > 0.0f ? s : 0.0f;
  const float w_abs = 1.0f / fmaf(sp, 1.7724539f, 1.0f);
  for (int it = 0; it < 64; it++) {
    float y;
    if (ps_uniform(r) < w_abs) {
      y = sqrtf(-logf(ps_uniform(r)));
      if (ps_uniform(r) < 0.5f) y = -y;
    } else {
      const float a = ps_uniform(r), b = ps_uniform(r);
      float sn, cn;
      sincospi_f(2.0f * b, &sn, &cn);
      y = sqrtf(-logf(a)) * cn;
    }
    const float z = s + y;
    if (fabsf(z) <= rel * (fabsf(s) + fabsf(y))) *amb = 1;
    if (z <= 0.0f) continue;
    const float lhs = ps_uniform(r) * (fabsf(y) + sp);
    if (near_tie(lhs, z, rel)) *amb = 1;
    if (lhs <= z) return z;
  }
  return s > 1e-3f ? s : 1e-3f;
}

/* k_inject_plan: the particles the face injects this step, the fraction
 * carried to the next. */
uint32_t orc_inject_plan(const orc_inflow* in, float dt, float* remainder, uint32_t max_k) {
  const float want = fmaf(in->number_flux * in->area, dt, *remainder);
  uint32_t k = want > 0.0f ? (uint32_t)want : 0u;
  if (k > max_k) k = max_k;
  *remainder = want - (float)k;
  return k;
}

uint32_t orc_inject_fast(const orc_inflow* in, const float gmin[3], const float gmax[3], float dt,
                         const uint32_t key[2], uint32_t step, float* remainder, uint32_t max_k,
                         float* x, float* y, float* z, float* u, float* v, float* w, uint8_t* amb,
                         float tie_rel) {
  const uint32_t k = orc_inject_plan(in, dt, remainder, max_k);
  /* k_inject_fill */
  /* k_inject_fill */
  const int face = in->face, ax = face >> 1;
  const float sign = (face & 1) ? -1.0f : 1.0f;
  const float cmp = in->vstd * 1.41421356f;
  const float s = sign * in->stream[ax] / cmp;
  long i;
#pragma omp parallel for schedule(static)
  for (i = 0; i < (long)k; i++) {
    pstream r;
    ps_init(&r, key, (uint32_t)i, step, FO_PURPOSE_INJECT + (uint32_t)face);
    int a = 0;
    const float vn = (flux_normal(s, &r, &a, tie_rel) * cmp) * sign;
    const float a1 = ps_uniform(&r), a2 = ps_uniform(&r);
    const float rad = in->vstd * sqrtf(-2.0f * logf(a1));
    float sn, cs;
    sincospi_f(2.0f * a2, &sn, &cs);
    const int t1 = (ax + 1) % 3, t2 = (ax + 2) % 3;
    float pos[3], vel[3];
    vel[ax] = vn;
    vel[t1] = fmaf(rad, cs, in->stream[t1]);
    vel[t2] = fmaf(rad, sn, in->stream[t2]);
    pos[ax] = (face & 1) ? gmax[ax] : gmin[ax];
    pos[t1] = fmaf(ps_uniform(&r), gmax[t1] - gmin[t1], gmin[t1]);
    pos[t2] = fmaf(ps_uniform(&r), gmax[t2] - gmin[t2], gmin[t2]);
    const float frac = ps_uniform(&r) * dt;
    for (int q = 0; q < 3; q++) pos[q] = fmaf(vel[q], frac, pos[q]);
    x[i] = pos[0]; y[i] = pos[1]; z[i] = pos[2];
    u[i] = vel[0]; v[i] = vel[1]; w[i] = vel[2];
    if (amb) amb[i] = (uint8_t)a;
  }
  return k;
}
