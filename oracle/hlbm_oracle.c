/*
 * hlbm_oracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY) for the D3Q19 hippoLBM step.
 *
 * A plain-C restatement of the reference algorithm on one rank.  Layout and
 * traversal follow the reference exactly so that every population, including the
 * ghost layers, can be compared bit for bit with the reference functors:
 *   - local box = global nodes + 2 ghost layers per side (make_domain.hpp:174-178),
 *     linear index idx = (z * Ly + y) * Lx + x, x fastest (box3d.hpp:112-117);
 *   - SoA populations f[c * ncell + idx] (field_view.hpp:56);
 *   - ext box drops the ghosts of non-periodic faces (make_domain.hpp:181-188).
 * Floating-point expressions keep the reference's evaluation order; build with
 * -ffp-contract=off.  Loops carry OpenMP static schedules, the reference's
 * Onika parallel_for semantics (parallel_for_core.hpp:80-94).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this file.
 */
#include "hlbm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define Q 19
#define FLUID (-1)
#define WALL (-2)

/* D3Q19 directions, scheme.hpp:47-69: odd i and i+1 are opposites. */
static const int EX[Q] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
static const int EY[Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
static const int EZ[Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
static const int WDEN[Q] = {3, 18, 18, 18, 18, 18, 18, 36, 36, 36, 36, 36, 36, 36, 36, 36, 36, 36, 36};
static inline int opp(int i) { return i == 0 ? 0 : ((i & 1) ? i + 1 : i - 1); }
static double W[Q];

/* plane bounce-back tables, bounce_back.hpp:65-140 (pre = saved, post = restored) */
static const int PRE_IDS[6][5] = {{2, 10, 8, 12, 14}, {1, 9, 7, 11, 13}, {4, 8, 9, 16, 18},
                                  {3, 7, 10, 15, 17}, {6, 13, 12, 17, 16}, {5, 14, 11, 18, 15}};
static const int POST_IDS[6][5] = {{1, 9, 7, 11, 13}, {2, 10, 8, 12, 14}, {3, 7, 10, 15, 17},
                                   {4, 8, 9, 16, 18}, {5, 14, 11, 18, 15}, {6, 13, 12, 17, 16}};
/* cavity coefficient directions, cavity.hpp:38-39 (always the DIMZ table) */
static const int CAVITY_IDS[2][5] = {{5, 14, 11, 18, 15}, {6, 13, 12, 17, 16}};

enum { OBS_NONE = -1, OBS_BALL = 0, OBS_WALL = 1, OBS_QUADRIC = 2 };
typedef struct {
  int type;
  double a[16];
} orc_obstacle;

typedef struct {
  int n[3];  /* global nodes per axis = cell_dims + 1 */
  int L[3];  /* local box lengths = n + 4 */
  int periodic[3];
  int ext_lo[3], ext_hi[3];
  double dx;
  double origin[3];
  int64_t ncell;
  double* f;
  double* m0;
  double* m1;
  int32_t* obst;
  int32_t* level;
  int64_t nplane[6];
  int32_t* plane[6];
  double* fi[6]; /* 5 * nplane values, only for non-periodic faces */
  /* LBMParameters (lbm_parameters.hpp:41-57) */
  double Fext[3], celerity, dtLB, nuth, nu, tau, avg_rho;
  int nobs;
  orc_obstacle* obs;
  double* fs; /* streamed populations, for zero_gradient */
} orc_lattice;

static inline int64_t IDX(const orc_lattice* g, int x, int y, int z) {
  return ((int64_t)z * g->L[1] + y) * g->L[0] + x;
}

static void init_weights(void) {
  for (int i = 0; i < Q; i++) W[i] = 1.0 / WDEN[i];
}

/* ---------------------------------------------------------------- domain */
void* orc_create(const int32_t cell_dims[3], const double bmin[3], const double bmax[3],
                 const int32_t periodic[3], int32_t* err) {
  init_weights();
  *err = 0;
  int n[3];
  for (int d = 0; d < 3; d++) n[d] = cell_dims[d] + 1; /* domain_lbm.cpp:68 */
  double reso[3];
  for (int d = 0; d < 3; d++) reso[d] = (bmax[d] - bmin[d]) / (double)(n[d] - 1);
  if (reso[0] != reso[1] || reso[0] != reso[2]) { /* domain_lbm.cpp:81-86 */
    *err = -2;
    return NULL;
  }
  for (int d = 0; d < 3; d++) /* domain_lbm.cpp:90-106 */
    if (bmin[d] + (n[d] - 1) * reso[0] != bmax[d]) {
      *err = -3;
      return NULL;
    }
  orc_lattice* g = (orc_lattice*)calloc(1, sizeof(orc_lattice));
  /* load_balancing, one rank: GridDx from x (make_domain.hpp:280) */
  g->dx = (bmax[0] - bmin[0]) / (double)(n[0] - 1);
  for (int d = 0; d < 3; d++) {
    g->n[d] = n[d];
    g->L[d] = n[d] + 4;
    g->periodic[d] = periodic[d] ? 1 : 0;
    g->origin[d] = bmin[d];
    g->ext_lo[d] = 0;
    g->ext_hi[d] = g->L[d] - 1;
    if (!g->periodic[d]) { /* make_domain.hpp:181-188 */
      g->ext_lo[d] += 2;
      g->ext_hi[d] -= 2;
    }
  }
  g->ncell = (int64_t)g->L[0] * g->L[1] * g->L[2];
  g->f = (double*)calloc((size_t)g->ncell * Q, sizeof(double));
  g->m0 = (double*)calloc((size_t)g->ncell, sizeof(double));
  g->m1 = (double*)calloc((size_t)g->ncell * 3, sizeof(double));
  g->obst = (int32_t*)malloc((size_t)g->ncell * sizeof(int32_t));
  g->level = (int32_t*)malloc((size_t)g->ncell * sizeof(int32_t));
  /* build_traversal levels (grid_region.hpp:107-132) */
  for (int z = 0; z < g->L[2]; z++)
    for (int y = 0; y < g->L[1]; y++)
      for (int x = 0; x < g->L[0]; x++) {
        int c[3] = {x, y, z};
        int in_ext = 1, in_real = 1, in_inside = 1;
        for (int d = 0; d < 3; d++) {
          if (c[d] < g->ext_lo[d] || c[d] > g->ext_hi[d]) in_ext = 0;
          if (c[d] < 2 || c[d] > g->L[d] - 3) in_real = 0;
          if (c[d] < 3 || c[d] > g->L[d] - 4) in_inside = 0;
        }
        int lv = 3;
        if (in_ext) {
          lv = 2;
          if (in_real) {
            lv = 1;
            if (in_inside) lv = 0;
          }
        }
        g->level[IDX(g, x, y, z)] = lv;
      }
  /* plane lists (grid_region.hpp:141-193): one rank owns every face */
  int Lx = g->L[0], Ly = g->L[1], Lz = g->L[2];
  g->nplane[ORC_X0] = g->nplane[ORC_XL] = (int64_t)Ly * Lz;
  g->nplane[ORC_Y0] = g->nplane[ORC_YL] = (int64_t)Lx * Lz;
  g->nplane[ORC_Z0] = g->nplane[ORC_ZL] = (int64_t)Lx * Ly;
  for (int p = 0; p < 6; p++) g->plane[p] = (int32_t*)malloc((size_t)g->nplane[p] * sizeof(int32_t));
  int64_t k = 0;
  for (int y = 0; y < Ly; y++)
    for (int x = 0; x < Lx; x++, k++) {
      g->plane[ORC_Z0][k] = (int32_t)IDX(g, x, y, 2);
      g->plane[ORC_ZL][k] = (int32_t)IDX(g, x, y, Lz - 3);
    }
  k = 0;
  for (int z = 0; z < Lz; z++)
    for (int x = 0; x < Lx; x++, k++) {
      g->plane[ORC_Y0][k] = (int32_t)IDX(g, x, 2, z);
      g->plane[ORC_YL][k] = (int32_t)IDX(g, x, Ly - 3, z);
    }
  k = 0;
  for (int z = 0; z < Lz; z++)
    for (int y = 0; y < Ly; y++, k++) {
      g->plane[ORC_X0][k] = (int32_t)IDX(g, 2, y, z);
      g->plane[ORC_XL][k] = (int32_t)IDX(g, Lx - 3, y, z);
    }
  /* bounce_back_manager::resize_data (bounce_back_manager.hpp:98-117): non-periodic faces */
  for (int p = 0; p < 6; p++)
    g->fi[p] = g->periodic[p / 2] ? NULL : (double*)calloc((size_t)g->nplane[p] * 5, sizeof(double));
  /* init_obst: every flag FLUIDE_ (init_obst.hpp:29-32) */
  for (int64_t i = 0; i < g->ncell; i++) g->obst[i] = FLUID;
  /* default set_distribution (config_initialize.msp:22-23): value 1 over All */
  orc_set_distribution(g, 1.0, NULL, 0);
  /* default lbm_parameters slots (lbm_parameters.cpp:57-64) */
  double F0[3] = {0, 0, 0};
  orc_lbm_parameters(g, F0, 1.0, 1e-4, 1000.0, 0, 0.0, 0.0);
  return g;
}

void orc_destroy(void* h) {
  orc_lattice* g = (orc_lattice*)h;
  if (!g) return;
  free(g->f);
  free(g->m0);
  free(g->m1);
  free(g->obst);
  free(g->level);
  for (int p = 0; p < 6; p++) {
    free(g->plane[p]);
    free(g->fi[p]);
  }
  free(g->obs);
  free(g->fs);
  free(g);
}

/* ------------------------------------------------------------ parameters */
void orc_lbm_parameters(void* h, const double Fext[3], double celerity, double nuth, double avg_rho,
                        int32_t has_tau, double tau, double dt) {
  orc_lattice* g = (orc_lattice*)h;
  double dx = g->dx;
  g->nuth = nuth;
  g->avg_rho = avg_rho;
  if (dt > 0.0) { /* define_by_dt, lbm_parameters.hpp:60-66 */
    g->dtLB = dt;
    g->tau = 3 * g->nuth * g->dtLB / (dx * dx) + 0.5;
    g->nu = (g->tau - 0.5) / 3.0;
    g->celerity = dx / g->dtLB;
  } else if (has_tau) { /* define_by_tau, lbm_parameters.hpp:68-74 */
    g->tau = tau;
    g->dtLB = dx * dx * (g->tau - 0.5) / (3.0 * g->nuth);
    g->nu = g->nuth * g->dtLB / (dx * dx);
    g->celerity = dx / g->dtLB;
  } else { /* define_by_c, lbm_parameters.hpp:76-81 */
    g->celerity = celerity;
    g->dtLB = dx / g->celerity;
    g->nu = g->nuth * g->dtLB / (dx * dx);
    g->tau = 3. * g->nu + 0.5;
  }
  /* convert_force<LBM_UNITS> (lbm_parameters.hpp:124-128) */
  double ddx = g->celerity * g->dtLB;
  for (int d = 0; d < 3; d++) g->Fext[d] = Fext[d] * g->dtLB * g->dtLB / ddx;
}

void orc_get_parameters(void* h, double out[9]) {
  orc_lattice* g = (orc_lattice*)h;
  out[0] = g->Fext[0];
  out[1] = g->Fext[1];
  out[2] = g->Fext[2];
  out[3] = g->celerity;
  out[4] = g->dtLB;
  out[5] = g->nuth;
  out[6] = g->nu;
  out[7] = g->tau;
  out[8] = g->avg_rho;
}

/* --------------------------------------------------------- ghost update */
/* update_ghost on one rank: every ghost cell of the ext box receives all 19
 * populations of its periodic image in the real box (comm boxes of
 * operator_ghost_manager.hpp:56-114 with a self neighbour). */
static inline int wrap_axis(const orc_lattice* g, int d, int c) {
  int n = g->n[d];
  if (c < 2) return c + n;
  if (c > n + 1) return c - n;
  return c;
}

void orc_update_ghost(void* h) {
  orc_lattice* g = (orc_lattice*)h;
  int64_t nc = g->ncell;
#pragma omp parallel for schedule(static)
  for (int z = g->ext_lo[2]; z <= g->ext_hi[2]; z++)
    for (int y = g->ext_lo[1]; y <= g->ext_hi[1]; y++)
      for (int x = g->ext_lo[0]; x <= g->ext_hi[0]; x++) {
        int64_t idx = IDX(g, x, y, z);
        if (g->level[idx] != 2) continue;
        int64_t src = IDX(g, wrap_axis(g, 0, x), wrap_axis(g, 1, y), wrap_axis(g, 2, z));
        for (int c = 0; c < Q; c++) g->f[c * nc + idx] = g->f[c * nc + src];
      }
}

/* ------------------------------------------------------- set_distribution */
static void init_cell(orc_lattice* g, int64_t idx, double value) {
  for (int i = 0; i < Q; i++) g->f[i * g->ncell + idx] = value * W[i]; /* set_distribution.hpp:39-42 */
}

/* restrict_box_to_grid<Local, Extend> (grid.hpp:406-428) of the global box
 * {int(min / dx), int(max / dx)}; returns 0 if there is no intersection. */
static int clip_box(const orc_lattice* g, const double mn[3], const double mx[3], int lo[3], int hi[3]) {
  for (int d = 0; d < 3; d++) {
    lo[d] = (int)(mn[d] / g->dx) + 2;
    hi[d] = (int)(mx[d] / g->dx) + 2;
  }
  for (int d = 0; d < 3; d++)
    if (g->ext_hi[d] < lo[d] || hi[d] < g->ext_lo[d]) return 0;
  for (int d = 0; d < 3; d++) {
    if (lo[d] < g->ext_lo[d]) lo[d] = g->ext_lo[d];
    if (hi[d] > g->ext_hi[d]) hi[d] = g->ext_hi[d];
  }
  return 1;
}

void orc_set_distribution(void* h, double value, const double* bounds6, int32_t do_update) {
  orc_lattice* g = (orc_lattice*)h;
  if (bounds6) { /* set_distribution.cu:85-98 */
    int lo[3], hi[3];
    if (!clip_box(g, bounds6, bounds6 + 3, lo, hi)) return;
#pragma omp parallel for schedule(static)
    for (int z = lo[2]; z <= hi[2]; z++)
      for (int y = lo[1]; y <= hi[1]; y++)
        for (int x = lo[0]; x <= hi[0]; x++) init_cell(g, IDX(g, x, y, z), value);
  } else if (do_update) { /* set_distribution.cu:99-103 */
#pragma omp parallel for schedule(static)
    for (int64_t idx = 0; idx < g->ncell; idx++)
      if (g->level[idx] <= 1) init_cell(g, idx, value);
    orc_update_ghost(g);
  } else {
#pragma omp parallel for schedule(static)
    for (int64_t idx = 0; idx < g->ncell; idx++) init_cell(g, idx, value);
  }
}

/* ------------------------------------------------------------- obstacles */
void orc_init_obstacles(void* h) {
  orc_lattice* g = (orc_lattice*)h;
  free(g->obs);
  g->obs = NULL;
  g->nobs = 0;
}

static orc_obstacle* obstacle_slot(orc_lattice* g, int id) {
  if (id >= g->nobs) { /* obstacles.hpp:84-107: grow, holes stay UNDEFINED */
    g->obs = (orc_obstacle*)realloc(g->obs, sizeof(orc_obstacle) * (size_t)(id + 1));
    for (int i = g->nobs; i <= id; i++) g->obs[i].type = OBS_NONE;
    g->nobs = id + 1;
  }
  return &g->obs[id];
}

void orc_register_ball(void* h, int32_t id, const double center[3], double radius) {
  orc_obstacle* o = obstacle_slot((orc_lattice*)h, id);
  o->type = OBS_BALL;
  o->a[0] = center[0];
  o->a[1] = center[1];
  o->a[2] = center[2];
  o->a[3] = radius;
  o->a[4] = radius * radius; /* Ball::r2_, obstacle.hpp:41 */
}

void orc_register_wall(void* h, int32_t id, const double bmin[3], const double bmax[3]) {
  orc_obstacle* o = obstacle_slot((orc_lattice*)h, id);
  o->type = OBS_WALL;
  for (int d = 0; d < 3; d++) {
    o->a[d] = bmin[d];
    o->a[3 + d] = bmax[d];
  }
}

void orc_register_quadric(void* h, int32_t id, const double q[16]) {
  orc_obstacle* o = obstacle_slot((orc_lattice*)h, id);
  o->type = OBS_QUADRIC;
  memcpy(o->a, q, sizeof(double) * 16);
}

/* p^T Q p with p = (x, y, z, 1), row by row (Onika's quadric_eval is not in the
 * reference tree: this restatement is the oracle's own, parity unpinned). */
static inline double quadric_value(const double* q, const double p3[3]) {
  double p[4] = {p3[0], p3[1], p3[2], 1.0};
  double acc = 0.0;
  for (int i = 0; i < 4; i++) {
    double row = 0.0;
    for (int j = 0; j < 4; j++) row = row + q[i * 4 + j] * p[j];
    acc = acc + p[i] * row;
  }
  return acc;
}

static inline int obstacle_solid(const orc_obstacle* o, const double p[3]) {
  if (o->type == OBS_BALL) { /* Ball::solid, obstacle.hpp:59-62 */
    double rx = p[0] - o->a[0], ry = p[1] - o->a[1], rz = p[2] - o->a[2];
    return rx * rx + ry * ry + rz * rz <= o->a[4];
  }
  if (o->type == OBS_WALL) { /* intersect, obstacle.hpp:13-17: strict interior */
    return o->a[0] < p[0] && p[0] < o->a[3] && o->a[1] < p[1] && p[1] < o->a[4] && o->a[2] < p[2] &&
           p[2] < o->a[5];
  }
  if (o->type == OBS_QUADRIC) return quadric_value(o->a, p) <= 0.0; /* obstacle.hpp:134-136 */
  return 0;
}

void orc_update_obstacles(void* h) {
  orc_lattice* g = (orc_lattice*)h;
  for (int i = 0; i < g->nobs; i++) { /* UpdateObstacles::execute, update_obstacles.cu:106-119 */
    const orc_obstacle* o = &g->obs[i];
    if (o->type == OBS_NONE) continue;
    double mn[3], mx[3];
    if (o->type == OBS_BALL) { /* Ball::covered, obstacle.hpp:46-49 */
      for (int d = 0; d < 3; d++) {
        mn[d] = o->a[d] - o->a[3];
        mx[d] = o->a[d] + o->a[3];
      }
    } else if (o->type == OBS_WALL) {
      for (int d = 0; d < 3; d++) {
        mn[d] = o->a[d];
        mx[d] = o->a[3 + d];
      }
    } else { /* Quadric::covered, obstacle.hpp:120-124 */
      for (int d = 0; d < 3; d++) {
        mn[d] = -1e6;
        mx[d] = 1e6;
      }
    }
    int lo[3], hi[3];
    if (!clip_box(g, mn, mx, lo, hi)) continue; /* update_obstacles.cu:58-67 */
#pragma omp parallel for schedule(static)
    for (int z = lo[2]; z <= hi[2]; z++)
      for (int y = lo[1]; y <= hi[1]; y++)
        for (int x = lo[0]; x <= hi[0]; x++) {
          /* compute_position<Global> (grid.hpp:355-361): (local + offset) * dx, no origin */
          double p[3] = {((double)x + (double)(-2)) * g->dx, ((double)y + (double)(-2)) * g->dx,
                         ((double)z + (double)(-2)) * g->dx};
          if (obstacle_solid(o, p)) g->obst[IDX(g, x, y, z)] = WALL;
        }
  }
}

/* -------------------------------------------------------- macro variables */
void orc_macro_variables(void* h) {
  orc_lattice* g = (orc_lattice*)h;
  const int64_t nc = g->ncell;
#pragma omp parallel for schedule(static)
  for (int64_t idx = 0; idx < nc; idx++) { /* macro_variables.hpp:48-79, over all_ */
    if (g->obst[idx] >= FLUID) {
      double rho = 0.0, ux = 0.0, uy = 0.0, uz = 0.0;
      for (int i = 0; i < Q; i++) {
        const double s = g->f[i * nc + idx];
        ux += s * EX[i];
        uy += s * EY[i];
        uz += s * EZ[i];
        rho += s;
      }
      if (rho > 1.0e-14) {
        ux /= rho;
        uy /= rho;
        uz /= rho;
      }
      g->m0[idx] = rho;
      g->m1[idx] = ux;
      g->m1[nc + idx] = uy;
      g->m1[2 * nc + idx] = uz;
    } else {
      g->m1[idx] = 0;
      g->m1[nc + idx] = 0;
      g->m1[2 * nc + idx] = 0;
    }
  }
}

/* ------------------------------------------------------------------- BGK */
void orc_bgk(void* h) {
  orc_lattice* g = (orc_lattice*)h;
  const int64_t nc = g->ncell;
  const double tau = g->tau, Fx = g->Fext[0], Fy = g->Fext[1], Fz = g->Fext[2];
#pragma omp parallel for schedule(static)
  for (int64_t idx = 0; idx < nc; idx++) { /* bgk.hpp:47-62, all cells masked to Real and fluid */
    const int update = (g->level[idx] <= 1) && (g->obst[idx] == FLUID);
    const double rho = g->m0[idx];
    const double ux = g->m1[idx], uy = g->m1[nc + idx], uz = g->m1[2 * nc + idx];
    const double u_squ = (ux * ux + uy * uy + uz * uz);
    for (int i = 0; i < Q; i++) {
      double* fp = &g->f[i * nc + idx];
      double ef = EX[i] * Fx + EY[i] * Fy + EZ[i] * Fz;
      double eu = EX[i] * ux + EY[i] * uy + EZ[i] * uz;
      double feq = W[i] * rho * (1. + 3. * eu + 4.5 * eu * eu - 1.5 * u_squ);
      *fp += update * ((feq - *fp) / tau + 3. * rho * W[i] * ef);
    }
  }
}

/* ------------------------------------------------------------------- MRT */
/* Moment rows of the d'Humieres D3Q19 basis in the order used by mrt.hpp:57-94.
 * Each moment is a sum over populations in increasing index, which is the
 * reference's term order, so adding coefficient * f term by term (skipping
 * zeros) reproduces its rounding. */
static const signed char MROW[19][19] = {
    /* rho  */ {1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1},
    /* e    */ {-30, -11, -11, -11, -11, -11, -11, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8},
    /* eps  */ {12, -4, -4, -4, -4, -4, -4, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1},
    /* jx   */ {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0},
    /* qx   */ {0, -4, 4, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0},
    /* jy   */ {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1},
    /* qy   */ {0, 0, 0, -4, 4, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1},
    /* jz   */ {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1},
    /* qz   */ {0, 0, 0, 0, 0, -4, 4, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1},
    /* pxx3 */ {0, 2, 2, -1, -1, -1, -1, 1, 1, 1, 1, 1, 1, 1, 1, -2, -2, -2, -2},
    /* pixx3*/ {0, -4, -4, 2, 2, 2, 2, 1, 1, 1, 1, 1, 1, 1, 1, -2, -2, -2, -2},
    /* pww  */ {0, 0, 0, 1, 1, -1, -1, 1, 1, 1, 1, -1, -1, -1, -1, 0, 0, 0, 0},
    /* piww */ {0, 0, 0, -2, -2, 2, 2, 1, 1, 1, 1, -1, -1, -1, -1, 0, 0, 0, 0},
    /* pxy  */ {0, 0, 0, 0, 0, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 0, 0, 0, 0},
    /* pyz  */ {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, -1, -1},
    /* pxz  */ {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0},
    /* mx   */ {0, 0, 0, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, -1, 1, 0, 0, 0, 0},
    /* my   */ {0, 0, 0, 0, 0, 0, 0, -1, 1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1},
    /* mz   */ {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, -1, -1, 1, -1, 1, 1, -1}};

/* Back-transform (mrt.hpp:129-173): f_i = sum_k BNUM[i][k] / BDEN[k-column] * m_k with
 * the moments in MROW order.  Coefficients are numerator/denominator pairs,
 * evaluated as (double)num / den exactly as the reference's constant folding. */
typedef struct {
  signed char num;
  short den;
} frac;
#define F0_ {0, 1}
static const frac BACK[19][19] = {
    /* f0 */ {{1, 19}, {-5, 399}, {1, 21}, F0_, F0_, F0_, F0_, F0_, F0_, F0_, F0_, F0_, F0_, F0_, F0_, F0_, F0_, F0_, F0_},
    /* f1 */ {{1, 19}, {-11, 2394}, {-1, 63}, {1, 10}, {-1, 10}, F0_, F0_, F0_, F0_, {1, 18}, {-1, 18}, F0_, F0_, F0_, F0_, F0_, F0_, F0_, F0_},
    /* f2 */ {{1, 19}, {-11, 2394}, {-1, 63}, {-1, 10}, {1, 10}, F0_, F0_, F0_, F0_, {1, 18}, {-1, 18}, F0_, F0_, F0_, F0_, F0_, F0_, F0_, F0_},
    /* f3 */ {{1, 19}, {-11, 2394}, {-1, 63}, F0_, F0_, {1, 10}, {-1, 10}, F0_, F0_, {-1, 36}, {1, 36}, {1, 12}, {-1, 12}, F0_, F0_, F0_, F0_, F0_, F0_},
    /* f4 */ {{1, 19}, {-11, 2394}, {-1, 63}, F0_, F0_, {-1, 10}, {1, 10}, F0_, F0_, {-1, 36}, {1, 36}, {1, 12}, {-1, 12}, F0_, F0_, F0_, F0_, F0_, F0_},
    /* f5 */ {{1, 19}, {-11, 2394}, {-1, 63}, F0_, F0_, F0_, F0_, {1, 10}, {-1, 10}, {-1, 36}, {1, 36}, {-1, 12}, {1, 12}, F0_, F0_, F0_, F0_, F0_, F0_},
    /* f6 */ {{1, 19}, {-11, 2394}, {-1, 63}, F0_, F0_, F0_, F0_, {-1, 10}, {1, 10}, {-1, 36}, {1, 36}, {-1, 12}, {1, 12}, F0_, F0_, F0_, F0_, F0_, F0_},
    /* f7 */ {{1, 19}, {4, 1197}, {1, 252}, {1, 10}, {1, 40}, {1, 10}, {1, 40}, F0_, F0_, {1, 36}, {1, 72}, {1, 12}, {1, 24}, {1, 4}, F0_, F0_, {1, 8}, {-1, 8}, F0_},
    /* f8 */ {{1, 19}, {4, 1197}, {1, 252}, {-1, 10}, {-1, 40}, {-1, 10}, {-1, 40}, F0_, F0_, {1, 36}, {1, 72}, {1, 12}, {1, 24}, {1, 4}, F0_, F0_, {-1, 8}, {1, 8}, F0_},
    /* f9 */ {{1, 19}, {4, 1197}, {1, 252}, {1, 10}, {1, 40}, {-1, 10}, {-1, 40}, F0_, F0_, {1, 36}, {1, 72}, {1, 12}, {1, 24}, {-1, 4}, F0_, F0_, {1, 8}, {1, 8}, F0_},
    /* f10*/ {{1, 19}, {4, 1197}, {1, 252}, {-1, 10}, {-1, 40}, {1, 10}, {1, 40}, F0_, F0_, {1, 36}, {1, 72}, {1, 12}, {1, 24}, {-1, 4}, F0_, F0_, {-1, 8}, {-1, 8}, F0_},
    /* f11*/ {{1, 19}, {4, 1197}, {1, 252}, {1, 10}, {1, 40}, F0_, F0_, {1, 10}, {1, 40}, {1, 36}, {1, 72}, {-1, 12}, {-1, 24}, F0_, F0_, {1, 4}, {-1, 8}, F0_, {1, 8}},
    /* f12*/ {{1, 19}, {4, 1197}, {1, 252}, {-1, 10}, {-1, 40}, F0_, F0_, {-1, 10}, {-1, 40}, {1, 36}, {1, 72}, {-1, 12}, {-1, 24}, F0_, F0_, {1, 4}, {1, 8}, F0_, {-1, 8}},
    /* f13*/ {{1, 19}, {4, 1197}, {1, 252}, {1, 10}, {1, 40}, F0_, F0_, {-1, 10}, {-1, 40}, {1, 36}, {1, 72}, {-1, 12}, {-1, 24}, F0_, F0_, {-1, 4}, {-1, 8}, F0_, {-1, 8}},
    /* f14*/ {{1, 19}, {4, 1197}, {1, 252}, {-1, 10}, {-1, 40}, F0_, F0_, {1, 10}, {1, 40}, {1, 36}, {1, 72}, {-1, 12}, {-1, 24}, F0_, F0_, {-1, 4}, {1, 8}, F0_, {1, 8}},
    /* f15*/ {{1, 19}, {4, 1197}, {1, 252}, F0_, F0_, {1, 10}, {1, 40}, {1, 10}, {1, 40}, {-1, 18}, {-1, 36}, F0_, F0_, F0_, {1, 4}, F0_, F0_, {1, 8}, {-1, 8}},
    /* f16*/ {{1, 19}, {4, 1197}, {1, 252}, F0_, F0_, {-1, 10}, {-1, 40}, {-1, 10}, {-1, 40}, {-1, 18}, {-1, 36}, F0_, F0_, F0_, {1, 4}, F0_, F0_, {-1, 8}, {1, 8}},
    /* f17*/ {{1, 19}, {4, 1197}, {1, 252}, F0_, F0_, {1, 10}, {1, 40}, {-1, 10}, {-1, 40}, {-1, 18}, {-1, 36}, F0_, F0_, F0_, {-1, 4}, F0_, F0_, {1, 8}, {1, 8}},
    /* f18*/ {{1, 19}, {4, 1197}, {1, 252}, F0_, F0_, {-1, 10}, {-1, 40}, {1, 10}, {1, 40}, {-1, 18}, {-1, 36}, F0_, F0_, F0_, {-1, 4}, F0_, F0_, {-1, 8}, {-1, 8}}};

/* MRT rates: s_e, s_eps, s_q, s_pi, s_m, w_eps, w_epsj, w_xx; s_nu = 1/tau.
 * Reference constants: mrt.hpp:43-47. */
static void mrt_reference_rates(double r[8]) {
  r[0] = 1.19;
  r[1] = 1.4;
  r[2] = 1.2;
  r[3] = 1.4;
  r[4] = 1.98;
  r[5] = 0;
  r[6] = -475. / 63.;
  r[7] = 0;
}

static void mrt_cell(double* f, int64_t nc, int64_t idx, double tau, const double* r) {
  const double s9 = 1 / tau, s13 = s9;
  const double s1 = r[0], s2 = r[1], s4 = r[2], s10 = r[3], s16 = r[4];
  const double weps = r[5], wepsj = r[6], wxx = r[7];
  double fl[Q], m[19];
  for (int i = 0; i < Q; i++) fl[i] = f[i * nc + idx];
  /* both loops are unrolled whole, so the table entries are constants: zero terms vanish and
   * num / den folds to the same double the division gives at run time */
#pragma GCC unroll 19
  for (int k = 0; k < 19; k++) {
    double acc = 0.0;
    int first = 1;
#pragma GCC unroll 19
    for (int i = 0; i < Q; i++) {
      const int c = MROW[k][i];
      if (c == 0) continue;
      const double term = (c == 1) ? fl[i] : (c == -1 ? -fl[i] : (double)c * fl[i]);
      acc = first ? term : acc + term;
      first = 0;
    }
    m[k] = acc;
  }
  const double rho = m[0], e = m[1], eps = m[2], jx = m[3], qx = m[4], jy = m[5], qy = m[6], jz = m[7],
               qz = m[8], pxx3 = m[9], pixx3 = m[10], pww = m[11], piww = m[12], pxy = m[13], pyz = m[14],
               pxz = m[15], mx = m[16], my = m[17], mz = m[18];
  const double rho0 = 1.;
  const double jx2 = jx * jx, jy2 = jy * jy, jz2 = jz * jz;
  const double jj = (jx2 + jy2 + jz2);
  /* relaxation, mrt.hpp:103-126 */
  double mo[19];
  const double e_eq = -11 * rho + 19 / rho0 * jj;
  const double eps_eq = weps * rho + wepsj / rho0 * jj;
  const double pxx3_eq = 1 / (rho0) * (2 * jx2 - (jy2 + jz2));
  const double pww_eq = 1 / rho0 * (jy2 - jz2);
  const double pxy_eq = 1 / rho0 * jx * jy;
  const double pyz_eq = 1 / rho0 * jy * jz;
  const double pxz_eq = 1 / rho0 * jx * jz;
  mo[0] = rho;
  mo[1] = e - s1 * (e - e_eq);
  mo[2] = eps - s2 * (eps - eps_eq);
  mo[3] = jx;
  mo[4] = qx - s4 * (qx + 2. / 3. * jx);
  mo[5] = jy;
  mo[6] = qy - s4 * (qy + 2. / 3. * jy);
  mo[7] = jz;
  mo[8] = qz - s4 * (qz + 2. / 3. * jz);
  mo[9] = pxx3 - s9 * (pxx3 - pxx3_eq);
  mo[10] = pixx3 - s10 * (pixx3 - wxx * pxx3_eq);
  mo[11] = pww - s9 * (pww - pww_eq);
  mo[12] = piww - s10 * (piww - wxx * pww_eq);
  mo[13] = pxy - s13 * (pxy - pxy_eq);
  mo[14] = pyz - s13 * (pyz - pyz_eq);
  mo[15] = pxz - s13 * (pxz - pxz_eq);
  mo[16] = mx - s16 * mx;
  mo[17] = my - s16 * my;
  mo[18] = mz - s16 * mz;
  /* back-transform, mrt.hpp:129-173 */
#pragma GCC unroll 19
  for (int i = 0; i < Q; i++) {
    double acc = 0.0;
    int first = 1;
#pragma GCC unroll 19
    for (int k = 0; k < 19; k++) {
      const frac c = BACK[i][k];
      if (c.num == 0) continue;
      const double coef = (double)(c.num < 0 ? -c.num : c.num) / (double)c.den;
      const double term = coef * mo[k];
      if (first) {
        acc = c.num < 0 ? -term : term;
        first = 0;
      } else {
        acc = c.num < 0 ? acc - term : acc + term;
      }
    }
    f[i * nc + idx] = acc;
  }
}

void orc_mrt(void* h, const double* rates8) {
  orc_lattice* g = (orc_lattice*)h;
  const int64_t nc = g->ncell;
  double r[8];
  if (rates8)
    memcpy(r, rates8, sizeof r);
  else
    mrt_reference_rates(r);
  const double Fx = g->Fext[0], Fy = g->Fext[1], Fz = g->Fext[2];
#pragma omp parallel for schedule(static)
  for (int64_t idx = 0; idx < nc; idx++) { /* mrt.hpp:177-193 over real_ */
    if (g->level[idx] > 1) continue;
    if (g->obst[idx] != FLUID) continue;
    const double rho = g->m0[idx];
    mrt_cell(g->f, nc, idx, g->tau, r);
    for (int i = 0; i < Q; i++) {
      const double ef = EX[i] * Fx + EY[i] * Fy + EZ[i] * Fz;
      g->f[i * nc + idx] += 3. * rho * W[i] * ef;
    }
  }
}

/* ------------------------------------------------ plane bounce-back + cavity */
void orc_pre_bounce_back(void* h) {
  orc_lattice* g = (orc_lattice*)h;
  for (int p = 0; p < 6; p++) { /* PreBounceBack::launcher order x0, xl, y0, yl, z0, zl */
    if (!g->fi[p]) continue;
    const int64_t n = g->nplane[p];
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++)
      for (int k = 0; k < 5; k++) g->fi[p][k * n + i] = g->f[PRE_IDS[p][k] * g->ncell + g->plane[p][i]];
  }
}

void orc_post_bounce_back(void* h) {
  orc_lattice* g = (orc_lattice*)h;
  for (int p = 0; p < 6; p++) {
    if (!g->fi[p]) continue;
    const int64_t n = g->nplane[p];
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++)
      for (int k = 0; k < 5; k++) g->f[POST_IDS[p][k] * g->ncell + g->plane[p][i]] = g->fi[p][k * n + i];
  }
}

void orc_cavity(void* h, int32_t side, const double U[3]) {
  orc_lattice* g = (orc_lattice*)h;
  const int face = side ? ORC_ZL : ORC_Z0;
  if (!g->fi[face]) return; /* periodic z: empty buffer, nothing to do */
  const double L = g->n[2]; /* domain_size_ z (cavity.hpp:56-59) */
  const double uxx = U[0] * (1 + 0.5 / (L - 1));
  const double uyy = U[1] * (1 + 0.5 / (L - 1));
  const double uzz = U[2] * (1 + 0.5 / (L - 1));
  double coeff[5];
  for (int k = 0; k < 5; k++) {
    int i = CAVITY_IDS[side ? 1 : 0][k];
    coeff[k] = 6. * W[i] * (EX[i] * uxx + EY[i] * uyy + EZ[i] * uzz);
  }
  const int64_t n = g->nplane[face];
#pragma omp parallel for schedule(static)
  for (int64_t idx = 0; idx < n; idx++) /* cavity.hpp:81-86: tests obst at the plane-local index */
    if (g->obst[idx] == FLUID)
      for (int k = 0; k < 5; k++) g->fi[face][k * n + idx] += coeff[k];
}

/* -------------------------------------------------------- wall bounce-back */
void orc_wall_bounce_back(void* h) {
  orc_lattice* g = (orc_lattice*)h;
  const int64_t nc = g->ncell;
#pragma omp parallel for schedule(static)
  for (int z = g->ext_lo[2]; z <= g->ext_hi[2]; z++) /* bounce_back.hpp:167-184 over the Extend box */
    for (int y = g->ext_lo[1]; y <= g->ext_hi[1]; y++)
      for (int x = g->ext_lo[0]; x <= g->ext_hi[0]; x++) {
        const int64_t idx = IDX(g, x, y, z);
        if (g->obst[idx] != WALL) continue;
        for (int i = 1; i < Q; i++) {
          int nx = x + EX[i], ny = y + EY[i], nz = z + EZ[i];
          if (nx < g->ext_lo[0] || nx > g->ext_hi[0] || ny < g->ext_lo[1] || ny > g->ext_hi[1] ||
              nz < g->ext_lo[2] || nz > g->ext_hi[2])
            continue;
          const int64_t nidx = IDX(g, nx, ny, nz);
          if (g->obst[nidx] != WALL) g->f[i * nc + idx] = g->f[opp(i) * nc + nidx];
        }
      }
}

/* --------------------------------------------------------------- streaming */
void orc_streaming(void* h) {
  orc_lattice* g = (orc_lattice*)h;
  const int64_t nc = g->ncell;
  /* step 1: local swap at Real cells (streaming.hpp:37-43) */
#pragma omp parallel for schedule(static)
  for (int64_t idx = 0; idx < nc; idx++) {
    if (g->level[idx] > 1) continue;
    for (int i = 1; i < Q; i += 2) {
      double t = g->f[i * nc + idx];
      g->f[i * nc + idx] = g->f[(i + 1) * nc + idx];
      g->f[(i + 1) * nc + idx] = t;
    }
  }
  orc_update_ghost(g);
  /* step 2: swap with the neighbour along e_i for odd i at Extend cells (streaming.hpp:53-68) */
#pragma omp parallel for schedule(static)
  for (int z = 0; z < g->L[2]; z++)
    for (int y = 0; y < g->L[1]; y++)
      for (int x = 0; x < g->L[0]; x++) {
        const int64_t idx = IDX(g, x, y, z);
        if (g->level[idx] > 2) continue;
        for (int i = 1; i < Q; i += 2) {
          int nx = x + EX[i], ny = y + EY[i], nz = z + EZ[i];
          if (nx < g->ext_lo[0] || nx > g->ext_hi[0] || ny < g->ext_lo[1] || ny > g->ext_hi[1] ||
              nz < g->ext_lo[2] || nz > g->ext_hi[2])
            continue;
          const int64_t nidx = IDX(g, nx, ny, nz);
          double t = g->f[(i + 1) * nc + idx];
          g->f[(i + 1) * nc + idx] = g->f[i * nc + nidx];
          g->f[i * nc + nidx] = t;
        }
      }
}

/* ------------------------------------------------ Zou/He ("neumann") planes */
/* One table per face (neumann.hpp:27-258).  rho = (sum of the 9 tangential
 * populations + 2 * sum of the 5 known ones) / (1 + sgn * u_n); two transverse
 * corrections n_t = 1/2 * (A0 + A1 + A2 - (B0 + B1 + B2)) - 1/3 * rho * u_t;
 * the axis-aligned unknown gets known + sgn_main * 1/3 * rho * u_n and each
 * diagonal unknown gets known + 1/6 * rho * (s_n * u_n + s_t * u_t) + s * n_t.
 * Index orders are the reference's so the sums round identically. */
typedef struct {
  int axis, t1, t2;
  int den_sign;
  int tang[9];
  int known[5];
  int A1[3], B1[3], A2[3], B2[3];
  int main_dst, main_src, main_sign;
  int diag[4][6]; /* dst, src, s_n, s_t, t (1|2), sign of n_t */
} zouhe_face;

static const zouhe_face ZOUHE[6] = {
    /* x_0 */ {0, 1, 2, -1, {3, 4, 5, 6, 15, 17, 18, 16, 0}, {2, 10, 8, 14, 12}, {3, 15, 17}, {4, 18, 16},
               {5, 18, 15}, {6, 17, 16}, 1, 2, 1,
               {{9, 10, 1, -1, 1, 1}, {7, 8, 1, 1, 1, -1}, {11, 12, 1, 1, 2, -1}, {13, 14, 1, -1, 2, 1}}},
    /* x_l */ {0, 1, 2, 1, {3, 4, 5, 6, 15, 17, 18, 16, 0}, {1, 7, 9, 11, 13}, {3, 15, 17}, {4, 18, 16},
               {5, 18, 15}, {6, 17, 16}, 2, 1, -1,
               {{10, 9, -1, 1, 1, -1}, {8, 7, -1, -1, 1, 1}, {12, 11, -1, -1, 2, 1}, {14, 13, -1, 1, 2, -1}}},
    /* y_0 */ {1, 0, 2, -1, {1, 2, 5, 6, 11, 13, 14, 12, 0}, {4, 9, 8, 18, 16}, {1, 11, 13}, {2, 14, 12},
               {5, 11, 14}, {6, 13, 12}, 3, 4, 1,
               {{7, 8, 1, 1, 1, -1}, {10, 9, 1, -1, 1, 1}, {15, 16, 1, 1, 2, -1}, {17, 18, 1, -1, 2, 1}}},
    /* y_l */ {1, 0, 2, 1, {1, 2, 5, 6, 11, 13, 14, 12, 0}, {3, 7, 10, 15, 17}, {1, 11, 13}, {2, 14, 12},
               {5, 11, 14}, {6, 13, 12}, 4, 3, -1,
               {{8, 7, -1, -1, 1, 1}, {9, 10, -1, 1, 1, -1}, {16, 15, -1, -1, 2, 1}, {18, 17, -1, 1, 2, -1}}},
    /* z_0 */ {2, 0, 1, -1, {0, 1, 2, 3, 4, 7, 9, 10, 8}, {6, 13, 12, 17, 16}, {1, 7, 9}, {2, 10, 8},
               {3, 7, 10}, {4, 9, 8}, 5, 6, 1,
               {{11, 12, 1, 1, 1, -1}, {14, 13, 1, -1, 1, 1}, {15, 16, 1, 1, 2, -1}, {18, 17, 1, -1, 2, 1}}},
    /* z_l */ {2, 0, 1, 1, {0, 1, 2, 3, 4, 7, 9, 10, 8}, {5, 11, 14, 15, 18}, {1, 7, 9}, {2, 10, 8},
               {3, 7, 10}, {4, 9, 8}, 6, 5, -1,
               {{13, 14, -1, 1, 1, -1}, {12, 11, -1, -1, 1, 1}, {17, 18, -1, 1, 2, -1}, {16, 15, -1, -1, 2, 1}}}};

static inline double sum3(const double* f, int64_t nc, int64_t idx, const int a[3]) {
  return f[a[0] * nc + idx] + f[a[1] * nc + idx] + f[a[2] * nc + idx];
}

int32_t orc_neumann(void* h, int32_t face, const double Uphys[3]) {
  orc_lattice* g = (orc_lattice*)h;
  if (face < 0 || face > 5) return -1;
  const zouhe_face* z = &ZOUHE[face];
  double u[3];
  for (int d = 0; d < 3; d++) u[d] = Uphys[d] / g->celerity; /* convert_velocity<LBM_UNITS> */
  const double un = u[z->axis], ut1 = u[z->t1], ut2 = u[z->t2];
  const int64_t nc = g->ncell, n = g->nplane[face];
  double* f = g->f;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) {
    const int64_t idx = g->plane[face][i];
    if (g->obst[idx] != FLUID) continue;
    double ts = f[z->tang[0] * nc + idx];
    for (int k = 1; k < 9; k++) ts = ts + f[z->tang[k] * nc + idx];
    double ks = f[z->known[0] * nc + idx];
    for (int k = 1; k < 5; k++) ks = ks + f[z->known[k] * nc + idx];
    const double den = z->den_sign > 0 ? (1. + un) : (1. - un);
    const double rho = (ts + 2. * ks) / den;
    const double n1 = (1. / 2.) * (sum3(f, nc, idx, z->A1) - sum3(f, nc, idx, z->B1)) - (1. / 3.) * rho * ut1;
    const double n2 = (1. / 2.) * (sum3(f, nc, idx, z->A2) - sum3(f, nc, idx, z->B2)) - (1. / 3.) * rho * ut2;
    const double mterm = (1. / 3.) * rho * un;
    f[z->main_dst * nc + idx] = z->main_sign > 0 ? f[z->main_src * nc + idx] + mterm : f[z->main_src * nc + idx] - mterm;
    for (int k = 0; k < 4; k++) {
      const int* dg = z->diag[k];
      const double ut = dg[4] == 1 ? ut1 : ut2;
      const double nt = dg[4] == 1 ? n1 : n2;
      const double a = dg[2] > 0 ? un : -un;
      const double comb = dg[3] > 0 ? a + ut : a - ut;
      const double v = f[dg[1] * nc + idx] + (1. / 6.) * rho * comb;
      f[dg[0] * nc + idx] = dg[5] > 0 ? v + nt : v - nt;
    }
  }
  return 0;
}

/* ------------------------------------------------------ lid-driven cavity */
int32_t orc_lid_driven_cavity(void* h, int32_t face, const double Uphys[3]) {
  orc_lattice* g = (orc_lattice*)h;
  if (face < 0 || face > 5) return -1;
  double U[3];
  for (int d = 0; d < 3; d++) U[d] = Uphys[d] / g->celerity;
  const double u_squ = U[0] * U[0] + U[1] * U[1] + U[2] * U[2]; /* onika::math::dot */
  const int64_t nc = g->ncell, n = g->nplane[face];
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) { /* lid_driven_cavity.hpp:49-61 */
    const int64_t idx = g->plane[face][i];
    if (g->obst[idx] != FLUID) continue;
    double rho = 0.0;
    for (int c = 0; c < Q; c++) rho += g->f[c * nc + idx];
    for (int c = 0; c < Q; c++) {
      double eu = EX[c] * U[0] + EY[c] * U[1] + EZ[c] * U[2];
      g->f[c * nc + idx] = W[c] * rho * (1. + 3. * eu + 4.5 * eu * eu - 1.5 * u_squ);
    }
  }
  return 0;
}

/* ------------------------------------------------------- zero-gradient outlet */
void orc_snapshot_streamed(void* h) {
  orc_lattice* g = (orc_lattice*)h;
  if (!g->fs) g->fs = (double*)malloc(sizeof(double) * Q * (size_t)g->ncell);
  memcpy(g->fs, g->f, sizeof(double) * Q * (size_t)g->ncell);
}

int32_t orc_zero_gradient(void* h, int32_t face) {
  orc_lattice* g = (orc_lattice*)h;
  if (face < 0 || face > 5 || !g->fs) return -1;
  const int axis = face / 2;
  const int step = (face & 1) ? -1 : 1; /* towards the interior */
  const int64_t nc = g->ncell, n = g->nplane[face];
  int64_t shift = 1;
  for (int d = 0; d < axis; d++) shift *= g->L[d];
  for (int64_t i = 0; i < n; i++) {
    const int64_t idx = g->plane[face][i];
    if (g->obst[idx] != FLUID) continue; /* like the neumann / lid operators: fluid nodes only */
    const int64_t nb = idx + step * shift;
    for (int k = 0; k < 5; k++) {
      const int c = POST_IDS[face][k];
      g->f[c * nc + idx] = g->fs[c * nc + nb];
    }
  }
  return 0;
}

/* ------------------------------------------------------- simulation state */
void orc_simulation_state(void* h, double out[3]) {
  orc_lattice* g = (orc_lattice*)h;
  const int64_t nc = g->ncell;
  double s = 0.0, vmin = 1.79769313486231570815e+308, vmax = -1.79769313486231570815e+308;
  /* simulation_state.hpp:47-54 over real_ (in traversal order) */
  for (int64_t idx = 0; idx < nc; idx++) {
    if (g->level[idx] > 1) continue;
    s += g->m0[idx];
    double ux = g->m1[idx], uy = g->m1[nc + idx], uz = g->m1[2 * nc + idx];
    double v = sqrt(ux * ux + uy * uy + uz * uz);
    if (v < vmin) vmin = v;
    if (v > vmax) vmax = v;
  }
  out[0] = s;
  out[1] = vmin;
  out[2] = vmax;
}

/* init_double_couette (double_couette.hpp:25-49, init_double_couette.cu:74-100): f = feq(1, u)
 * with u = Uc - dU * g over the Real box, g the global index along dim, Uc = U / c,
 * dU = Uc / (0.5 * (n[dim] - 1)); the functor's operation order. */
void orc_init_double_couette(void* h, const double U[3], int32_t dim) {
  orc_lattice* g = (orc_lattice*)h;
  const int64_t nc = g->ncell;
  double uc[3], du[3];
  for (int d = 0; d < 3; d++) uc[d] = U[d] / g->celerity;
  for (int d = 0; d < 3; d++) du[d] = uc[d] / (0.5 * (g->n[dim] - 1));
  for (int z = 2; z < g->L[2] - 2; z++)
    for (int y = 2; y < g->L[1] - 2; y++)
      for (int x = 2; x < g->L[0] - 2; x++) {
        const int64_t idx = IDX(g, x, y, z);
        const double v = (double)((dim == 0 ? x : (dim == 1 ? y : z)) - 2);
        const double ux = uc[0] - du[0] * v, uy = uc[1] - du[1] * v, uz = uc[2] - du[2] * v;
        const double u_squ = ux * ux + uy * uy + uz * uz;
        for (int i = 0; i < Q; i++) {
          const double eu = ux * EX[i] + uy * EY[i] + uz * EZ[i];
          g->f[i * nc + idx] = 1. * W[i] * (1. + 3. * eu + 4.5 * eu * eu - 1.5 * u_squ);
        }
      }
}

/* plane_velocity_profile (plane_velocity_profile.cu:64-90, 179-260): per plane of the Real box
 * normal to dim, sum / count / min / max of |dx / dtLB * u| over fluid nodes, from the current m1
 * (call orc_macro_variables first for the current state).  avg = sum / count (0 when empty). */
void orc_plane_velocity_profile(void* h, int32_t dim, double* avg, double* vmin, double* vmax, int64_t* count) {
  orc_lattice* g = (orc_lattice*)h;
  const int64_t nc = g->ncell;
  const int n = g->n[dim];
  const double ratio = g->dx / g->dtLB;
  double* sum = (double*)calloc((size_t)n, sizeof(double));
  for (int i = 0; i < n; i++) {
    vmin[i] = 1.79769313486231570815e+308;
    vmax[i] = -1.79769313486231570815e+308;
    count[i] = 0;
  }
  for (int z = 2; z < g->L[2] - 2; z++)
    for (int y = 2; y < g->L[1] - 2; y++)
      for (int x = 2; x < g->L[0] - 2; x++) {
        const int64_t idx = IDX(g, x, y, z);
        if (g->obst[idx] != FLUID) continue;
        const int out = (dim == 0 ? x : (dim == 1 ? y : z)) - 2;
        const double ax = ratio * g->m1[idx], ay = ratio * g->m1[nc + idx], az = ratio * g->m1[2 * nc + idx];
        const double v = sqrt(ax * ax + ay * ay + az * az);
        sum[out] += v;
        count[out] += 1;
        if (vmin[out] > v) vmin[out] = v;
        if (vmax[out] < v) vmax[out] = v;
      }
  for (int i = 0; i < n; i++) avg[i] = count[i] > 0 ? sum[i] / (double)count[i] : 0.0;
  free(sum);
}

/* ---------------------------------------------------------------- access */
void orc_info(void* h, int64_t info[13]) {
  orc_lattice* g = (orc_lattice*)h;
  for (int d = 0; d < 3; d++) {
    info[d] = g->L[d];
    info[3 + d] = g->n[d];
  }
  info[6] = g->ncell;
  for (int p = 0; p < 6; p++) info[7 + p] = g->nplane[p];
}
double* orc_f(void* h) { return ((orc_lattice*)h)->f; }
double* orc_m0(void* h) { return ((orc_lattice*)h)->m0; }
double* orc_m1(void* h) { return ((orc_lattice*)h)->m1; }
int32_t* orc_obst(void* h) { return ((orc_lattice*)h)->obst; }
int32_t* orc_level(void* h) { return ((orc_lattice*)h)->level; }
