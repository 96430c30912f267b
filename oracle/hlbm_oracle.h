/*
 * hlbm_oracle.h -- CPU oracle for the D3Q19 hippoLBM time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This header and hlbm_oracle.c restate, in plain C,
 * the reference hippoLBM algorithm for one lattice on one MPI rank: the ghosted
 * local box, the level/plane traversal lists, the swap streaming with its
 * single-rank periodic ghost exchange, BGK, MRT, the plane bounce-back buffers,
 * cavity, wall bounce-back, the Zou/He "neumann" operators, lid-driven cavity,
 * set_distribution, the obstacle rasteriser and simulation_state.  Every
 * operator follows the reference's floating-point operation order so that, built
 * with -ffp-contract=off, it reproduces the reference functors bit for bit.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
 * this library.  The product path (hippolbm_b200) never calls it.
 *
 * The same symbol set is exported by oracle/_ref/libhlbm_ref.so, which drives the
 * reference's own functor headers; the Python driver in oracle/oracle.py runs
 * either library through identical calls.
 */
#ifndef HLBM_ORACLE_H
#define HLBM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Face numbering follows bounce_back_manager.hpp:50-56 (dim * 2 + side). */
enum { ORC_X0 = 0, ORC_XL = 1, ORC_Y0 = 2, ORC_YL = 3, ORC_Z0 = 4, ORC_ZL = 5 };

/* domain (domain_lbm.cpp:66-110) + build_traversal (grid_region.hpp:89-197)
 * + define_grid_3dq19 (define_lbm_fields.cpp:58-86) + init_obst (init_obst.hpp:29-32).
 * Returns NULL and sets *err (<0) on an inconsistent domain. */
void* orc_create(const int32_t cell_dims[3], const double bmin[3], const double bmax[3],
                 const int32_t periodic[3], int32_t* err);
void orc_destroy(void* h);

/* lbm_parameters (lbm_parameters.cpp:73-99). has_tau selects define_by_tau. */
void orc_lbm_parameters(void* h, const double Fext[3], double celerity, double nuth, double avg_rho,
                        int32_t has_tau, double tau, double dt);
/* out: Fext[3], celerity, dtLB, nuth, nu, tau, avg_rho */
void orc_get_parameters(void* h, double out[9]);

/* set_distribution (set_distribution.cu:69-109); bounds6 = {min xyz, max xyz} or NULL. */
void orc_set_distribution(void* h, double value, const double* bounds6, int32_t do_update);

/* obstacles (obstacle.hpp, obstacles.hpp:84-107, update_obstacles.cu:32-119) */
void orc_init_obstacles(void* h);
void orc_register_ball(void* h, int32_t id, const double center[3], double radius);
void orc_register_wall(void* h, int32_t id, const double bmin[3], const double bmax[3]);
void orc_register_quadric(void* h, int32_t id, const double q[16]);
void orc_update_obstacles(void* h);

/* step operators */
void orc_macro_variables(void* h);                      /* macro_variables.cu:71-90 */
void orc_bgk(void* h);                                  /* bgk.cu:77-94 */
void orc_mrt(void* h, const double* rates8);            /* mrt.cu:71-89; rates8 NULL = reference */
void orc_pre_bounce_back(void* h);                      /* pre_bounce_back.cu:89-118 */
void orc_post_bounce_back(void* h);                     /* post_bounce_back.cu:101-123 */
void orc_cavity(void* h, int32_t side, const double U[3]); /* cavity.cu:66-88, side 0 = z_0, 1 = z_l */
void orc_wall_bounce_back(void* h);                     /* wall_bounce_back.cu:58-73 */
void orc_streaming(void* h);                            /* streaming.cu:68-118 (asynchrone: false) */
void orc_update_ghost(void* h);                         /* update_ghost.hpp:57-70, one rank */
int32_t orc_neumann(void* h, int32_t face, const double U[3]);           /* neuman.cu:69-122 */
int32_t orc_lid_driven_cavity(void* h, int32_t face, const double U[3]); /* lid_driven_cavity.cu:69-93 */
/* zero_gradient outlet: an operator this project adds (no reference counterpart).  After
 * orc_snapshot_streamed (called right after streaming), on the plane of `face` the populations
 * entering from outside take the streamed values of the interior neighbour one node inside. */
void orc_snapshot_streamed(void* h);
int32_t orc_zero_gradient(void* h, int32_t face);
/* simulation_state (simulation_state.cu:73-98): out = {sum rho, min |u|, max |u|} over Real */
void orc_simulation_state(void* h, double out[3]);

/* init_double_couette (init_double_couette.cu:74-100); dim 0 x, 1 y, 2 z */
void orc_init_double_couette(void* h, const double U[3], int32_t dim);
/* plane_velocity_profile (plane_velocity_profile.cu:64-90, 179-260) from the current m1 */
void orc_plane_velocity_profile(void* h, int32_t dim, double* avg, double* vmin, double* vmax, int64_t* count);

/* accessors: info = {L[3], n[3], ncell, plane sizes[6]} */
void orc_info(void* h, int64_t info[13]);
double* orc_f(void* h);
double* orc_m0(void* h);
double* orc_m1(void* h);
int32_t* orc_obst(void* h);
int32_t* orc_level(void* h);

#ifdef __cplusplus
}
#endif

#endif
