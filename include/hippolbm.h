/*
 * hippolbm.h -- C-ABI of the B200 D3Q19 lattice Boltzmann step.
 *
 * Each entry point stands in for one hippoLBM Onika operator on the time-step path (the
 * operator's `execute()` is cited beside it).  A caller builds a lattice the way a deck's
 * `initialize` list does (domain -> lbm_parameters -> set_distribution -> obstacles), records
 * the compute-loop hooks in deck order (`pre_stream_bcs`, `post_stream_bcs`,
 * `boundary_conditions`, `start_iteration`), then calls hlbm_step(), which runs whole
 * compute_loop iterations (config_compute_loop.msp:27-37) as fused CUDA kernels.
 *
 * Conventions
 *   - Every function returns 0 on success and a negative HLBM_E* code on failure;
 *     hlbm_last_error() returns the message of the calling thread's last failure.  The
 *     library never exits the process (the reference prints and calls std::exit,
 *     domain_lbm.cpp:85 and :105).
 *   - A context is not thread-safe: callers serialise calls per context.  Each context owns
 *     one CUDA stream; work is asynchronous on it unless the function copies to the host.
 *   - Arrays are plain host pointers.  Populations are exchanged as FP64, SoA,
 *     out[i * nz*ny*nx + (z*ny + y)*nx + x] over the real nodes (no ghost layers),
 *     the reference's FieldView layout (field_view.hpp:56) without its 2 ghost layers.
 *   - Velocities given to hlbm_neumann / hlbm_lid_driven_cavity are physical and are
 *     divided by the celerity (convert_velocity<LBM_UNITS>, lbm_parameters.hpp:102-106);
 *     cavity velocities are raw lattice values (cavity.cu:54,70), as in the reference.
 */
#ifndef HIPPOLBM_H
#define HIPPOLBM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hlbm_ctx hlbm_ctx;

/* error codes */
#define HLBM_OK 0
#define HLBM_EINVAL (-1)   /* bad argument */
#define HLBM_EDOMAIN (-2)  /* inconsistent domain (domain_lbm.cpp:81-106) */
#define HLBM_ECUDA (-3)    /* CUDA runtime failure */
#define HLBM_ENOMEM (-4)   /* device allocation failed */
#define HLBM_EPLAN (-5)    /* operator list the fused step cannot express */
#define HLBM_ESTATE (-6)   /* call not valid in the current state */

/* precision tiers */
#define HLBM_F64 0        /* FP64 storage and compute, FMA + reciprocal multiplies */
#define HLBM_F64_STRICT 1 /* FP64, reference operation order, no FMA contraction */
#define HLBM_F32 2        /* FP32 storage and compute */
#define HLBM_F16 3        /* FP32 compute, FP16 storage of (f_i - w_i rho0) * scale */
#define HLBM_BF16 4       /* FP32 compute, BF16 storage of (f_i - w_i rho0) * scale */

/* compute-loop hooks (config_compute_loop.msp:7-21) */
#define HLBM_HOOK_START_ITERATION 0
#define HLBM_HOOK_PRE_STREAM 1
#define HLBM_HOOK_POST_STREAM 2
#define HLBM_HOOK_BOUNDARY_CONDITIONS 3

/* plane regions, traversal names of grid_region.hpp:360-373 */
#define HLBM_PLAN_YZ_0 0
#define HLBM_PLAN_YZ_L 1
#define HLBM_PLAN_XZ_0 2
#define HLBM_PLAN_XZ_L 3
#define HLBM_PLAN_XY_0 4
#define HLBM_PLAN_XY_L 5

const char* hlbm_last_error(void);
/* Library version string. */
const char* hlbm_version(void);

/* domain (domain_lbm.cpp:66-110) followed by define_grid_3dq19 (define_lbm_fields.cpp:58-86),
 * build_traversal (grid_region.hpp:89-197), init_obst (init_obst.hpp:29-32) and the default
 * set_distribution of value 1 over the lattice (config_initialize.msp:22-23).  Nodes per axis
 * = cell_dims + 1; dx = (bmax - bmin) / cell_dims must agree on all axes.  `device` selects the
 * CUDA device.  On success *out owns device memory until hlbm_destroy(). */
int hlbm_domain(const int32_t cell_dims[3], const double bmin[3], const double bmax[3], const int32_t periodic[3],
                int32_t precision, int32_t device, hlbm_ctx** out);
int hlbm_destroy(hlbm_ctx* ctx);
/* Device memory of contexts and batches comes from a stream-ordered pool per device that keeps
 * freed blocks for the next allocation, so that creating and destroying lattices while others run
 * costs no device-wide synchronisation (no reference counterpart).  hlbm_trim_memory waits for the
 * device and returns the pool's unused blocks to the driver. */
int hlbm_trim_memory(int32_t device);

/* lbm_parameters (lbm_parameters.cpp:73-99): tau if has_tau, else dt if dt > 0, else the
 * celerity defines the lattice time step; Fext is converted to lattice units. */
int hlbm_lbm_parameters(hlbm_ctx* ctx, const double Fext[3], double celerity, double nuth, double avg_rho,
                        int32_t has_tau, double tau, double dt);
/* out = {Fext_lb[3], celerity, dtLB, nuth, nu, tau, avg_rho} */
int hlbm_get_parameters(hlbm_ctx* ctx, double out[9]);

/* collision: bgk (bgk.cu:77-94) when kind == 0, mrt (mrt.cu:71-89) when kind == 1.
 * rates8 = {s_e, s_eps, s_q, s_pi, s_m, w_eps, w_epsj, w_xx}; NULL keeps the reference's
 * constants (mrt.hpp:43-47); s_nu = 1 / tau always. */
int hlbm_collision(hlbm_ctx* ctx, int32_t kind, const double* rates8);

/* Reduced-precision storage keeps (f_i - d_i) * scale, d_i the rest equilibrium of the lattice's
 * collision at density rho0 (BGK: w_i * rho0; MRT: the isotropic state with the model's rest
 * moments), rho0 = 1 and scale 1024 (HLBM_F16) or 1 (HLBM_BF16) by default.  Changing rho0, the
 * scale or the collision re-encodes the current state on the device.  The 16-bit tiers collide in
 * deviation form (f_i - d_i) in FP32.  No reference counterpart: part of the precision tiers. */
int hlbm_storage_scale(hlbm_ctx* ctx, double rho0, double scale);
/* Rounding of the 16-bit storage tiers when a step stores the state: 1 (the default) stochastic
 * -- round up with probability equal to the discarded fraction, from a hash of (node, step
 * number, direction), so results are reproducible and the same alone or in a batch -- or 0 round
 * to nearest.  Read-outs always round to nearest.  No effect on FP64 / FP32. */
int hlbm_storage_rounding(hlbm_ctx* ctx, int32_t mode);

/* set_distribution (set_distribution.cu:69-109), applied now: f_i = value * w_i on the
 * nodes of the box {int(min/dx), int(max/dx)} clipped to the lattice, or on all nodes when
 * bounds6 is NULL.  do_update is accepted for compatibility (there are no ghost layers). */
int hlbm_set_distribution(hlbm_ctx* ctx, double value, const double* bounds6, int32_t do_update);
/* init_double_couette (init_double_couette.cu:74-100, double_couette.hpp:25-49): f = feq(rho = 1,
 * u = U / c - dU * g) at every node, g the node's index along dim (0 x, 1 y, 2 z) and
 * dU = (U / c) / (0.5 * (n[dim] - 1)): a linear profile from U at g = 0 to -U at the far face. */
int hlbm_init_double_couette(hlbm_ctx* ctx, const double U[3], int32_t dim);

/* obstacles: init_obstacles (init_obstacles.cpp), register_solid_ball
 * (register_solid_ball.cpp), register_solid_wall (register_solid_wall.cpp), register_quadrics
 * (register_quadrics.cpp:72-79, q = the transformed 4x4 matrix, row-major), and the rasteriser
 * update_obstacles (update_obstacles.cu:106-119), which marks WALL_ (-2) in the flag bytes. */
int hlbm_init_obstacles(hlbm_ctx* ctx);
int hlbm_register_solid_ball(hlbm_ctx* ctx, int32_t id, const double center[3], double radius);
int hlbm_register_solid_wall(hlbm_ctx* ctx, int32_t id, const double bmin[3], const double bmax[3]);
int hlbm_register_quadric(hlbm_ctx* ctx, int32_t id, const double q[16]);
int hlbm_update_obstacles(hlbm_ctx* ctx);

/* Compute-loop hooks, recorded in call order and executed inside every hlbm_step().
 * pre_bounce_back (pre_bounce_back.cu:89-118), cavity_z_0 / cavity_z_l (cavity.cu:66-88,
 * side 0 / 1) and wall_bounce_back (wall_bounce_back.cu:58-73) belong to pre_stream_bcs;
 * post_bounce_back (post_bounce_back.cu:101-123), neumann (neuman.cu:69-122) and
 * lid_driven_cavity (lid_driven_cavity.cu:69-93) to post_stream_bcs or boundary_conditions
 * (`hook`); set_distribution with bounds to start_iteration. */
int hlbm_clear_hooks(hlbm_ctx* ctx);
int hlbm_pre_bounce_back(hlbm_ctx* ctx);
int hlbm_cavity(hlbm_ctx* ctx, int32_t side, const double U[3]);
int hlbm_wall_bounce_back(hlbm_ctx* ctx);
int hlbm_post_bounce_back(hlbm_ctx* ctx, int32_t hook);
int hlbm_neumann(hlbm_ctx* ctx, int32_t hook, const double U[3], const int32_t* regions, int32_t nregions);
int hlbm_lid_driven_cavity(hlbm_ctx* ctx, int32_t hook, const double U[3], const int32_t* regions,
                           int32_t nregions);
int hlbm_start_set_distribution(hlbm_ctx* ctx, double value, const double bounds6[6]);
/* zero_gradient outlet (no reference counterpart: the reference's "neumann" is a Zou/He velocity
 * condition): on each listed plane, the populations entering from outside take the streamed values
 * of the interior neighbour one node inside along the face normal.  post_stream_bcs or
 * boundary_conditions. */
int hlbm_zero_gradient(hlbm_ctx* ctx, int32_t hook, const int32_t* regions, int32_t nregions);

/* nsteps iterations of compute_loop: macro_variables -> collision -> pre_stream_bcs ->
 * streaming (streaming.cu:68-118, asynchrone: false) -> post_stream_bcs ->
 * boundary_conditions.  Asynchronous on the context stream. */
int hlbm_step(hlbm_ctx* ctx, int64_t nsteps);
int hlbm_sync(hlbm_ctx* ctx);

/* macro_variables (macro_variables.cu:71-90) of the current state, copied to the host:
 * rho[n] and u[3 * n] (SoA); walls get u = 0 and rho = 0.  Either pointer may be NULL. */
int hlbm_macro_variables(hlbm_ctx* ctx, double* rho, double* u);
/* simulation_state (simulation_state.cu:73-98): out = {sum rho, min |u|, max |u|} over the
 * nodes, FP64 on the device. */
int hlbm_simulation_state(hlbm_ctx* ctx, double out[3]);

/* plane_velocity_profile (plane_velocity_profile.cu:179-260): for each plane normal to dim (0 x,
 * 1 y, 2 z), the mean, minimum and maximum over fluid nodes of |dx / dtLB * u| and the fluid node
 * count, from the current state (FP64 on the device, deterministic).  Arrays hold n[dim] values;
 * any may be NULL.  A plane without fluid nodes has mean 0, min DBL_MAX and max -DBL_MAX, as in the
 * reference. */
int hlbm_plane_velocity_profile(hlbm_ctx* ctx, int32_t dim, double* avg, double* vmin, double* vmax,
                                int64_t* count);

/* FP64 reductions on the device (no reference counterparts; used by the precision study and the
 * solve server).  hlbm_residual: relative L2 change of the velocity field since the previous call
 * on this context, sqrt(sum |u - u_prev|^2 / sum |u|^2) (HUGE_VAL on the first call; keeps an
 * FP32 velocity snapshot on the device).  hlbm_moments: {sum rho, sum rho u_x, sum rho u_y,
 * sum rho u_z} over fluid nodes.  hlbm_wall_force: force on the wall obstacles by momentum exchange,
 * sum over fluid-to-wall links of 2 f*_i e_i, from the post-collision state (after >= 1 step). */
int hlbm_residual(hlbm_ctx* ctx, double* out);
int hlbm_moments(hlbm_ctx* ctx, double out[4]);
int hlbm_wall_force(hlbm_ctx* ctx, double out[3]);

/* populations of the current state (FP64, layout above); put replaces them */
int hlbm_get_populations(hlbm_ctx* ctx, double* out);
int hlbm_put_populations(hlbm_ctx* ctx, const double* in);
/* Checkpoint / restore of the carried state (no reference counterpart).  The image holds a
 * header (shape, precision, step count, storage parameters), the flag bytes and the populations
 * exactly as stored (FP64 / FP32 / 16-bit), so a lattice restored into a context built from the
 * same deck continues bit for bit in every tier.  The copies are asynchronous on the context's
 * stream (pinned host memory makes them DMA transfers) and complete before the call returns. */
int hlbm_checkpoint_bytes(hlbm_ctx* ctx, int64_t* bytes);
int hlbm_checkpoint_save(hlbm_ctx* ctx, void* host, int64_t bytes);
int hlbm_checkpoint_load(hlbm_ctx* ctx, const void* host, int64_t bytes);

/* flag bytes: -1 fluid, -2 wall (enum.hpp:59-60) */
int hlbm_get_flags(hlbm_ctx* ctx, int8_t* out);
int hlbm_put_flags(hlbm_ctx* ctx, const int8_t* in);

/* info = {nx, ny, nz, precision, steps done, kernel launches, bytes per population, device} */
int hlbm_info(hlbm_ctx* ctx, int64_t info[8]);
/* Step kernel selection (no reference counterpart).  Variants 0..5: variant % 2 picks the kernel,
 * 0 = one node per thread (two per thread for the 16-bit tiers), 1 = vectorised (consecutive
 * x-nodes per thread in one vector per direction plane -- 16 bytes at variant 1, 8 bytes at 3 and
 * 5 for the FP32 and 16-bit tiers, 16 bytes always for FP64; used when nx splits into >= 32
 * vectors, else the first kernel runs; with wall obstacles a fix-up pass re-steps the nodes next
 * to walls); variant / 2 = 0, 1, 2 targets at least 1, 2 or 3 blocks of 256 threads per SM.
 * The FP32 and 16-bit tiers update node pairs in packed FP32 where a plan has no body force, no
 * start_iteration boxes and no wall nodes outside wall_bounce_back; other plans run one node per
 * thread.  A context starts at its tier's default (hlbm_autotune's pick on 512^3 Couette: FP64 4,
 * FP32 1, FP16 / BF16 9) until hlbm_tune or hlbm_autotune chooses.  Variants 6, 7: persistent
 * kernel fed by bulk asynchronous copies of whole rows
 * into shared-memory stages (256 or 512 threads per CTA; needs nx * bytes per population to be a
 * multiple of 16; otherwise variant 4 runs).  hlbm_autotune times `reps` fused launches of every
 * variant on this lattice (from the current populations into the idle buffer, so the state does
 * not advance), keeps the fastest, and returns it in *chosen and the per-variant times (ms, -1 if
 * skipped) in ms_per_variant[HLBM_NUM_VARIANTS].  Variants 8, 9 (FP16 / BF16): the row pipeline --
 * a producer warp bulk-copies each tile's source rows and flags into shared-memory stages,
 * consumer warps update node pairs from there in packed FP32 -- with two CTAs of 8 consumer warps
 * (8) or one CTA of 12 (9) per SM; fused steps of lattices with nx % 16 == 0, nx <= 1024 (8) or
 * 1536 (9) and the pair kernels' plan conditions.  Other lattices with nx >= 4, fewer than 2^32
 * nodes and those plan conditions take the span pipeline at the same shape: tiles are spans of
 * the linear node index, one bulk copy per direction, so rows of any length stream from shared
 * memory.  Otherwise variant 5 runs. */
#define HLBM_NUM_VARIANTS 10
int hlbm_tune(hlbm_ctx* ctx, int32_t variant);
int hlbm_autotune(hlbm_ctx* ctx, int32_t reps, int32_t* chosen, double* ms_per_variant);
/* the context's cudaStream_t, as a pointer-sized handle */
void* hlbm_stream(hlbm_ctx* ctx);
/* Bound on each wait of the pipelined kernels (variants 6 - 9) in polls of their shared-memory
 * barriers (the first poll a test, the others a hardware-suspended try_wait of up to about a
 * microsecond); 0 restores the default of 2e7 polls.  Every wait also gives up after two seconds
 * whatever the bound.  No reference counterpart.  A wait that runs
 * out records an error on the device and its CTA returns after its copies in flight have landed;
 * the next call that reads the state (hlbm_get_populations, hlbm_simulation_state, ...) fails with
 * HLBM_ECUDA and clears the record, and the context stays usable (put populations back and step
 * on).  A small bound lets a test exercise that path, and a host that prefers to fail fast on a
 * stalled GPU can shorten the default. */
int hlbm_set_wait_limit(hlbm_ctx* ctx, int64_t polls);

/* ---------------------------------------------------------------------------------------------
 * Batches (no reference counterpart).  A batch advances many independent lattices -- contexts
 * made with hlbm_domain on the same device and precision, each with its own size, plan, collision
 * and boundary operators -- with ONE launch of the pipelined persistent kernel per time step, over
 * the concatenated tile list of all members; steps are replayed from a captured CUDA graph of two
 * steps.  Kernel (hlbm_batch_tune): tiles of about 256 nodes with direct pulls, any lattice
 * shape -- 8 (default) one CTA per tile, 9 a persistent grid of resident CTAs each walking a
 * contiguous range of tiles; 6 / 7 = the pipelined kernel
 * (rows bulk-copied into shared memory; members need nx * bytes per population % 16 == 0);
 * 10 = no shared launch: every member runs its own single-lattice step kernel (its hlbm_tune
 * variant, 4 for 6 / 7) on its own stream, all members forked from and joined to the batch stream
 * inside one captured graph of two steps.  A
 * member that has not stepped yet takes its first step inside the batched launch.  While a
 * lattice is in a batch, step it only through hlbm_batch_step; read-outs stay valid.  A lattice
 * belongs to at most one batch; hlbm_destroy of a member removes it from its batch first.
 * hlbm_batch_step(b, n) advances every member n steps. */
typedef struct hlbm_batch hlbm_batch;
int hlbm_batch_create(int32_t precision, int32_t device, hlbm_batch** out);
int hlbm_batch_add(hlbm_batch* b, hlbm_ctx* lattice);
int hlbm_batch_remove(hlbm_batch* b, hlbm_ctx* lattice);
int hlbm_batch_step(hlbm_batch* b, int64_t nsteps);
int hlbm_batch_tune(hlbm_batch* b, int32_t variant);
/* The batch's kernel chosen by measurement (no reference counterpart): times `reps` replays of one
 * step of every batch variant that applies (6, 7: pipelined kernel; 8, 9: tile-list kernel; 10:
 * every member's own tuned kernel on its own stream) on the batch itself -- each reading the
 * members' current state and writing their idle buffers, so no member advances -- keeps the fastest
 * and returns it in *chosen and the per-variant times (ms per step, -1 if skipped) in
 * ms_per_variant[HLBM_BATCH_VARIANTS], index variant - 6. */
#define HLBM_BATCH_VARIANTS 5
int hlbm_batch_autotune(hlbm_batch* b, int32_t reps, int32_t* chosen, double* ms_per_variant);
/* info = {members, tiles, tile elements, stages, graph replays, kernel launches} */
int hlbm_batch_info(hlbm_batch* b, int64_t info[6]);
/* the batch's cudaStream_t (every batched launch is issued on it), as a pointer-sized handle */
void* hlbm_batch_stream(hlbm_batch* b);
int hlbm_batch_destroy(hlbm_batch* b);

/* simulation_state for callers that cannot allocate device memory, such as an analysis hook
 * inside a host application that owns the whole device budget, or a loop that must not pay
 * cudaMalloc's device-wide synchronisation.  No counterpart in the reference.  The caller
 * passes device pointers: FP64 populations f[i * stride + node] (stride >= node count), one
 * flag byte per node, and out3 = {sum rho, min |u|, max |u|}; `stream` is a cudaStream_t or
 * NULL; the call is asynchronous on it.  It allocates nothing: block partial sums go to a
 * static __device__ array of HLBM_STATIC_PARTIALS slots (384 KiB held by every GPU that
 * loads the library, until exit), so lattices above HLBM_STATIC_MAX_NODES nodes are rejected
 * with HLBM_EINVAL.  The first call on a device looks up the array's address in the device's
 * current context, and so does the first call after another context became current there (a
 * cudaDeviceReset, or a driver-API caller's own context); make those calls before any stream
 * capture.  All calls share the array: calls that overlap on the GPU race. */
#define HLBM_STATIC_PARTIALS 16384
#define HLBM_STATIC_MAX_NODES (16384LL * HLBM_STATIC_PARTIALS)
int hlbm_simulation_state_static(const double* f, int64_t stride, const int8_t* flags, const int32_t n[3],
                                 double* out3, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* HIPPOLBM_H */
