// capi.cu -- host runtime behind include/hippolbm.h.
//
// A context owns one lattice on one device: two SoA population buffers (pull scheme), one
// flag byte per node, a step plan compiled from the recorded hook operators, and a stream.
// State phases:
//   RAW     f[cur] holds S_k, the reference's state after k steps (post-stream + BCs);
//   POSTCOL f[cur] holds C_{k-1}, the post-collision state inside step k (what the fused
//           kernel carries from launch to launch);
//   MATER   as POSTCOL, and f[1-cur] also holds S_k, produced by the finish kernel for a
//           read-out (the next step overwrites it).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "aux_kernels.cuh"
#include "hippolbm.h"
#include "launch.cuh"

using namespace hlbm;

namespace {
thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define HLBM_CK(call)                                                                         \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess) return fail(HLBM_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

enum HookKind { H_PRE_BB, H_CAVITY, H_WALL_BB, H_POST_BB, H_NEUMANN, H_LID, H_SETDIST, H_ZERO_GRADIENT };

struct HookOp {
  int hook;
  int kind;
  int face;  // cavity side (0, 1) or plane face (0..5)
  double u[3];
  double value;
  double bounds[6];
};

enum Phase { RAW = 0, POSTCOL = 1, MATER = 2 };

size_t elem_size(int prec) {
  switch (prec) {
    case HLBM_F64:
    case HLBM_F64_STRICT: return 8;
    case HLBM_F32: return 4;
    default: return 2;
  }
}

constexpr double W_OF(int i) { return 1.0 / D3Q19::wden[i]; }

// Device memory of lattices and batches comes from one stream-ordered pool per device that keeps
// freed blocks for reuse (release threshold: unlimited).  Creating and destroying lattices while
// others are stepping then costs no device-wide synchronisation: cudaFree waits for every stream
// of the device, and in a solve server that can stall each retirement for hundreds of
// milliseconds.  hlbm_trim_memory hands the cached blocks back to the driver.
std::mutex g_pool_mutex;
cudaMemPool_t g_pools[64] = {};

cudaMemPool_t device_pool(int dev) {
  if (dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lock(g_pool_mutex);
  if (!g_pools[dev]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    if (cudaMemPoolCreate(&g_pools[dev], &props) != cudaSuccess) {
      cudaGetLastError();
      g_pools[dev] = nullptr;
      return nullptr;
    }
    uint64_t keep = ~uint64_t(0);
    cudaMemPoolSetAttribute(g_pools[dev], cudaMemPoolAttrReleaseThreshold, &keep);
  }
  return g_pools[dev];
}

// allocation in stream order on s (usable by work queued on s after it, or by other streams once
// s has been synchronised); freed with pool_free on a stream whose earlier work used it last
cudaError_t pool_alloc(void** ptr, size_t bytes, int dev, cudaStream_t s) {
  cudaMemPool_t pool = device_pool(dev);
  if (!pool) return cudaErrorMemoryAllocation;
  return cudaMallocFromPoolAsync(ptr, bytes, pool, s);
}

void pool_free(void* ptr, cudaStream_t s) {
  if (ptr) cudaFreeAsync(ptr, s);
}
}  // namespace

namespace hlbm {
// sets the message hlbm_last_error() returns, for entry points defined in other files
int record_error(int code, const std::string& msg) { return fail(code, msg); }
}  // namespace hlbm

struct hlbm_ctx {
  int n[3];
  int periodic[3];
  double bmin[3], bmax[3], dx;
  int precision;
  int device;
  // LBMParameters (lbm_parameters.hpp:41-57)
  double Fext[3], celerity, dtLB, nuth, nu, tau, avg_rho;
  int collision = 0;
  double mrt[8];
  double rho0 = 1.0, scale = 1.0;
  std::vector<HookOp> hooks;
  std::vector<ObstacleDesc> obstacles;
  void* f[2] = {nullptr, nullptr};
  int cur = 0;
  int8_t* flags = nullptr;
  int8_t* nearwall = nullptr;  // per node: some pull comes from a wall node (k_near_wall)
  bool maybe_walls = false;     // the flags may hold wall nodes (an obstacle was rasterised or put)
  bool variant_tuned = false;   // hlbm_tune / hlbm_autotune chose the variant (else the tier default)
  long long wait_limit = TMA_WAIT_LIMIT;  // polls before a wait of the pipelined kernel gives up
  double* partials = nullptr;
  double* stats_dev = nullptr;
  double* plane_tmp = nullptr;
  float* uprev = nullptr;  // velocity snapshot of hlbm_residual
  cudaStream_t stream = nullptr;
  int phase = RAW;
  int variant = 0;  // step kernel variant (launch.cuh): kernel = variant % 2, occupancy = variant / 2
  int rounding = 1;  // 16-bit storage: 1 stochastic rounding (default), 0 round to nearest
  int64_t steps = 0;
  int64_t launches = 0;
  int64_t ncell = 0, stride = 0;
  StepPlan plan;
  bool plan_dirty = true;
  // pipelined persistent kernel: plan and lattice descriptor in device memory, tile list
  StepPlan* plan_dev = nullptr;
  LatticeDesc* desc_dev = nullptr;
  Tile* tiles_dev = nullptr;
  int* err_dev = nullptr;
  int ntiles = 0, tile_elems = 0, tma_stages = 0, tma_stages2 = 0, sms = 148;
  hlbm_batch* batch = nullptr;  // the batch this lattice is a member of
  int64_t plan_version = 0;       // bumped whenever the step plan is rebuilt
  uint32_t* seed_dev = nullptr;   // step-number pair of graph-replayed launches (16-bit tiers)
  uint32_t seed_host[2] = {0, 0};
  cudaEvent_t join_ev = nullptr;  // end of this member's work in a concurrent batch graph
};

namespace {

void mrt_reference(double r[8]) {  // mrt.hpp:43-47
  r[0] = 1.19;
  r[1] = 1.4;
  r[2] = 1.2;
  r[3] = 1.4;
  r[4] = 1.98;
  r[5] = 0;
  r[6] = -475. / 63.;
  r[7] = 0;
}

// The 16-bit tiers store f_i - d_i with d_i the rest equilibrium of the lattice's collision at
// density rho0: w_i * rho0 for BGK; for MRT the isotropic state with the MRT model's rest moments
// (rho0, e = -11 rho0, eps = w_eps * rho0), which differs from w_i * rho0 unless w_eps = 3.  Stored
// deviations then stay of the order of the flow's own perturbation, and so do the rounding steps.
void storage_reference(const hlbm_ctx* c, float dref[Q]) {
  double a = 1.0 / 3.0, b = 1.0 / 18.0, cc = 1.0 / 36.0;  // rest populations f0, f1..6, f7..18
  if (c->collision == 1) {
    // a + 6b + 12c = 1, -30a - 66b + 96c = -11, 12a - 24b + 12c = w_eps (Cramer's rule)
    const double A[3][3] = {{1, 6, 12}, {-30, -66, 96}, {12, -24, 12}}, r[3] = {1, -11, c->mrt[5]};
    auto det3 = [](const double M[3][3]) {
      return M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
             M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
    };
    const double D = det3(A);
    double x[3];
    for (int k = 0; k < 3; k++) {
      double B[3][3];
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) B[i][j] = j == k ? r[i] : A[i][j];
      x[k] = det3(B) / D;
    }
    a = x[0], b = x[1], cc = x[2];
  }
  for (int i = 0; i < Q; i++) dref[i] = float((i == 0 ? a : (i <= 6 ? b : cc)) * c->rho0);
}

// the near-wall map after the flags changed (stream-ordered after the change)
int refresh_near_wall(hlbm_ctx* c) {
  c->launches++;
  HLBM_CK(launch_near_wall(c->flags, c->nearwall, c->n, c->periodic, c->stream));
  return HLBM_OK;
}

void base_plan(hlbm_ctx* c, StepPlan& p) {
  std::memset(&p, 0, sizeof(p));
  p.nx = c->n[0];
  p.ny = c->n[1];
  p.nz = c->n[2];
  for (int d = 0; d < 3; d++) p.periodic[d] = c->periodic[d];
  p.ncell = c->ncell;
  p.stride = c->stride;
  p.rho0 = c->rho0;
  p.nearwall = c->nearwall;
  p.wall_flags = c->maybe_walls ? 1 : 0;
  p.scale = c->scale;
  p.inv_scale = 1.0 / c->scale;
  storage_reference(c, p.dref);
  p.rounding = c->rounding;
  p.seed = uint32_t(c->steps);
  const int bx = p.nx < 128 ? ((p.nx + 31) / 32) * 32 : 128;  // row geometry (launch.cuh)
  const bool idle_lanes = ((p.nx + bx - 1) / bx) * bx != p.nx;
  p.linear = (idle_lanes && int64_t(p.nx) * p.ny < (int64_t(1) << 24)) ? 1 : 0;
  p.inv_nx = 1.0f / float(p.nx);
}

// the box {int(min / dx), int(max / dx)} of set_distribution / update_obstacles in real
// coordinates, clipped to the lattice (restrict_box_to_grid, grid.hpp:406-428)
bool clip_box(const hlbm_ctx* c, const double mn[3], const double mx[3], int lo[3], int hi[3]) {
  for (int d = 0; d < 3; d++) {
    lo[d] = int(mn[d] / c->dx);
    hi[d] = int(mx[d] / c->dx);
    if (hi[d] < 0 || lo[d] > c->n[d] - 1) return false;
  }
  for (int d = 0; d < 3; d++) {
    lo[d] = lo[d] < 0 ? 0 : lo[d];
    hi[d] = hi[d] > c->n[d] - 1 ? c->n[d] - 1 : hi[d];
  }
  return true;
}

// Tiles of whole x-rows of about 512 nodes (256 in FP64); stages of one CTA per SM fit 226 KB of
// shared memory, of two CTAs per SM 112 KB each; at least two stages are needed.
bool pipeline_geometry(int nx, int ny, size_t es, int& rows, int& stages1, int& stages2) {
  if ((size_t(nx) * es) % 16 != 0) return false;
  const int target = es == 8 ? 256 : 512;
  rows = target / nx;
  rows = rows < 1 ? 1 : (rows > 32 ? 32 : rows);
  if (rows > ny) rows = ny;
  const size_t stage_bytes = size_t(Q) * rows * nx * es;
  const size_t head = tma_head_bytes();
  stages1 = int((226 * 1024 - head) / stage_bytes);
  stages2 = int((112 * 1024 - head) / stage_bytes);
  stages1 = stages1 > 4 ? 4 : stages1;
  stages2 = stages2 > 4 ? 4 : stages2;
  return stages1 >= 2;
}

// Tile list and stage geometry of the pipelined kernel (lbm_step_tma.cuh).
int setup_pipeline(hlbm_ctx* c) {
  const StepPlan& p = c->plan;
  if (!c->plan_dev) {
    if (pool_alloc((void**)&c->plan_dev, sizeof(StepPlan), c->device, c->stream) != cudaSuccess ||
        pool_alloc((void**)&c->desc_dev, sizeof(LatticeDesc), c->device, c->stream) != cudaSuccess)
      return fail(HLBM_ENOMEM, "cannot allocate the step plan");
  }
  HLBM_CK(cudaMemcpyAsync(c->plan_dev, &p, sizeof(StepPlan), cudaMemcpyHostToDevice, c->stream));
  LatticeDesc d{};
  d.plan = c->plan_dev;
  d.f[0] = c->f[0];
  d.f[1] = c->f[1];
  d.flags = c->flags;
  d.cur = 0;
  HLBM_CK(cudaMemcpyAsync(c->desc_dev, &d, sizeof(d), cudaMemcpyHostToDevice, c->stream));
  c->tma_stages = 0;
  c->tma_stages2 = 0;
  const size_t es = elem_size(c->precision);
  int rows = 0, stages1 = 0, stages2 = 0;
  if (!pipeline_geometry(p.nx, p.ny, es, rows, stages1, stages2)) return HLBM_OK;
  const int tile_elems = rows * p.nx;
  const int stages = stages1;
  std::vector<Tile> tiles;
  for (int z = 0; z < p.nz; z++)
    for (int y0 = 0; y0 < p.ny; y0 += rows) tiles.push_back(make_int4(0, z, y0, (p.ny - y0) < rows ? (p.ny - y0) : rows));
  if (int(tiles.size()) != c->ntiles) {
    pool_free(c->tiles_dev, c->stream);
    c->tiles_dev = nullptr;
    if (pool_alloc((void**)&c->tiles_dev, tiles.size() * sizeof(Tile), c->device, c->stream) != cudaSuccess)
      return fail(HLBM_ENOMEM, "cannot allocate the tile list");
  }
  HLBM_CK(cudaMemcpyAsync(c->tiles_dev, tiles.data(), tiles.size() * sizeof(Tile), cudaMemcpyHostToDevice, c->stream));
  HLBM_CK(cudaStreamSynchronize(c->stream));
  c->ntiles = int(tiles.size());
  c->tile_elems = tile_elems;
  c->tma_stages = stages;
  c->tma_stages2 = stages2;
  return HLBM_OK;
}

int build_plan(hlbm_ctx* c) {
  if (!c->plan_dirty) return HLBM_OK;
  StepPlan& p = c->plan;
  base_plan(c, p);
  p.collision = c->collision;
  p.tau = c->tau;
  p.inv_tau = 1.0 / c->tau;
  for (int d = 0; d < 3; d++) p.F[d] = c->Fext[d];
  p.has_force = (c->Fext[0] != 0.0 || c->Fext[1] != 0.0 || c->Fext[2] != 0.0) ? 1 : 0;
  for (int i = 0; i < Q; i++) {
    p.fw3[i] = 3. * W_OF(i) * (D3Q19::ex[i] * c->Fext[0] + D3Q19::ey[i] * c->Fext[1] + D3Q19::ez[i] * c->Fext[2]);
    p.ffw3[i] = float(p.fw3[i]);
  }
  for (int k = 0; k < 8; k++) p.mrt[k] = c->mrt[k];
  bool pre_seen = false;
  for (const HookOp& h : c->hooks) {
    if (h.hook == HLBM_HOOK_PRE_STREAM) {
      if (h.kind == H_PRE_BB) {
        pre_seen = true;
      } else if (h.kind == H_WALL_BB) {
        p.walls = 1;
      } else if (h.kind == H_CAVITY) {
        // cavity<DIMZ,S,19>::compute_coeff (cavity.hpp:55-72): L = nodes along z
        const int face = h.face ? 5 : 4;
        if (!pre_seen || c->periodic[2]) continue;  // edits a buffer that pre_bounce_back rewrites / none
        if (p.ncav[face] >= MAX_CAVITY) return fail(HLBM_EPLAN, "too many cavity operators on one face");
        static const int ids[2][5] = {{5, 14, 11, 18, 15}, {6, 13, 12, 17, 16}};
        const double L = c->n[2];
        const double uxx = h.u[0] * (1 + 0.5 / (L - 1));
        const double uyy = h.u[1] * (1 + 0.5 / (L - 1));
        const double uzz = h.u[2] * (1 + 0.5 / (L - 1));
        for (int k = 0; k < 5; k++) {
          const int i = ids[h.face ? 1 : 0][k];
          p.cav[face][p.ncav[face]][k] =
              6. * W_OF(i) * (D3Q19::ex[i] * uxx + D3Q19::ey[i] * uyy + D3Q19::ez[i] * uzz);
        }
        p.ncav[face]++;
      }
    }
  }
  for (int stage : {HLBM_HOOK_POST_STREAM, HLBM_HOOK_BOUNDARY_CONDITIONS}) {
    for (const HookOp& h : c->hooks) {
      if (h.hook != stage) continue;
      if (p.nops >= MAX_PLANE_OPS) return fail(HLBM_EPLAN, "too many boundary operators");
      PlaneOp& op = p.ops[p.nops];
      if (h.kind == H_POST_BB) {
        if (!pre_seen)
          return fail(HLBM_EPLAN,
                      "post_bounce_back needs pre_bounce_back in pre_stream_bcs (it restores the saved populations)");
        op.kind = OP_POST_BB;
        op.face = 0;
      } else if (h.kind == H_ZERO_GRADIENT) {
        op.kind = OP_ZERO_GRADIENT;
        op.face = h.face;
      } else {
        op.kind = h.kind == H_LID ? OP_LID : OP_ZOUHE;
        op.face = h.face;
        for (int d = 0; d < 3; d++) op.u[d] = h.u[d] / c->celerity;  // convert_velocity<LBM_UNITS>
      }
      p.nops++;
    }
  }
  for (const HookOp& h : c->hooks) {
    if (h.hook != HLBM_HOOK_START_ITERATION) continue;
    int lo[3], hi[3];
    if (!clip_box(c, h.bounds, h.bounds + 3, lo, hi)) continue;
    if (p.nsets >= MAX_SETS) return fail(HLBM_EPLAN, "too many start_iteration set_distribution operators");
    SetBox& b = p.sets[p.nsets++];
    for (int d = 0; d < 3; d++) {
      b.lo[d] = lo[d];
      b.hi[d] = hi[d];
    }
    b.value = h.value;
  }
  p.face_mask = face_pass_mask(p);
  if (int rc = setup_pipeline(c)) return rc;
  c->plan_dirty = false;
  c->plan_version++;
  return HLBM_OK;
}

// the zero-gradient outlet passes of a plan: every pull of a step (or a read-out) sees them
cudaError_t outlet_passes(int prec, const StepPlan& p, const LatticeDesc* descs, int m, int parity, const int n[3],
                          cudaStream_t s, int64_t& launches) {
  for (int o = 0; o < p.nops; o++) {
    if (p.ops[o].kind != OP_ZERO_GRADIENT) continue;
    launches++;
    if (cudaError_t e = launch_zero_gradient(prec, descs, m, p.ops[o].face, parity, n, s)) return e;
  }
  return cudaSuccess;
}

// One step (or read-out) of lattice c with plan p on stream s: the outlet passes, then the step
// kernel of `variant`.
cudaError_t launch_with_plan(hlbm_ctx* c, int mode, const void* fin, void* fout, const StepPlan& p, int variant,
                             cudaStream_t s) {
  if (mode != MODE_PROLOGUE)  // the descriptor holds f[0], f[1] with cur = 0
    if (cudaError_t e = outlet_passes(c->precision, p, c->desc_dev, 0, fin == c->f[0] ? 0 : 1, c->n, s,
                                      c->launches))
      return e;
  const int walls = p.walls;
  TmaArgs t;
  t.desc = c->desc_dev;
  t.tiles = c->tiles_dev;
  t.ntiles = c->ntiles;
  t.tile_elems = c->tile_elems;
  // variant 6: two CTAs per SM when two CTAs' stages fit, variant 7: one CTA, deeper staging
  t.ctas_per_sm = (variant == 6 && c->tma_stages2 >= 2) ? 2 : 1;
  t.stages = t.ctas_per_sm == 2 ? c->tma_stages2 : c->tma_stages;
  t.parity = (fin == c->f[0]) ? 0 : 1;
  t.err = c->err_dev;
  t.wait_limit = c->wait_limit;
  t.grid = std::min(c->ntiles, c->sms * t.ctas_per_sm);
  t.seed = p.seed;
  t.rows = true;
  t.sms = c->sms;
  const int bytes = int(elem_size(c->precision));
  c->launches++;
  if (rows_runs(p, variant, mode, bytes)) {  // the row pipeline, then the face pass and the wall fix-up
    if (p.face_mask != 0) c->launches++;
    if (walls) c->launches++;
  } else {
    if (variant >= 8) variant = 5;  // what launch_step runs for variants 8 and 9 here
    if (face_pass_runs(p, walls, variant, mode == MODE_PROLOGUE, bytes))
      c->launches++;  // the face pass after the step kernel
    if (walls && mode != MODE_PROLOGUE && variant < 6 && variant % 2 == 1 && vec_eligible_bytes(p, walls, bytes, variant))
      c->launches++;  // the wall fix-up after the vectorised kernel
  }
  switch (c->precision) {
    case HLBM_F64: return step_f64(mode, walls, fin, fout, c->flags, p, s, variant, t);
    case HLBM_F64_STRICT: return step_f64_strict(mode, walls, fin, fout, c->flags, p, s, variant, t);
    case HLBM_F32: return step_f32(mode, walls, fin, fout, c->flags, p, s, variant, t);
    case HLBM_F16: return step_f16(mode, walls, fin, fout, c->flags, p, s, variant, t);
    default: return step_bf16(mode, walls, fin, fout, c->flags, p, s, variant, t);
  }
}

cudaError_t launch_step_variant(hlbm_ctx* c, int mode, const void* fin, void* fout, int variant) {
  c->plan.seed = uint32_t(c->steps);  // the step number salts the stochastic rounding
  return launch_with_plan(c, mode, fin, fout, c->plan, variant, c->stream);
}

// a pipelined-kernel wait that timed out leaves a code in the device error word
int check_device_error(hlbm_ctx* c) {
  int e = 0;
  HLBM_CK(cudaMemcpyAsync(&e, c->err_dev, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  HLBM_CK(cudaStreamSynchronize(c->stream));
  if (e != 0) {
    cudaMemsetAsync(c->err_dev, 0, sizeof(int), c->stream);
    return fail(HLBM_ECUDA, "step kernel: a shared-memory pipeline wait timed out (error " + std::to_string(e) + ")");
  }
  return HLBM_OK;
}

cudaError_t launch_step_kernel(hlbm_ctx* c, int mode, const void* fin, void* fout) {
  return launch_step_variant(c, mode, fin, fout, c->variant);
}

// the vectorised kernel of `variant` applies (d3q19.cuh: vec_eligible_bytes)
bool vec_applies(const hlbm_ctx* c, int variant) {
  return vec_eligible_bytes(c->plan, c->plan.walls, int(elem_size(c->precision)), variant);
}

// make S_k available; returns the buffer holding it
int state_buffer(hlbm_ctx* c, void** out) {
  if (int rc = check_device_error(c)) return rc;
  if (c->phase == RAW) {
    *out = c->f[c->cur];
    return HLBM_OK;
  }
  if (c->phase == POSTCOL) {
    int rc = build_plan(c);
    if (rc) return rc;
    HLBM_CK(launch_step_kernel(c, MODE_FINISH, c->f[c->cur], c->f[1 - c->cur]));
    c->phase = MATER;
  }
  *out = c->f[1 - c->cur];
  return HLBM_OK;
}

// turn the context into RAW (S_k in f[cur]) so that S can be edited in place
int make_raw(hlbm_ctx* c) {
  if (c->phase == RAW) return HLBM_OK;
  void* s;
  int rc = state_buffer(c, &s);
  if (rc) return rc;
  c->cur = 1 - c->cur;
  c->phase = RAW;
  return HLBM_OK;
}

int set_device(hlbm_ctx* c) {
  HLBM_CK(cudaSetDevice(c->device));
  return HLBM_OK;
}

int add_hook(hlbm_ctx* c, HookOp h) {
  c->hooks.push_back(h);
  c->plan_dirty = true;
  return HLBM_OK;
}
}  // namespace

extern "C" {

const char* hlbm_last_error(void) { return g_err.c_str(); }
const char* hlbm_version(void) { return "hippolbm-b200 0.1.0 (sm_100a)"; }

// Default step-kernel variant of a tier and collision: hlbm_autotune's pick on 512^3 Couette on a
// B200.  FP64: one node per thread at >= 3 blocks/SM (4); FP32: 16-byte vectors at one block/SM
// (1); FP16 / BF16: the row pipeline at two CTAs/SM (8) for BGK, one CTA/SM (9) for MRT (lattices
// the row pipeline does not take run variant 5).
static int default_variant(int precision, int collision) {
  if (precision == HLBM_F64 || precision == HLBM_F64_STRICT) return 4;
  if (precision == HLBM_F32) return 1;
  (void)collision;
  return 9;
}

int hlbm_domain(const int32_t cell_dims[3], const double bmin[3], const double bmax[3], const int32_t periodic[3],
                int32_t precision, int32_t device, hlbm_ctx** out) {
  if (!cell_dims || !bmin || !bmax || !periodic || !out) return fail(HLBM_EINVAL, "hlbm_domain: NULL argument");
  *out = nullptr;
  if (precision < HLBM_F64 || precision > HLBM_BF16) return fail(HLBM_EINVAL, "hlbm_domain: unknown precision");
  int n[3];
  for (int d = 0; d < 3; d++) {
    if (cell_dims[d] < 1) return fail(HLBM_EDOMAIN, "[Error, domain], cell_dims must be >= 1");
    n[d] = cell_dims[d] + 1;  // domain_lbm.cpp:68
  }
  double reso[3];
  for (int d = 0; d < 3; d++) reso[d] = (bmax[d] - bmin[d]) / double(n[d] - 1);
  if (reso[0] != reso[1] || reso[0] != reso[2]) return fail(HLBM_EDOMAIN, "[Error, domain], Dx is not the same for all dimension");
  for (int d = 0; d < 3; d++)
    if (bmin[d] + (n[d] - 1) * reso[0] != bmax[d])
      return fail(HLBM_EDOMAIN, "[Error, domain], The resolution slot and bounds slot mismatch.");
  auto* c = new hlbm_ctx();
  for (int d = 0; d < 3; d++) {
    c->n[d] = n[d];
    c->periodic[d] = periodic[d] ? 1 : 0;
    c->bmin[d] = bmin[d];
    c->bmax[d] = bmax[d];
  }
  c->dx = (bmax[0] - bmin[0]) / double(n[0] - 1);  // load_balancing GridDx, make_domain.hpp:280
  c->precision = precision;
  c->device = device;
  c->ncell = int64_t(n[0]) * n[1] * n[2];
  c->stride = (c->ncell + 127) / 128 * 128;
  if (precision == HLBM_F16) c->scale = 1024.0;
  c->variant = default_variant(precision, 0);
  mrt_reference(c->mrt);
  auto cleanup = [&](int rc) {
    hlbm_destroy(c);
    return rc;
  };
  if (int rc = set_device(c)) return cleanup(rc);
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
    return cleanup(fail(HLBM_ECUDA, "cudaStreamCreate failed"));
  const size_t fbytes = size_t(Q) * c->stride * elem_size(precision);
  for (int k = 0; k < 2; k++)
    if (pool_alloc(&c->f[k], fbytes, c->device, c->stream) != cudaSuccess) {
      cudaGetLastError();
      return cleanup(fail(HLBM_ENOMEM, "hlbm_domain: cannot allocate " + std::to_string(fbytes >> 20) +
                                           " MiB of populations"));
    }
  cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device);
  if (pool_alloc((void**)&c->err_dev, sizeof(int), c->device, c->stream) != cudaSuccess ||
      cudaMemsetAsync(c->err_dev, 0, sizeof(int), c->stream) != cudaSuccess) {
    cudaGetLastError();
    return cleanup(fail(HLBM_ENOMEM, "hlbm_domain: cannot allocate the error word"));
  }
  // the flag bytes are padded to 128 (the span pipeline bulk-copies whole 16-byte chunks of them)
  const size_t flag_bytes = size_t((c->ncell + 127) / 128 * 128);
  if (pool_alloc((void**)&c->flags, flag_bytes, c->device, c->stream) != cudaSuccess ||
      pool_alloc((void**)&c->nearwall, size_t(c->ncell), c->device, c->stream) != cudaSuccess ||
      pool_alloc((void**)&c->partials, sizeof(double) * 4 * 148 * 8, c->device, c->stream) != cudaSuccess ||
      pool_alloc((void**)&c->stats_dev, sizeof(double) * 4, c->device, c->stream) != cudaSuccess) {
    cudaGetLastError();
    return cleanup(fail(HLBM_ENOMEM, "hlbm_domain: cannot allocate flags"));
  }
  // init_obst: every flag FLUIDE_ (-1 = 0xff)
  if (cudaMemsetAsync(c->flags, 0xff, flag_bytes, c->stream) != cudaSuccess ||
      cudaMemsetAsync(c->nearwall, 0, size_t(c->ncell), c->stream) != cudaSuccess)
    return cleanup(fail(HLBM_ECUDA, "cudaMemsetAsync failed"));
  // default lbm_parameters slots (lbm_parameters.cpp:57-64)
  const double F0[3] = {0, 0, 0};
  if (int rc = hlbm_lbm_parameters(c, F0, 1.0, 1e-4, 1000.0, 0, 0.0, 0.0)) return cleanup(rc);
  // default set_distribution: value 1 on every node (config_initialize.msp:22-23)
  if (int rc = hlbm_set_distribution(c, 1.0, nullptr, 0)) return cleanup(rc);
  *out = c;
  return HLBM_OK;
}

int hlbm_destroy(hlbm_ctx* c) {
  if (!c) return HLBM_OK;
  if (c->batch) hlbm_batch_remove(c->batch, c);  // a batch never keeps a destroyed member
  cudaSetDevice(c->device);
  if (c->stream) {  // the memory returns to the pool once the stream's work is done
    void* bufs[] = {c->f[0], c->f[1], c->flags, c->nearwall, c->partials, c->stats_dev, c->plane_tmp, c->uprev,
                    c->plan_dev, c->desc_dev, c->tiles_dev, c->err_dev, c->seed_dev};
    for (void* b : bufs) pool_free(b, c->stream);
    cudaStreamDestroy(c->stream);
  }
  if (c->join_ev) cudaEventDestroy(c->join_ev);
  delete c;
  return HLBM_OK;
}

int hlbm_lbm_parameters(hlbm_ctx* c, const double Fext[3], double celerity, double nuth, double avg_rho,
                        int32_t has_tau, double tau, double dt) {
  if (!c || !Fext) return fail(HLBM_EINVAL, "hlbm_lbm_parameters: NULL argument");
  const double dx = c->dx;
  c->nuth = nuth;
  c->avg_rho = avg_rho;
  if (dt > 0.0) {  // define_by_dt (lbm_parameters.hpp:60-66)
    c->dtLB = dt;
    c->tau = 3 * c->nuth * c->dtLB / (dx * dx) + 0.5;
    c->nu = (c->tau - 0.5) / 3.0;
    c->celerity = dx / c->dtLB;
  } else if (has_tau) {  // define_by_tau (lbm_parameters.hpp:68-74)
    c->tau = tau;
    c->dtLB = dx * dx * (c->tau - 0.5) / (3.0 * c->nuth);
    c->nu = c->nuth * c->dtLB / (dx * dx);
    c->celerity = dx / c->dtLB;
  } else {  // define_by_c (lbm_parameters.hpp:76-81)
    c->celerity = celerity;
    c->dtLB = dx / c->celerity;
    c->nu = c->nuth * c->dtLB / (dx * dx);
    c->tau = 3. * c->nu + 0.5;
  }
  const double ddx = c->celerity * c->dtLB;  // convert_force<LBM_UNITS> (lbm_parameters.hpp:124-128)
  for (int d = 0; d < 3; d++) c->Fext[d] = Fext[d] * c->dtLB * c->dtLB / ddx;
  if (!(c->tau > 0.5) || !std::isfinite(c->tau))
    return fail(HLBM_EINVAL, "hlbm_lbm_parameters: tau = " + std::to_string(c->tau) + " must be > 0.5");
  c->plan_dirty = true;
  return HLBM_OK;
}

int hlbm_get_parameters(hlbm_ctx* c, double out[9]) {
  if (!c || !out) return fail(HLBM_EINVAL, "hlbm_get_parameters: NULL argument");
  out[0] = c->Fext[0];
  out[1] = c->Fext[1];
  out[2] = c->Fext[2];
  out[3] = c->celerity;
  out[4] = c->dtLB;
  out[5] = c->nuth;
  out[6] = c->nu;
  out[7] = c->tau;
  out[8] = c->avg_rho;
  return HLBM_OK;
}

// Re-encode the carried state after the storage reference or scale changed (16-bit tiers): each
// stored value is decoded under the old plan and encoded under the new one, on the device.
static int reencode_storage(hlbm_ctx* c, const StepPlan& old_plan) {
  if (c->precision != HLBM_F16 && c->precision != HLBM_BF16) return HLBM_OK;
  if (c->phase == MATER) c->phase = POSTCOL;  // the read-out copy is recomputed when needed
  StepPlan p;
  base_plan(c, p);
  bool same = p.scale == old_plan.scale;
  for (int i = 0; i < Q; i++) same = same && p.dref[i] == old_plan.dref[i];
  if (same) return HLBM_OK;
  c->launches++;
  HLBM_CK(launch_reencode(c->precision, c->f[c->cur], old_plan, p, c->stream));
  return HLBM_OK;
}

int hlbm_collision(hlbm_ctx* c, int32_t kind, const double* rates8) {
  if (!c || (kind != 0 && kind != 1)) return fail(HLBM_EINVAL, "hlbm_collision: kind must be 0 (bgk) or 1 (mrt)");
  if (int rc = set_device(c)) return rc;
  StepPlan old_plan;
  base_plan(c, old_plan);
  c->collision = kind;
  if (!c->variant_tuned) c->variant = default_variant(c->precision, kind);
  if (rates8)
    std::memcpy(c->mrt, rates8, sizeof(c->mrt));
  else
    mrt_reference(c->mrt);
  c->plan_dirty = true;
  return reencode_storage(c, old_plan);  // the 16-bit storage reference follows the collision
}

int hlbm_storage_scale(hlbm_ctx* c, double rho0, double scale) {
  if (!c || !(scale > 0)) return fail(HLBM_EINVAL, "hlbm_storage_scale: scale must be > 0");
  if (int rc = set_device(c)) return rc;
  StepPlan old_plan;
  base_plan(c, old_plan);
  c->rho0 = rho0;
  c->scale = scale;
  c->plan_dirty = true;
  return reencode_storage(c, old_plan);
}

int hlbm_storage_rounding(hlbm_ctx* c, int32_t mode) {
  if (!c || (mode != 0 && mode != 1)) return fail(HLBM_EINVAL, "hlbm_storage_rounding: mode must be 0 or 1");
  c->rounding = mode;
  c->plan_dirty = true;
  return HLBM_OK;
}

int hlbm_set_distribution(hlbm_ctx* c, double value, const double* bounds6, int32_t /*do_update*/) {
  if (!c) return fail(HLBM_EINVAL, "hlbm_set_distribution: NULL context");
  if (int rc = set_device(c)) return rc;
  if (int rc = make_raw(c)) return rc;
  int lo[3] = {0, 0, 0}, hi[3] = {c->n[0] - 1, c->n[1] - 1, c->n[2] - 1};
  if (bounds6 && !clip_box(c, bounds6, bounds6 + 3, lo, hi)) return HLBM_OK;
  StepPlan p;
  base_plan(c, p);
  c->launches++;
  HLBM_CK(launch_set_distribution(c->precision, c->f[c->cur], p, lo, hi, value, c->stream));
  return HLBM_OK;
}

int hlbm_init_double_couette(hlbm_ctx* c, const double U[3], int32_t dim) {
  if (!c || !U) return fail(HLBM_EINVAL, "hlbm_init_double_couette: NULL argument");
  if (dim < 0 || dim > 2)
    return fail(HLBM_EINVAL, "[init_double_couette] Please, select a valid dimension \"X\", \"Y\", or \"Z\".");
  if (int rc = set_device(c)) return rc;
  if (int rc = make_raw(c)) return rc;
  double uc[3], du[3];
  for (int d = 0; d < 3; d++) uc[d] = U[d] / c->celerity;  // init_double_couette.cu:77
  const double half_span = 0.5 * (c->n[dim] - 1);
  for (int d = 0; d < 3; d++) du[d] = uc[d] / half_span;
  StepPlan p;
  base_plan(c, p);
  c->launches++;
  HLBM_CK(launch_double_couette(c->precision, c->f[c->cur], p, dim, uc, du, c->stream));
  return HLBM_OK;
}

int hlbm_init_obstacles(hlbm_ctx* c) {
  if (!c) return fail(HLBM_EINVAL, "hlbm_init_obstacles: NULL context");
  c->obstacles.clear();
  return HLBM_OK;
}

static ObstacleDesc& obstacle_slot(hlbm_ctx* c, int id) {
  if (size_t(id) >= c->obstacles.size()) {  // obstacles.hpp:84-107
    ObstacleDesc none{};
    none.type = OBS_NONE;
    c->obstacles.resize(id + 1, none);
  }
  return c->obstacles[id];
}

int hlbm_register_solid_ball(hlbm_ctx* c, int32_t id, const double center[3], double radius) {
  if (!c || !center || id < 0) return fail(HLBM_EINVAL, "hlbm_register_solid_ball: bad argument");
  ObstacleDesc& o = obstacle_slot(c, id);
  o = ObstacleDesc{};
  o.type = OBS_BALL;
  o.a[0] = center[0];
  o.a[1] = center[1];
  o.a[2] = center[2];
  o.a[3] = radius;
  o.a[4] = radius * radius;  // Ball::r2_
  return HLBM_OK;
}

int hlbm_register_solid_wall(hlbm_ctx* c, int32_t id, const double bmin[3], const double bmax[3]) {
  if (!c || !bmin || !bmax || id < 0) return fail(HLBM_EINVAL, "hlbm_register_solid_wall: bad argument");
  ObstacleDesc& o = obstacle_slot(c, id);
  o = ObstacleDesc{};
  o.type = OBS_WALL;
  for (int d = 0; d < 3; d++) {
    o.a[d] = bmin[d];
    o.a[3 + d] = bmax[d];
  }
  return HLBM_OK;
}

int hlbm_register_quadric(hlbm_ctx* c, int32_t id, const double q[16]) {
  if (!c || !q || id < 0) return fail(HLBM_EINVAL, "hlbm_register_quadric: bad argument");
  ObstacleDesc& o = obstacle_slot(c, id);
  o = ObstacleDesc{};
  o.type = OBS_QUADRIC;
  std::memcpy(o.a, q, sizeof(double) * 16);
  return HLBM_OK;
}

int hlbm_update_obstacles(hlbm_ctx* c) {
  if (!c) return fail(HLBM_EINVAL, "hlbm_update_obstacles: NULL context");
  if (int rc = set_device(c)) return rc;
  StepPlan p;
  base_plan(c, p);
  for (const ObstacleDesc& o : c->obstacles) {  // UpdateObstacles::execute (update_obstacles.cu:106-119)
    if (o.type == OBS_NONE) continue;
    double mn[3], mx[3];
    for (int d = 0; d < 3; d++) {
      if (o.type == OBS_BALL) {  // Ball::covered (obstacle.hpp:46-49)
        mn[d] = o.a[d] - o.a[3];
        mx[d] = o.a[d] + o.a[3];
      } else if (o.type == OBS_WALL) {
        mn[d] = o.a[d];
        mx[d] = o.a[3 + d];
      } else {  // Quadric::covered (obstacle.hpp:119-124)
        mn[d] = -1e6;
        mx[d] = 1e6;
      }
    }
    int lo[3], hi[3];
    if (!clip_box(c, mn, mx, lo, hi)) continue;
    c->launches++;
    HLBM_CK(launch_rasterize(c->flags, p, lo, hi, c->dx, o, c->stream));
    c->maybe_walls = true;
    c->plan_dirty = true;
  }
  return refresh_near_wall(c);
}

// whether a host flag array holds a wall node
static bool any_wall(const int8_t* flags, int64_t n) {
  for (int64_t i = 0; i < n; i++)
    if (flags[i] == FLAG_WALL) return true;
  return false;
}

int hlbm_clear_hooks(hlbm_ctx* c) {
  if (!c) return fail(HLBM_EINVAL, "hlbm_clear_hooks: NULL context");
  c->hooks.clear();
  c->plan_dirty = true;
  return HLBM_OK;
}

int hlbm_pre_bounce_back(hlbm_ctx* c) {
  if (!c) return fail(HLBM_EINVAL, "hlbm_pre_bounce_back: NULL context");
  return add_hook(c, HookOp{HLBM_HOOK_PRE_STREAM, H_PRE_BB, 0, {0, 0, 0}, 0, {0}});
}

int hlbm_cavity(hlbm_ctx* c, int32_t side, const double U[3]) {
  if (!c || !U || (side != 0 && side != 1)) return fail(HLBM_EINVAL, "hlbm_cavity: side must be 0 (z_0) or 1 (z_l)");
  return add_hook(c, HookOp{HLBM_HOOK_PRE_STREAM, H_CAVITY, side, {U[0], U[1], U[2]}, 0, {0}});
}

int hlbm_wall_bounce_back(hlbm_ctx* c) {
  if (!c) return fail(HLBM_EINVAL, "hlbm_wall_bounce_back: NULL context");
  return add_hook(c, HookOp{HLBM_HOOK_PRE_STREAM, H_WALL_BB, 0, {0, 0, 0}, 0, {0}});
}

static bool post_hook(int32_t hook) {
  return hook == HLBM_HOOK_POST_STREAM || hook == HLBM_HOOK_BOUNDARY_CONDITIONS;
}

int hlbm_post_bounce_back(hlbm_ctx* c, int32_t hook) {
  if (!c || !post_hook(hook)) return fail(HLBM_EINVAL, "hlbm_post_bounce_back: hook must be post_stream_bcs or boundary_conditions");
  return add_hook(c, HookOp{hook, H_POST_BB, 0, {0, 0, 0}, 0, {0}});
}

static int plane_hooks(hlbm_ctx* c, int32_t hook, int kind, const double U[3], const int32_t* regions, int32_t nreg,
                       const char* name) {
  if (!c || !U || !regions || nreg < 0 || !post_hook(hook))
    return fail(HLBM_EINVAL, std::string(name) + ": bad argument");
  for (int i = 0; i < nreg; i++) {  // check_traversal_allowed (grid_region.hpp:381-387)
    if (regions[i] < 0 || regions[i] > 5) return fail(HLBM_EINVAL, std::string(name) + ": Traversal name not allowed");
    if (kind == H_ZERO_GRADIENT && c->n[regions[i] / 2] < 2)  // the interior neighbour must exist
      return fail(HLBM_EINVAL, std::string(name) + ": the face needs at least two nodes along its normal");
    add_hook(c, HookOp{hook, kind, regions[i], {U[0], U[1], U[2]}, 0, {0}});
  }
  return HLBM_OK;
}

int hlbm_neumann(hlbm_ctx* c, int32_t hook, const double U[3], const int32_t* regions, int32_t nregions) {
  return plane_hooks(c, hook, H_NEUMANN, U, regions, nregions, "hlbm_neumann");
}

int hlbm_lid_driven_cavity(hlbm_ctx* c, int32_t hook, const double U[3], const int32_t* regions, int32_t nregions) {
  return plane_hooks(c, hook, H_LID, U, regions, nregions, "hlbm_lid_driven_cavity");
}

int hlbm_zero_gradient(hlbm_ctx* c, int32_t hook, const int32_t* regions, int32_t nregions) {
  const double zero[3] = {0, 0, 0};
  return plane_hooks(c, hook, H_ZERO_GRADIENT, zero, regions, nregions, "hlbm_zero_gradient");
}

int hlbm_start_set_distribution(hlbm_ctx* c, double value, const double bounds6[6]) {
  if (!c || !bounds6) return fail(HLBM_EINVAL, "hlbm_start_set_distribution: bounds are required");
  HookOp h{HLBM_HOOK_START_ITERATION, H_SETDIST, 0, {0, 0, 0}, value, {0}};
  std::memcpy(h.bounds, bounds6, sizeof(h.bounds));
  return add_hook(c, h);
}

int hlbm_step(hlbm_ctx* c, int64_t nsteps) {
  if (!c || nsteps < 0) return fail(HLBM_EINVAL, "hlbm_step: bad argument");
  if (nsteps == 0) return HLBM_OK;
  if (int rc = set_device(c)) return rc;
  if (int rc = build_plan(c)) return rc;
  if (c->phase == MATER) c->phase = POSTCOL;
  if (c->phase == RAW) {
    HLBM_CK(launch_step_kernel(c, MODE_PROLOGUE, c->f[c->cur], c->f[1 - c->cur]));
    c->cur = 1 - c->cur;
    c->phase = POSTCOL;
    c->steps++;
    nsteps--;
  }
  for (int64_t s = 0; s < nsteps; s++) {
    HLBM_CK(launch_step_kernel(c, MODE_FUSED, c->f[c->cur], c->f[1 - c->cur]));
    c->cur = 1 - c->cur;
    c->steps++;
  }
  return HLBM_OK;
}

int hlbm_sync(hlbm_ctx* c) {
  if (!c) return fail(HLBM_EINVAL, "hlbm_sync: NULL context");
  HLBM_CK(cudaStreamSynchronize(c->stream));
  return check_device_error(c);
}

int hlbm_macro_variables(hlbm_ctx* c, double* rho, double* u) {
  if (!c) return fail(HLBM_EINVAL, "hlbm_macro_variables: NULL context");
  if (int rc = set_device(c)) return rc;
  void* s;
  if (int rc = state_buffer(c, &s)) return rc;
  double *drho = nullptr, *du = nullptr;
  const size_t n = size_t(c->ncell);
  if (rho && pool_alloc((void**)&drho, n * 8, c->device, c->stream) != cudaSuccess)
    return fail(HLBM_ENOMEM, "hlbm_macro_variables: no memory");
  if (u && pool_alloc((void**)&du, 3 * n * 8, c->device, c->stream) != cudaSuccess) {
    pool_free(drho, c->stream);
    return fail(HLBM_ENOMEM, "hlbm_macro_variables: no memory");
  }
  StepPlan p;
  base_plan(c, p);
  c->launches += 2;
  cudaError_t e = launch_macro_stats(c->precision, s, c->flags, p, drho, du, c->partials, c->stats_dev, c->stream);
  if (e == cudaSuccess && rho) e = cudaMemcpyAsync(rho, drho, n * 8, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess && u) e = cudaMemcpyAsync(u, du, 3 * n * 8, cudaMemcpyDeviceToHost, c->stream);
  pool_free(drho, c->stream);
  pool_free(du, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return fail(HLBM_ECUDA, std::string("hlbm_macro_variables: ") + cudaGetErrorString(e));
  return HLBM_OK;
}

int hlbm_simulation_state(hlbm_ctx* c, double out[3]) {
  if (!c || !out) return fail(HLBM_EINVAL, "hlbm_simulation_state: NULL argument");
  if (int rc = set_device(c)) return rc;
  void* s;
  if (int rc = state_buffer(c, &s)) return rc;
  StepPlan p;
  base_plan(c, p);
  c->launches += 2;
  HLBM_CK(launch_macro_stats(c->precision, s, c->flags, p, nullptr, nullptr, c->partials, c->stats_dev, c->stream));
  HLBM_CK(cudaMemcpyAsync(out, c->stats_dev, 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  HLBM_CK(cudaStreamSynchronize(c->stream));
  return HLBM_OK;
}

int hlbm_residual(hlbm_ctx* c, double* out) {
  if (!c || !out) return fail(HLBM_EINVAL, "hlbm_residual: NULL argument");
  if (int rc = set_device(c)) return rc;
  void* s;
  if (int rc = state_buffer(c, &s)) return rc;
  int first = 0;
  if (!c->uprev) {
    if (pool_alloc((void**)&c->uprev, size_t(c->ncell) * 3 * sizeof(float), c->device, c->stream) != cudaSuccess)
      return fail(HLBM_ENOMEM, "hlbm_residual: no memory for the velocity snapshot");
    first = 1;
  }
  StepPlan p;
  base_plan(c, p);
  c->launches += 2;
  double h[4];
  HLBM_CK(launch_residual(c->precision, s, c->flags, p, c->uprev, first, c->partials, c->stats_dev, c->stream));
  HLBM_CK(cudaMemcpyAsync(h, c->stats_dev, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  HLBM_CK(cudaStreamSynchronize(c->stream));
  *out = first ? HUGE_VAL : (h[1] > 0 ? std::sqrt(h[0] / h[1]) : (h[0] > 0 ? HUGE_VAL : 0.0));
  return HLBM_OK;
}

int hlbm_moments(hlbm_ctx* c, double out[4]) {
  if (!c || !out) return fail(HLBM_EINVAL, "hlbm_moments: NULL argument");
  if (int rc = set_device(c)) return rc;
  void* s;
  if (int rc = state_buffer(c, &s)) return rc;
  StepPlan p;
  base_plan(c, p);
  c->launches += 2;
  HLBM_CK(launch_moments(c->precision, s, c->flags, p, c->partials, c->stats_dev, c->stream));
  HLBM_CK(cudaMemcpyAsync(out, c->stats_dev, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  HLBM_CK(cudaStreamSynchronize(c->stream));
  return HLBM_OK;
}

int hlbm_wall_force(hlbm_ctx* c, double out[3]) {
  if (!c || !out) return fail(HLBM_EINVAL, "hlbm_wall_force: NULL argument");
  if (c->phase == RAW) return fail(HLBM_ESTATE, "hlbm_wall_force: needs a post-collision state (step once first)");
  if (int rc = set_device(c)) return rc;
  if (int rc = check_device_error(c)) return rc;
  StepPlan p;
  base_plan(c, p);
  c->launches += 2;
  double h[4];
  HLBM_CK(launch_wall_force(c->precision, c->f[c->cur], c->flags, p, c->partials, c->stats_dev, c->stream));
  HLBM_CK(cudaMemcpyAsync(h, c->stats_dev, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  HLBM_CK(cudaStreamSynchronize(c->stream));
  out[0] = h[0];
  out[1] = h[1];
  out[2] = h[2];
  return HLBM_OK;
}

int hlbm_get_populations(hlbm_ctx* c, double* out) {
  if (!c || !out) return fail(HLBM_EINVAL, "hlbm_get_populations: NULL argument");
  if (int rc = set_device(c)) return rc;
  void* s;
  if (int rc = state_buffer(c, &s)) return rc;
  const size_t n = size_t(c->ncell);
  if (elem_size(c->precision) == 8) {
    HLBM_CK(cudaMemcpy2DAsync(out, n * 8, s, size_t(c->stride) * 8, n * 8, Q, cudaMemcpyDeviceToHost, c->stream));
  } else {
    if (!c->plane_tmp && pool_alloc((void**)&c->plane_tmp, n * 8, c->device, c->stream) != cudaSuccess)
      return fail(HLBM_ENOMEM, "hlbm_get_populations: no memory");
    StepPlan p;
    base_plan(c, p);
    for (int i = 0; i < Q; i++) {
      c->launches++;
      HLBM_CK(launch_decode(c->precision, s, c->plane_tmp, i, p, c->stream));
      HLBM_CK(cudaMemcpyAsync(out + i * n, c->plane_tmp, n * 8, cudaMemcpyDeviceToHost, c->stream));
    }
  }
  HLBM_CK(cudaStreamSynchronize(c->stream));
  return HLBM_OK;
}

int hlbm_put_populations(hlbm_ctx* c, const double* in) {
  if (!c || !in) return fail(HLBM_EINVAL, "hlbm_put_populations: NULL argument");
  if (int rc = set_device(c)) return rc;
  const size_t n = size_t(c->ncell);
  c->phase = RAW;
  if (elem_size(c->precision) == 8) {
    HLBM_CK(cudaMemcpy2DAsync(c->f[c->cur], size_t(c->stride) * 8, in, n * 8, n * 8, Q, cudaMemcpyHostToDevice,
                              c->stream));
  } else {
    if (!c->plane_tmp && pool_alloc((void**)&c->plane_tmp, n * 8, c->device, c->stream) != cudaSuccess)
      return fail(HLBM_ENOMEM, "hlbm_put_populations: no memory");
    StepPlan p;
    base_plan(c, p);
    for (int i = 0; i < Q; i++) {
      HLBM_CK(cudaMemcpyAsync(c->plane_tmp, in + i * n, n * 8, cudaMemcpyHostToDevice, c->stream));
      c->launches++;
      HLBM_CK(launch_encode(c->precision, c->f[c->cur], c->plane_tmp, i, p, c->stream));
    }
  }
  HLBM_CK(cudaStreamSynchronize(c->stream));
  return HLBM_OK;
}

int hlbm_get_flags(hlbm_ctx* c, int8_t* out) {
  if (!c || !out) return fail(HLBM_EINVAL, "hlbm_get_flags: NULL argument");
  if (int rc = set_device(c)) return rc;
  HLBM_CK(cudaMemcpyAsync(out, c->flags, size_t(c->ncell), cudaMemcpyDeviceToHost, c->stream));
  HLBM_CK(cudaStreamSynchronize(c->stream));
  return HLBM_OK;
}

int hlbm_put_flags(hlbm_ctx* c, const int8_t* in) {
  if (!c || !in) return fail(HLBM_EINVAL, "hlbm_put_flags: NULL argument");
  if (int rc = set_device(c)) return rc;
  HLBM_CK(cudaMemcpyAsync(c->flags, in, size_t(c->ncell), cudaMemcpyHostToDevice, c->stream));
  if (int rc = refresh_near_wall(c)) return rc;
  c->maybe_walls = any_wall(in, c->ncell);
  c->plan_dirty = true;
  HLBM_CK(cudaStreamSynchronize(c->stream));
  return HLBM_OK;
}

int hlbm_plane_velocity_profile(hlbm_ctx* c, int32_t dim, double* avg, double* vmin, double* vmax, int64_t* count) {
  if (!c || dim < 0 || dim > 2) return fail(HLBM_EINVAL, "hlbm_plane_velocity_profile: dimension must be 0, 1 or 2");
  if (int rc = set_device(c)) return rc;
  void* s;
  if (int rc = state_buffer(c, &s)) return rc;
  const int n = c->n[dim];
  double* dev = nullptr;
  if (pool_alloc((void**)&dev, size_t(4) * n * sizeof(double), c->device, c->stream) != cudaSuccess)
    return fail(HLBM_ENOMEM, "hlbm_plane_velocity_profile: no memory");
  std::vector<double> host(size_t(4) * n);
  StepPlan p;
  base_plan(c, p);
  c->launches++;
  cudaError_t e = launch_plane_profile(c->precision, s, c->flags, p, dim, c->dx / c->dtLB, dev, c->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(host.data(), dev, host.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  pool_free(dev, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return fail(HLBM_ECUDA, std::string("hlbm_plane_velocity_profile: ") + cudaGetErrorString(e));
  for (int i = 0; i < n; i++) {
    const double sum = host[4 * i], cnt = host[4 * i + 1];
    if (avg) avg[i] = cnt > 0 ? sum / cnt : 0.0;  // plane_velocity_profile.cu:206-212
    if (vmin) vmin[i] = host[4 * i + 2];
    if (vmax) vmax[i] = host[4 * i + 3];
    if (count) count[i] = int64_t(cnt);
  }
  return HLBM_OK;
}

// ------------------------------------------------------------------ checkpoint / restore
namespace {
struct CheckpointHeader {
  char magic[8];  // "HLBMCKP1"
  int32_t version, precision;
  int32_t n[3], periodic[3];
  int32_t phase, rounding;
  int64_t steps, ncell;
  double rho0, scale;
};
constexpr char CKPT_MAGIC[8] = {'H', 'L', 'B', 'M', 'C', 'K', 'P', '1'};
int64_t checkpoint_bytes(const hlbm_ctx* c) {
  return int64_t(sizeof(CheckpointHeader)) + c->ncell + int64_t(Q) * c->ncell * int64_t(elem_size(c->precision));
}
}  // namespace

int hlbm_checkpoint_bytes(hlbm_ctx* c, int64_t* bytes) {
  if (!c || !bytes) return fail(HLBM_EINVAL, "hlbm_checkpoint_bytes: NULL argument");
  *bytes = checkpoint_bytes(c);
  return HLBM_OK;
}

int hlbm_checkpoint_save(hlbm_ctx* c, void* host, int64_t bytes) {
  if (!c || !host) return fail(HLBM_EINVAL, "hlbm_checkpoint_save: NULL argument");
  if (bytes < checkpoint_bytes(c)) return fail(HLBM_EINVAL, "hlbm_checkpoint_save: buffer too small");
  if (int rc = set_device(c)) return rc;
  if (int rc = check_device_error(c)) return rc;
  if (c->phase == MATER) c->phase = POSTCOL;  // f[cur] holds the carried state in every phase
  CheckpointHeader h{};
  std::memcpy(h.magic, CKPT_MAGIC, 8);
  h.version = 1;
  h.precision = c->precision;
  for (int d = 0; d < 3; d++) {
    h.n[d] = c->n[d];
    h.periodic[d] = c->periodic[d];
  }
  h.phase = c->phase;
  h.rounding = c->rounding;
  h.steps = c->steps;
  h.ncell = c->ncell;
  h.rho0 = c->rho0;
  h.scale = c->scale;
  unsigned char* out = static_cast<unsigned char*>(host);
  std::memcpy(out, &h, sizeof(h));
  out += sizeof(h);
  const size_t n = size_t(c->ncell), es = elem_size(c->precision);
  HLBM_CK(cudaMemcpyAsync(out, c->flags, n, cudaMemcpyDeviceToHost, c->stream));
  out += n;
  HLBM_CK(cudaMemcpy2DAsync(out, n * es, c->f[c->cur], size_t(c->stride) * es, n * es, Q, cudaMemcpyDeviceToHost,
                            c->stream));
  HLBM_CK(cudaStreamSynchronize(c->stream));
  return HLBM_OK;
}

int hlbm_checkpoint_load(hlbm_ctx* c, const void* host, int64_t bytes) {
  if (!c || !host) return fail(HLBM_EINVAL, "hlbm_checkpoint_load: NULL argument");
  if (bytes < int64_t(sizeof(CheckpointHeader))) return fail(HLBM_EINVAL, "hlbm_checkpoint_load: truncated header");
  CheckpointHeader h;
  std::memcpy(&h, host, sizeof(h));
  if (std::memcmp(h.magic, CKPT_MAGIC, 8) != 0 || h.version != 1)
    return fail(HLBM_EINVAL, "hlbm_checkpoint_load: not a checkpoint of this library");
  if (h.precision != c->precision) return fail(HLBM_EINVAL, "hlbm_checkpoint_load: precision differs");
  for (int d = 0; d < 3; d++)
    if (h.n[d] != c->n[d] || h.periodic[d] != c->periodic[d])
      return fail(HLBM_EDOMAIN, "hlbm_checkpoint_load: lattice shape or periodicity differs");
  if (h.phase != RAW && h.phase != POSTCOL) return fail(HLBM_EINVAL, "hlbm_checkpoint_load: bad phase");
  if (bytes < checkpoint_bytes(c)) return fail(HLBM_EINVAL, "hlbm_checkpoint_load: truncated data");
  if (int rc = set_device(c)) return rc;
  const unsigned char* in = static_cast<const unsigned char*>(host) + sizeof(h);
  const size_t n = size_t(c->ncell), es = elem_size(c->precision);
  HLBM_CK(cudaMemcpyAsync(c->flags, in, n, cudaMemcpyHostToDevice, c->stream));
  if (int rc = refresh_near_wall(c)) return rc;
  c->maybe_walls = any_wall(reinterpret_cast<const int8_t*>(in), int64_t(n));
  in += n;
  HLBM_CK(cudaMemcpy2DAsync(c->f[c->cur], size_t(c->stride) * es, in, n * es, n * es, Q, cudaMemcpyHostToDevice,
                            c->stream));
  HLBM_CK(cudaStreamSynchronize(c->stream));
  c->phase = h.phase;
  c->steps = h.steps;
  c->rounding = h.rounding;
  c->rho0 = h.rho0;  // the stored deviations are relative to these
  c->scale = h.scale;
  c->plan_dirty = true;
  return HLBM_OK;
}

int hlbm_info(hlbm_ctx* c, int64_t info[8]) {
  if (!c || !info) return fail(HLBM_EINVAL, "hlbm_info: NULL argument");
  info[0] = c->n[0];
  info[1] = c->n[1];
  info[2] = c->n[2];
  info[3] = c->precision;
  info[4] = c->steps;
  info[5] = c->launches;
  info[6] = int64_t(elem_size(c->precision));
  info[7] = c->device;
  return HLBM_OK;
}

int hlbm_set_wait_limit(hlbm_ctx* c, int64_t polls) {
  if (!c || polls < 0) return fail(HLBM_EINVAL, "hlbm_set_wait_limit: polls must be >= 0");
  c->wait_limit = polls == 0 ? TMA_WAIT_LIMIT : polls;
  return HLBM_OK;
}

int hlbm_tune(hlbm_ctx* c, int32_t variant) {
  if (!c || variant < 0 || variant >= NUM_VARIANTS)
    return fail(HLBM_EINVAL, "hlbm_tune: variant must be in [0, " + std::to_string(NUM_VARIANTS) + ")");
  c->variant = variant;
  c->variant_tuned = true;
  return HLBM_OK;
}

int hlbm_autotune(hlbm_ctx* c, int32_t reps, int32_t* chosen, double* ms_per_variant) {
  if (!c || reps < 1) return fail(HLBM_EINVAL, "hlbm_autotune: bad argument");
  if (int rc = set_device(c)) return rc;
  if (int rc = build_plan(c)) return rc;
  // time fused launches from the current buffer into the idle one: the state does not advance
  void* fin = c->f[c->cur];
  void* fout = c->f[1 - c->cur];
  if (c->phase == MATER) c->phase = POSTCOL;
  cudaEvent_t e0, e1;
  HLBM_CK(cudaEventCreate(&e0));
  HLBM_CK(cudaEventCreate(&e1));
  int best = c->variant;
  float best_ms = 1e30f;
  for (int v = 0; v < NUM_VARIANTS; v++) {
    if (ms_per_variant) ms_per_variant[v] = -1.0;
    if (v < 6 && (v % 2) == 1 && !vec_applies(c, v)) continue;
    if (v >= 8 && !rows_runs(c->plan, v, MODE_FUSED, int(elem_size(c->precision)))) continue;
    if (v >= 6 && c->tma_stages < 2) continue;
    cudaError_t e = launch_step_variant(c, MODE_FUSED, fin, fout, v);  // warm-up
    if (e == cudaSuccess) e = cudaEventRecord(e0, c->stream);
    for (int r = 0; r < reps && e == cudaSuccess; r++) e = launch_step_variant(c, MODE_FUSED, fin, fout, v);
    if (e == cudaSuccess) e = cudaEventRecord(e1, c->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e != cudaSuccess) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      return fail(HLBM_ECUDA, std::string("hlbm_autotune: ") + cudaGetErrorString(e));
    }
    ms /= reps;
    if (ms_per_variant) ms_per_variant[v] = ms;
    if (ms < best_ms) {
      best_ms = ms;
      best = v;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (int rc = check_device_error(c)) return rc;
  c->variant = best;
  c->variant_tuned = true;
  if (chosen) *chosen = best;
  return HLBM_OK;
}

void* hlbm_stream(hlbm_ctx* c) { return c ? static_cast<void*>(c->stream) : nullptr; }

}  // extern "C"

// ------------------------------------------------------------------------------------------
// Batches: many lattices, one pipelined persistent-kernel launch per time step.
struct hlbm_batch {
  int precision;
  int device;
  int sms = 148;
  cudaStream_t stream = nullptr;
  std::vector<hlbm_ctx*> members;
  bool dirty = true;
  LatticeDesc* desc_dev = nullptr;
  Tile* tiles_dev = nullptr;
  size_t desc_cap = 0, tiles_cap = 0;
  int ntiles = 0, tile_elems = 0, stages = 0, stages2 = 0, walls = 0;
  int variant = 8;  // 8, 9: tile-list kernel (>= 3 or 2 CTAs per SM); 6, 7: pipelined kernel
  bool descs_stale = true;
  int* err_dev = nullptr;
  cudaGraphExec_t graph = nullptr;  // two steps: parity 0 then parity 1
  int64_t replays = 0, launches = 0;
  // variant 10 (concurrent): a captured graph of two steps of every member, and what it was
  // captured for (members, their buffer parity and plan versions)
  cudaGraphExec_t cgraph = nullptr;
  cudaEvent_t fork_ev = nullptr;
  std::vector<hlbm_ctx*> cg_members;
  std::vector<int64_t> cg_state;
  int64_t cg_kernels = 0;
  std::vector<int64_t> cg_member_kernels;
};

namespace {

int batch_fail(int code, const std::string& m) { return fail(code, m); }

void batch_drop_graph(hlbm_batch* b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  b->graph = nullptr;
  if (b->cgraph) cudaGraphExecDestroy(b->cgraph);
  b->cgraph = nullptr;
  b->cg_members.clear();
  b->cg_state.clear();
}

// ------------------------------------------------------------------ concurrent batches (variant 10)
// Every member steps with its own single-lattice kernel (its plan in kernel parameters, the
// collision specialised, vectorised where eligible); the members' launches are forked onto their
// own streams so that small lattices run side by side, and two steps of all of them are replayed
// from one captured graph.  Graph-replayed launches of the 16-bit tiers read their step number
// (the stochastic-rounding salt) from a per-member device counter pair, so every member rounds
// exactly as it does stepped alone.
int concurrent_variant(const hlbm_ctx* c) { return (c->variant < 6 || c->variant >= 8) ? c->variant : 4; }

int64_t concurrent_state(const hlbm_ctx* c) { return (c->plan_version * 2 + c->cur) * 16 + concurrent_variant(c); }

int batch_capture_concurrent(hlbm_batch* b) {
  if (b->cgraph) cudaGraphExecDestroy(b->cgraph);
  b->cgraph = nullptr;
  const bool sr = b->precision == HLBM_F16 || b->precision == HLBM_BF16;
  if (!b->fork_ev) HLBM_CK(cudaEventCreateWithFlags(&b->fork_ev, cudaEventDisableTiming));
  for (hlbm_ctx* c : b->members) {
    if (!c->join_ev) HLBM_CK(cudaEventCreateWithFlags(&c->join_ev, cudaEventDisableTiming));
    if (sr && !c->seed_dev) {
      if (pool_alloc((void**)&c->seed_dev, 2 * sizeof(uint32_t), c->device, c->stream) != cudaSuccess)
        return fail(HLBM_ENOMEM, "hlbm_batch_step: step counters");
      HLBM_CK(cudaStreamSynchronize(c->stream));
    }
  }
  cudaGraph_t g = nullptr;
  std::vector<int64_t> launches_before;
  for (hlbm_ctx* c : b->members) launches_before.push_back(c->launches);
  HLBM_CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = cudaEventRecord(b->fork_ev, b->stream);
  for (hlbm_ctx* c : b->members) {
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream, b->fork_ev, 0);
    for (int k = 0; k < 2 && e == cudaSuccess; k++) {
      StepPlan pk = c->plan;
      pk.seed_dev = sr ? c->seed_dev : nullptr;
      pk.seed_parity = k;
      e = launch_with_plan(c, MODE_FUSED, c->f[c->cur ^ k], c->f[c->cur ^ k ^ 1], pk, concurrent_variant(c), c->stream);
    }
    if (e == cudaSuccess) e = cudaEventRecord(c->join_ev, c->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, c->join_ev, 0);
  }
  const cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
  b->cg_kernels = 0;  // kernels of one replay, per member and in all (the capture launched none)
  b->cg_member_kernels.clear();
  for (size_t m = 0; m < b->members.size(); m++) {
    const int64_t k = b->members[m]->launches - launches_before[m];
    b->members[m]->launches = launches_before[m];
    b->cg_member_kernels.push_back(k);
    b->cg_kernels += k;
  }
  if (e != cudaSuccess || e2 != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return fail(HLBM_ECUDA, "hlbm_batch_step: capture of the concurrent graph failed");
  }
  const cudaError_t e3 = cudaGraphInstantiate(&b->cgraph, g, 0);
  cudaGraphDestroy(g);
  if (e3 != cudaSuccess) return fail(HLBM_ECUDA, "hlbm_batch_step: graph instantiation failed");
  b->cg_members = b->members;
  b->cg_state.clear();
  for (hlbm_ctx* c : b->members) b->cg_state.push_back(concurrent_state(c));
  return HLBM_OK;
}

int batch_step_concurrent(hlbm_batch* b, int64_t nsteps) {
  const bool sr = b->precision == HLBM_F16 || b->precision == HLBM_BF16;
  bool fresh = false;
  for (hlbm_ctx* c : b->members) {
    if (int rc = build_plan(c)) return rc;
    if (c->phase == MATER) c->phase = POSTCOL;
    fresh |= c->phase == RAW;
    HLBM_CK(cudaStreamSynchronize(c->stream));
  }
  auto direct_step = [&]() -> int {  // one step of every member, launched on its own stream
    for (hlbm_ctx* c : b->members) {
      const int mode = c->phase == RAW ? MODE_PROLOGUE : MODE_FUSED;
      HLBM_CK(launch_step_variant(c, mode, c->f[c->cur], c->f[1 - c->cur], concurrent_variant(c)));
      c->cur = 1 - c->cur;
      c->phase = POSTCOL;
      c->steps++;
      b->launches++;
    }
    for (hlbm_ctx* c : b->members) HLBM_CK(cudaStreamSynchronize(c->stream));
    return HLBM_OK;
  };
  int64_t todo = nsteps;
  if (fresh) {
    if (int rc = direct_step()) return rc;
    todo--;
  }
  if (todo >= 2) {
    bool valid = b->cgraph && b->cg_members == b->members;
    for (size_t m = 0; valid && m < b->members.size(); m++)
      valid = b->cg_state[m] == concurrent_state(b->members[m]);
    if (!valid)
      if (int rc = batch_capture_concurrent(b)) return rc;
    if (sr) {  // the counters start at each member's own step count
      for (hlbm_ctx* c : b->members) {
        c->seed_host[0] = uint32_t(c->steps);
        c->seed_host[1] = uint32_t(c->steps + 1);
        HLBM_CK(cudaMemcpyAsync(c->seed_dev, c->seed_host, sizeof(c->seed_host), cudaMemcpyHostToDevice, c->stream));
      }
      for (hlbm_ctx* c : b->members) HLBM_CK(cudaStreamSynchronize(c->stream));
    }
    while (todo >= 2) {
      HLBM_CK(cudaGraphLaunch(b->cgraph, b->stream));
      b->replays++;
      b->launches += b->cg_kernels;
      for (size_t m = 0; m < b->members.size(); m++) {
        b->members[m]->steps += 2;
        b->members[m]->launches += b->cg_member_kernels[m];
      }
      todo -= 2;
    }
    HLBM_CK(cudaStreamSynchronize(b->stream));
  }
  if (todo == 1)
    if (int rc = direct_step()) return rc;
  for (hlbm_ctx* c : b->members)
    if (int rc = check_device_error(c)) return rc;
  return HLBM_OK;
}

// rebuild the concatenated tile list and the descriptors of the members
int batch_rebuild(hlbm_batch* b) {
  if (!b->dirty) return HLBM_OK;
  batch_drop_graph(b);
  const size_t es = elem_size(b->precision);
  int tile_elems = 0, walls = 0;
  std::vector<int> rows_of(b->members.size());
  for (size_t m = 0; m < b->members.size(); m++) {
    hlbm_ctx* c = b->members[m];
    if (int rc = build_plan(c)) return rc;
    int rows, s1, s2;
    if (b->variant >= 8) {  // tile-list kernel: about 256 nodes (one per thread) per tile, any nx
      rows = std::max(1, std::min(c->n[1], 256 / c->n[0]));
    } else if (!pipeline_geometry(c->n[0], c->n[1], es, rows, s1, s2)) {
      return batch_fail(HLBM_EPLAN, "pipelined batch: nx * bytes per population must be a multiple of 16");
    }
    rows_of[m] = rows;
    tile_elems = std::max(tile_elems, rows * c->n[0]);
    walls |= c->plan.walls;
  }
  std::vector<Tile> tiles;
  for (size_t m = 0; m < b->members.size(); m++) {
    hlbm_ctx* c = b->members[m];
    for (int z = 0; z < c->n[2]; z++)
      for (int y0 = 0; y0 < c->n[1]; y0 += rows_of[m])
        tiles.push_back(make_int4(int(m), z, y0, std::min(rows_of[m], c->n[1] - y0)));
  }
  const size_t stage_bytes = size_t(Q) * tile_elems * es;
  const size_t head = tma_head_bytes();
  int stages = stage_bytes ? int((226 * 1024 - head) / stage_bytes) : 0;
  int stages2 = stage_bytes ? int((112 * 1024 - head) / stage_bytes) : 0;
  stages = stages > 4 ? 4 : stages;
  stages2 = stages2 > 4 ? 4 : stages2;
  if (b->variant < 8 && !b->members.empty() && stages < 2)
    return batch_fail(HLBM_EPLAN, "batch tiles do not fit two pipeline stages");
  b->stages2 = stages2;
  if (b->members.size() > b->desc_cap) {
    pool_free(b->desc_dev, b->stream);
    b->desc_cap = std::max<size_t>(b->members.size(), 2 * b->desc_cap);
    if (pool_alloc((void**)&b->desc_dev, b->desc_cap * sizeof(LatticeDesc), b->device, b->stream) != cudaSuccess)
      return batch_fail(HLBM_ENOMEM, "batch descriptors");
  }
  if (tiles.size() > b->tiles_cap) {
    pool_free(b->tiles_dev, b->stream);
    b->tiles_cap = std::max<size_t>(tiles.size(), 2 * b->tiles_cap);
    if (pool_alloc((void**)&b->tiles_dev, b->tiles_cap * sizeof(Tile), b->device, b->stream) != cudaSuccess)
      return batch_fail(HLBM_ENOMEM, "batch tile list");
  }
  if (!tiles.empty())
    HLBM_CK(cudaMemcpyAsync(b->tiles_dev, tiles.data(), tiles.size() * sizeof(Tile), cudaMemcpyHostToDevice,
                            b->stream));
  HLBM_CK(cudaStreamSynchronize(b->stream));
  b->ntiles = int(tiles.size());
  b->tile_elems = tile_elems;
  b->stages = stages;
  b->walls = walls;
  b->dirty = false;
  b->descs_stale = true;
  return HLBM_OK;
}

// upload the members' descriptors: buffers, current index, first-step flag
int batch_refresh_descs(hlbm_batch* b) {
  if (!b->descs_stale) return HLBM_OK;
  std::vector<LatticeDesc> descs(b->members.size());
  for (size_t m = 0; m < b->members.size(); m++) {
    hlbm_ctx* c = b->members[m];
    descs[m].plan = c->plan_dev;
    descs[m].f[0] = c->f[0];
    descs[m].f[1] = c->f[1];
    descs[m].flags = c->flags;
    descs[m].cur = c->cur;
    descs[m].prologue = c->phase == RAW ? 1 : 0;
    descs[m].step[0] = uint32_t(c->steps);  // batched launches start at parity 0
    descs[m].step[1] = uint32_t(c->steps + 1);
  }
  if (!descs.empty())
    HLBM_CK(cudaMemcpyAsync(b->desc_dev, descs.data(), descs.size() * sizeof(LatticeDesc), cudaMemcpyHostToDevice,
                            b->stream));
  HLBM_CK(cudaStreamSynchronize(b->stream));
  b->descs_stale = false;
  return HLBM_OK;
}

cudaError_t batch_launch(hlbm_batch* b, int parity) {
  TmaArgs t;
  t.desc = b->desc_dev;
  t.tiles = b->tiles_dev;
  t.ntiles = b->ntiles;
  t.tile_elems = b->tile_elems;
  t.ctas_per_sm = (b->variant == 6 && b->stages2 >= 2) ? 2 : 1;
  t.stages = t.ctas_per_sm == 2 ? b->stages2 : b->stages;
  t.parity = parity;
  t.err = b->err_dev;
  t.grid = std::min(b->ntiles, b->sms * t.ctas_per_sm);
  t.seed = -1;
  t.ndesc = int(b->members.size());
  for (size_t m = 0; m < b->members.size(); m++) {  // members that pull this launch (not fresh)
    hlbm_ctx* c = b->members[m];
    if (c->phase == RAW) continue;
    if (cudaError_t e = outlet_passes(b->precision, c->plan, b->desc_dev, int(m), parity, c->n, b->stream,
                                      b->launches))
      return e;
  }
  StepPlan dummy;
  std::memset(&dummy, 0, sizeof(dummy));
  b->launches++;
  switch (b->precision) {
    case HLBM_F64: return step_f64(MODE_FUSED, b->walls, nullptr, nullptr, nullptr, dummy, b->stream, b->variant, t);
    case HLBM_F64_STRICT: return step_f64_strict(MODE_FUSED, b->walls, nullptr, nullptr, nullptr, dummy, b->stream, b->variant, t);
    case HLBM_F32: return step_f32(MODE_FUSED, b->walls, nullptr, nullptr, nullptr, dummy, b->stream, b->variant, t);
    case HLBM_F16: return step_f16(MODE_FUSED, b->walls, nullptr, nullptr, nullptr, dummy, b->stream, b->variant, t);
    default: return step_bf16(MODE_FUSED, b->walls, nullptr, nullptr, nullptr, dummy, b->stream, b->variant, t);
  }
}

}  // namespace

extern "C" {

int hlbm_batch_create(int32_t precision, int32_t device, hlbm_batch** out) {
  if (!out || precision < HLBM_F64 || precision > HLBM_BF16) return fail(HLBM_EINVAL, "hlbm_batch_create: bad argument");
  *out = nullptr;
  auto* b = new hlbm_batch();
  b->precision = precision;
  b->device = device;
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      pool_alloc((void**)&b->err_dev, sizeof(int), device, b->stream) != cudaSuccess ||
      cudaMemsetAsync(b->err_dev, 0, sizeof(int), b->stream) != cudaSuccess ||
      cudaStreamSynchronize(b->stream) != cudaSuccess) {
    cudaGetLastError();
    hlbm_batch_destroy(b);
    return fail(HLBM_ECUDA, "hlbm_batch_create: cannot set up the device");
  }
  cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, device);
  *out = b;
  return HLBM_OK;
}

int hlbm_batch_add(hlbm_batch* b, hlbm_ctx* c) {
  if (!b || !c) return fail(HLBM_EINVAL, "hlbm_batch_add: NULL argument");
  if (c->precision != b->precision || c->device != b->device)
    return fail(HLBM_EINVAL, "hlbm_batch_add: lattice precision or device differs from the batch");
  if (c->batch == b) return fail(HLBM_EINVAL, "hlbm_batch_add: lattice already in the batch");
  if (c->batch) return fail(HLBM_EINVAL, "hlbm_batch_add: lattice is a member of another batch");
  if (b->variant < 8 && (size_t(c->n[0]) * elem_size(c->precision)) % 16 != 0)
    return fail(HLBM_EPLAN, "hlbm_batch_add: the pipelined batch kernel needs nx * bytes per population % 16 == 0");
  b->members.push_back(c);
  c->batch = b;
  b->dirty = true;
  batch_drop_graph(b);  // an in-flight replay still completes
  return HLBM_OK;
}

int hlbm_batch_remove(hlbm_batch* b, hlbm_ctx* c) {
  if (!b || !c) return fail(HLBM_EINVAL, "hlbm_batch_remove: NULL argument");
  for (size_t m = 0; m < b->members.size(); m++)
    if (b->members[m] == c) {
      if (b->stream) cudaStreamSynchronize(b->stream);  // no batched launch still reads its memory
      b->members.erase(b->members.begin() + m);
      c->batch = nullptr;
      b->dirty = true;
      batch_drop_graph(b);
      return HLBM_OK;
    }
  return fail(HLBM_EINVAL, "hlbm_batch_remove: lattice not in the batch");
}

int hlbm_batch_step(hlbm_batch* b, int64_t nsteps) {
  if (!b || nsteps < 0) return fail(HLBM_EINVAL, "hlbm_batch_step: bad argument");
  if (nsteps == 0 || b->members.empty()) return HLBM_OK;
  HLBM_CK(cudaSetDevice(b->device));
  if (b->variant == 10) return batch_step_concurrent(b, nsteps);
  b->descs_stale = true;  // members may have been read out or rewritten since the last call
  bool fresh = false;
  for (hlbm_ctx* c : b->members) {
    if (int rc = build_plan(c)) return rc;
    if (c->phase == MATER) c->phase = POSTCOL;
    fresh |= c->phase == RAW;
    HLBM_CK(cudaStreamSynchronize(c->stream));  // member work is ordered before the batch stream's
  }
  if (int rc = batch_rebuild(b)) return rc;
  if (int rc = batch_refresh_descs(b)) return rc;
  int64_t todo = nsteps;
  int parity = 0;
  if (fresh) {  // fresh members take their first step (collide S_0) inside this launch
    HLBM_CK(batch_launch(b, 0));
    for (hlbm_ctx* c : b->members) {
      c->steps++;
      c->cur = 1 - c->cur;
      c->phase = POSTCOL;
    }
    b->descs_stale = true;
    if (int rc = batch_refresh_descs(b)) return rc;
    todo--;
  }
  if (!b->graph && todo >= 2) {
    cudaGraph_t g;
    HLBM_CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e0 = batch_launch(b, 0);
    cudaError_t e1 = batch_launch(b, 1);
    cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
    b->launches -= 2;
    if (e0 != cudaSuccess || e1 != cudaSuccess || e2 != cudaSuccess)
      return fail(HLBM_ECUDA, "hlbm_batch_step: graph capture failed");
    cudaError_t e3 = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e3 != cudaSuccess) return fail(HLBM_ECUDA, "hlbm_batch_step: graph instantiation failed");
  }
  while (todo >= 2) {
    HLBM_CK(cudaGraphLaunch(b->graph, b->stream));
    b->replays++;
    b->launches += 2;
    todo -= 2;
  }
  if (todo == 1) {
    HLBM_CK(batch_launch(b, 0));
    parity = 1;
  }
  // the graph replays leave cur unchanged; a trailing single launch flips it
  for (hlbm_ctx* c : b->members) {
    c->steps += nsteps - (fresh ? 1 : 0);
    if (parity) c->cur = 1 - c->cur;
  }
  if (parity) b->descs_stale = true;
  HLBM_CK(cudaStreamSynchronize(b->stream));
  int e = 0;
  HLBM_CK(cudaMemcpy(&e, b->err_dev, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) {
    cudaMemset(b->err_dev, 0, sizeof(int));
    return fail(HLBM_ECUDA, "hlbm_batch_step: a shared-memory pipeline wait timed out");
  }
  return HLBM_OK;
}

int hlbm_batch_tune(hlbm_batch* b, int32_t variant) {
  if (!b || variant < 6 || variant > 10)
    return fail(HLBM_EINVAL, "hlbm_batch_tune: variant must be 6, 7, 8, 9 or 10");
  if (variant < 8)
    for (hlbm_ctx* c : b->members)
      if ((size_t(c->n[0]) * elem_size(c->precision)) % 16 != 0)
        return fail(HLBM_EPLAN, "hlbm_batch_tune: a member's rows do not suit the pipelined kernel");
  b->variant = variant;
  b->dirty = true;
  return HLBM_OK;
}

// One timed replay per candidate: the batch's own launches (variants 6 - 9) or every member's own
// kernel forked onto its stream (variant 10), each reading the current state and writing the idle
// buffers, so no member's state advances (the zero-gradient outlet passes rewrite the same values).
int hlbm_batch_autotune(hlbm_batch* b, int32_t reps, int32_t* chosen, double* ms_per_variant) {
  if (!b || reps < 1) return fail(HLBM_EINVAL, "hlbm_batch_autotune: bad argument");
  for (int v = 0; v < HLBM_BATCH_VARIANTS; v++)
    if (ms_per_variant) ms_per_variant[v] = -1.0;
  if (b->members.empty()) {
    if (chosen) *chosen = b->variant;
    return HLBM_OK;
  }
  HLBM_CK(cudaSetDevice(b->device));
  for (hlbm_ctx* c : b->members) {
    if (int rc = build_plan(c)) return rc;
    if (c->phase == MATER) c->phase = POSTCOL;  // the state is the post-collision one either way
    HLBM_CK(cudaStreamSynchronize(c->stream));
  }
  cudaEvent_t e0, e1;
  HLBM_CK(cudaEventCreate(&e0));
  HLBM_CK(cudaEventCreate(&e1));
  auto timed = [&](auto&& launch) -> double {  // ms of one replay, after one untimed one
    if (launch() != cudaSuccess) return -1.0;
    if (cudaEventRecord(e0, b->stream) != cudaSuccess) return -1.0;
    for (int r = 0; r < reps; r++)
      if (launch() != cudaSuccess) return -1.0;
    float ms = 0.0f;
    if (cudaEventRecord(e1, b->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
        cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
      return -1.0;
    return double(ms) / reps;
  };
  const int saved = b->variant;
  int best = saved;
  double best_ms = 1e300;
  int rc = HLBM_OK;
  for (int v = 6; v <= 10 && rc == HLBM_OK; v++) {
    double ms = -1.0;
    if (v <= 9) {
      bool fits = true;
      if (v < 8)
        for (hlbm_ctx* c : b->members) fits = fits && (size_t(c->n[0]) * elem_size(c->precision)) % 16 == 0;
      if (!fits) continue;
      b->variant = v;
      b->dirty = true;
      if (batch_rebuild(b) != HLBM_OK) continue;  // tiles do not fit this kernel's stages
      b->descs_stale = true;
      if ((rc = batch_refresh_descs(b)) != HLBM_OK) break;
      ms = timed([&] { return batch_launch(b, 0); });
    } else {
      cudaGraph_t g = nullptr;
      cudaGraphExec_t exec = nullptr;
      if (!b->fork_ev && cudaEventCreateWithFlags(&b->fork_ev, cudaEventDisableTiming) != cudaSuccess) continue;
      cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) e = cudaEventRecord(b->fork_ev, b->stream);
      for (hlbm_ctx* c : b->members) {
        if (e == cudaSuccess && !c->join_ev) e = cudaEventCreateWithFlags(&c->join_ev, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream, b->fork_ev, 0);
        if (e == cudaSuccess)
          e = launch_with_plan(c, c->phase == RAW ? MODE_PROLOGUE : MODE_FUSED, c->f[c->cur], c->f[1 - c->cur],
                               c->plan, concurrent_variant(c), c->stream);
        if (e == cudaSuccess) e = cudaEventRecord(c->join_ev, c->stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, c->join_ev, 0);
      }
      const cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
      if (e == cudaSuccess && e2 == cudaSuccess && cudaGraphInstantiate(&exec, g, 0) == cudaSuccess)
        ms = timed([&] { return cudaGraphLaunch(exec, b->stream); });
      if (exec) cudaGraphExecDestroy(exec);
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
    }
    if (ms_per_variant) ms_per_variant[v - 6] = ms;
    if (ms > 0.0 && ms < best_ms) {
      best_ms = ms;
      best = v;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != HLBM_OK) {
    b->variant = saved;
    b->dirty = true;
    return rc;
  }
  int e = 0;
  HLBM_CK(cudaMemcpy(&e, b->err_dev, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) {
    cudaMemset(b->err_dev, 0, sizeof(int));
    b->variant = saved;
    b->dirty = true;
    return fail(HLBM_ECUDA, "hlbm_batch_autotune: a shared-memory pipeline wait timed out");
  }
  b->variant = best;
  b->dirty = true;  // tiles and graphs follow the chosen kernel at the next step
  b->descs_stale = true;
  if (chosen) *chosen = best;
  return HLBM_OK;
}

int hlbm_batch_info(hlbm_batch* b, int64_t info[6]) {
  if (!b || !info) return fail(HLBM_EINVAL, "hlbm_batch_info: NULL argument");
  if (int rc = batch_rebuild(b)) return rc;
  info[0] = int64_t(b->members.size());
  info[1] = b->ntiles;
  info[2] = b->tile_elems;
  info[3] = b->stages;
  info[4] = b->replays;
  info[5] = b->launches;
  return HLBM_OK;
}

void* hlbm_batch_stream(hlbm_batch* b) { return b ? (void*)b->stream : nullptr; }

int hlbm_trim_memory(int32_t device) {
  if (device < 0 || device >= 64) return fail(HLBM_EINVAL, "hlbm_trim_memory: bad device");
  cudaMemPool_t pool = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    pool = g_pools[device];
  }
  if (!pool) return HLBM_OK;
  HLBM_CK(cudaSetDevice(device));
  HLBM_CK(cudaDeviceSynchronize());
  HLBM_CK(cudaMemPoolTrimTo(pool, 0));
  return HLBM_OK;
}

int hlbm_batch_destroy(hlbm_batch* b) {
  if (!b) return HLBM_OK;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (hlbm_ctx* c : b->members) c->batch = nullptr;
  batch_drop_graph(b);
  if (b->fork_ev) cudaEventDestroy(b->fork_ev);
  if (b->stream) {
    pool_free(b->desc_dev, b->stream);
    pool_free(b->tiles_dev, b->stream);
    pool_free(b->err_dev, b->stream);
    cudaStreamDestroy(b->stream);
  }
  delete b;
  return HLBM_OK;
}

}  // extern "C"
