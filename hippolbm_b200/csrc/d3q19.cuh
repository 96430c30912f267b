// d3q19.cuh -- D3Q19 lattice constants and the node-local operator algebra shared by the
// step kernels.  Direction order, weights and opposites follow LBMScheme<19>
// (scheme.hpp:47-69): direction 0 is rest; for odd i, i and i+1 are opposites.
#pragma once
#include <cstdint>

namespace hlbm {

constexpr int Q = 19;
constexpr int8_t FLAG_FLUID = -1;  // FLUIDE_ (enum.hpp:59)
constexpr int8_t FLAG_WALL = -2;   // WALL_   (enum.hpp:60)

struct D3Q19 {
  static constexpr int ex[Q] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
  static constexpr int ey[Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
  static constexpr int ez[Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
  static constexpr int wden[Q] = {3, 18, 18, 18, 18, 18, 18, 36, 36, 36, 36, 36, 36, 36, 36, 36, 36, 36, 36};
  static constexpr int opp(int i) { return i == 0 ? 0 : ((i & 1) ? i + 1 : i - 1); }
};

// Plane bounce-back tables (bounce_back.hpp:65-140): the populations saved before
// streaming (pre) and where they are written back after streaming (post), per face
// x_0, x_l, y_0, y_l, z_0, z_l (bounce_back_manager.hpp:50-56 numbering).
struct PlaneBB {
  static constexpr int pre[6][5] = {{2, 10, 8, 12, 14}, {1, 9, 7, 11, 13}, {4, 8, 9, 16, 18},
                                    {3, 7, 10, 15, 17}, {6, 13, 12, 17, 16}, {5, 14, 11, 18, 15}};
  static constexpr int post[6][5] = {{1, 9, 7, 11, 13}, {2, 10, 8, 12, 14}, {3, 7, 10, 15, 17},
                                     {4, 8, 9, 16, 18}, {5, 14, 11, 18, 15}, {6, 13, 12, 17, 16}};
};

// Step plan: the node-local form of the operator lists of one deck.
enum OpKind : int32_t { OP_POST_BB = 0, OP_ZOUHE = 1, OP_LID = 2, OP_SETDIST = 3, OP_ZERO_GRADIENT = 4 };
constexpr int MAX_PLANE_OPS = 16;
constexpr int MAX_CAVITY = 4;
constexpr int MAX_SETS = 8;

struct PlaneOp {
  int32_t kind;  // OP_POST_BB (all non-periodic faces), OP_ZOUHE / OP_LID (one face)
  int32_t face;  // 0..5
  double u[3];   // lattice units
};

struct SetBox {  // set_distribution over a clipped box, applied at start_iteration
  int32_t lo[3], hi[3];
  double value;
};

struct StepPlan {
  int32_t nx, ny, nz;
  int32_t periodic[3];
  int64_t ncell;
  int64_t stride;  // elements between direction planes (>= ncell, padded)
  int32_t collision;  // 0 BGK, 1 MRT
  int32_t walls;      // wall_bounce_back active
  int32_t has_force;
  int32_t nops;
  int32_t nsets;
  int32_t ncav[6];    // cavity coefficient sets per face (z faces only)
  double tau, inv_tau;
  double F[3];
  double fw3[Q];      // 3 w_i (e_i . F): the force term of a collision is fw3_i * rho
  float ffw3[Q];      // the same in FP32
  double mrt[8];      // s_e, s_eps, s_q, s_pi, s_m, w_eps, w_epsj, w_xx
  double cav[6][MAX_CAVITY][5];
  double rho0;        // reference density of the deviation storage
  double scale, inv_scale;  // deviation storage scale
  float dref[Q];      // 16-bit storage keeps (f_i - dref_i) * scale; dref_i = feq_i(rho0, u0)
  uint32_t seed;      // step number of the launch: salt of the stochastic rounding
  int32_t rounding;   // 16-bit storage: 0 round to nearest, 1 stochastic rounding
  // when set, the step number comes from seed_dev[seed_parity] instead of `seed`, and the launch
  // writes seed_dev[seed_parity ^ 1] = that + 1 (launches replayed from a captured graph)
  uint32_t* seed_dev;
  int32_t seed_parity;
  // geometry of the one-node-per-thread kernel: 0 = x on threadIdx.x, y on threadIdx.y (rows of
  // whole warps); 1 = blocks of 256 consecutive nodes of a z-plane, for rows that would leave
  // lanes idle (x = i mod nx, y = i / nx through inv_nx and one correction; planes < 2^24 nodes)
  int32_t linear;
  float inv_nx;
  int32_t face_mask;  // face_pass_mask of the plan: faces whose nodes the boundary operators change
  // per node: 1 when some direction pulls from a wall node (k_near_wall); nodes with 0 skip the
  // wall test of every pull.  Null: test every pull.
  const int8_t* nearwall;
  // the flags may hold wall nodes (an obstacle was rasterised or wall flags were put)
  int32_t wall_flags;
  PlaneOp ops[MAX_PLANE_OPS];
  SetBox sets[MAX_SETS];
};

// Whether the kernels that update node pairs in packed FP32 (the vectorised kernel of the 4- and
// 2-byte tiers, the 16-bit pair kernel) take a plan: no start_iteration boxes, no body force (the
// force term would hold the pair's density in registers through the whole update), and wall nodes
// only where wall_bounce_back makes their populations scratch (a pair collides both lanes).  Other
// plans run the one-node kernel.
inline bool pair_kernels_apply(const StepPlan& p, int bytes) {
  return bytes == 8 || (p.nsets == 0 && !p.has_force && (!p.wall_flags || p.walls));
}

// Nodes per thread of the vectorised step kernel for a storage type of `bytes` bytes: one 16-byte
// vector per direction plane (double2; float4 and 8 packed 16-bit values at the lowest occupancy
// target, 1 CTA of 256 threads per SM, up to 255 registers), or one 8-byte vector for the 4- and
// 2-byte types at the higher targets (128 / 80 registers); and whether a lattice can use it:
// whole vectors per row, at least one warp of them, node offsets that fit 32 bits, and the
// conditions of pair_kernels_apply.
inline constexpr int vec_npt_bytes(int bytes, int minb) {
  return bytes == 8 ? 2 : (minb <= 1 ? 16 : 8) / bytes;
}
inline constexpr int variant_minb(int variant) { return variant / 2 + 1; }
inline bool vec_eligible_bytes(const StepPlan& p, int walls, int bytes, int variant) {
  (void)walls;  // wall obstacles: the wall fix-up pass follows the vectorised kernel
  const int npt = vec_npt_bytes(bytes, variant_minb(variant));
  return p.nx % npt == 0 && p.nx / npt >= 32 && p.ncell <= int64_t(0xffffffffu) && pair_kernels_apply(p, bytes);
}

// Whether the 16-bit one-node kernel can run two nodes per thread: even z-planes (every pair on a
// 4-byte boundary) of fewer than 2^24 nodes, and pair_kernels_apply.
inline bool pairs_eligible(const StepPlan& p) {
  const int64_t plane = int64_t(p.nx) * p.ny;
  return plane % 2 == 0 && plane < (int64_t(1) << 24) && pair_kernels_apply(p, 2);
}

// Whether a single-lattice launch of step variant `variant` (not the prologue) is followed by the
// face pass: the vectorised kernel always, the one-node kernel for the 4- and 2-byte tiers; the
// pipelined kernel (variants 6, 7) applies the operators inline.
inline bool face_pass_runs(const StepPlan& p, int walls, int variant, bool prologue, int bytes) {
  if (variant >= 6 || prologue || p.face_mask == 0) return false;
  return (variant % 2 == 1 && vec_eligible_bytes(p, walls, bytes, variant)) || bytes < 8;
}

// Faces whose nodes the boundary operators of the plan can change: every non-periodic face for
// post_bounce_back, the operator's own face for neumann / lid_driven_cavity.  Bit F = face F
// (x0, xl, y0, yl, z0, zl).
inline int face_pass_mask(const StepPlan& p) {
  int m = 0;
  for (int o = 0; o < p.nops; o++) {
    const PlaneOp& op = p.ops[o];
    if (op.kind == OP_POST_BB) {
      for (int f = 0; f < 6; f++)
        if (!p.periodic[f / 2]) m |= 1 << f;
    } else if (op.kind == OP_ZOUHE || op.kind == OP_LID) {
      m |= 1 << op.face;
    }
  }
  return m;
}

}  // namespace hlbm
