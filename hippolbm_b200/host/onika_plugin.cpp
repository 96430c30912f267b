// onika_plugin.cpp -- hippoLBM's step-path operators as an Onika plugin over the C-ABI.
//
// Each class answers to the reference operator of the same name (the `register_factory` sites:
// domain_lbm.cpp, lbm_parameters.cpp, bgk.cu:100-102, mrt.cu, set_distribution.cu,
// update_obstacles.cu, register_solid_ball.cpp, register_solid_wall.cpp, register_quadrics.cpp,
// pre_bounce_back.cu, cavity.cu:98-99, wall_bounce_back.cu, post_bounce_back.cu, neuman.cu:127,
// lid_driven_cavity.cu, macro_variables.cu, streaming.cu:123, simulation_state.cu) and takes the
// deck slots of that operator, so a deck runs unchanged with this plugin in place of the
// reference's hippoLBM plugins.  The operators share one slot, `hlbm`: the library context.
//
// The C-ABI runs whole compute_loop iterations as fused kernels, so the loop's operators map as
// follows.  The collision and the hook operators (pre/post bounce-back, cavity, neumann, ...)
// record themselves into the context's step plan the first time they execute and are no-ops
// afterwards.  `streaming` marks one iteration pending; the pending iterations are launched by
// the next operator that needs the state -- the next iteration's `macro_variables`, or a read-out
// such as `simulation_state` -- by which time every hook of the deck has been recorded once.
// Operators that follow streaming in the first iteration (post_stream_bcs, then
// boundary_conditions) are recorded in that order as post-stream hooks, which applies them in the
// reference's order.
//
// Build (Onika's include paths and link flags added by the project's CMake):
//   g++ -std=c++17 -fPIC -shared onika_plugin.cpp -I<repo>/include -L<repo>/hippolbm_b200 -lhippolbm
#include <hippolbm.h>

#include <array>
#include <string>
#include <vector>

#include <onika/log.h>
#include <onika/math/basic_types.h>
#include <onika/scg/operator.h>
#include <onika/scg/operator_factory.h>
#include <onika/scg/operator_slot.h>

namespace hlbm_onika {

using onika::math::AABB;
using onika::math::IJK;
using onika::math::Vec3d;
using namespace onika::scg;
using State3 = std::array<double, 3>;

// the library context, shared by every operator of the graph
struct HlbmHandle {
  hlbm_ctx* ctx = nullptr;
  bool in_loop = false;    // the compute loop has started (its first macro_variables ran)
  bool recording = true;   // hook operators still record themselves (first iteration)
  int64_t pending = 0;     // iterations requested by streaming, not yet launched
  static void check(int rc) {
    if (rc != HLBM_OK) onika::fatal_error() << "hippolbm: " << hlbm_last_error() << std::endl;
  }
  void flush() {
    if (pending > 0) {
      check(hlbm_step(ctx, pending));
      pending = 0;
      recording = false;
    }
  }
  int32_t post_hook() const { return HLBM_HOOK_POST_STREAM; }
};

inline void vec3(const Vec3d& v, double out[3]) {
  out[0] = v.x;
  out[1] = v.y;
  out[2] = v.z;
}

// plan_yz_0 ... plan_xy_l (grid_region.hpp:360-373) -> HLBM_PLAN_*
inline std::vector<int32_t> plane_regions(const std::vector<std::string>& names) {
  static const char* known[6] = {"plan_yz_0", "plan_yz_l", "plan_xz_0", "plan_xz_l", "plan_xy_0", "plan_xy_l"};
  std::vector<int32_t> out;
  for (const std::string& n : names) {
    int found = -1;
    for (int k = 0; k < 6; k++)
      if (n == known[k]) found = k;
    if (found < 0) onika::fatal_error() << "hippolbm: unknown region " << n << std::endl;
    out.push_back(found);
  }
  return out;
}

// ------------------------------------------------------------------ initialize
class Domain : public OperatorNode {  // "domain" (domain_lbm.cpp:66-110)
 public:
  ADD_SLOT(IJK, cell_dims, INPUT, REQUIRED, DocString{"cells per axis; nodes = cells + 1"});
  ADD_SLOT(AABB, bounds, INPUT, REQUIRED, DocString{"physical extent"});
  ADD_SLOT(std::vector<bool>, periodic, INPUT, REQUIRED, DocString{"periodic axes x, y, z"});
  ADD_SLOT(int, precision, INPUT, int(HLBM_F64), DocString{"HLBM_F64, HLBM_F64_STRICT, HLBM_F32, HLBM_F16, HLBM_BF16"});
  ADD_SLOT(int, device, INPUT, 0, DocString{"CUDA device"});
  ADD_SLOT(HlbmHandle, hlbm, INPUT_OUTPUT, REQUIRED);
  void execute() final {
    const int32_t dims[3] = {int32_t(cell_dims->i), int32_t(cell_dims->j), int32_t(cell_dims->k)};
    double lo[3], hi[3];
    vec3(bounds->bmin, lo);
    vec3(bounds->bmax, hi);
    int32_t per[3] = {0, 0, 0};
    for (int d = 0; d < 3 && d < int(periodic->size()); d++) per[d] = (*periodic)[d] ? 1 : 0;
    HlbmHandle::check(hlbm_domain(dims, lo, hi, per, *precision, *device, &hlbm->ctx));
  }
};

class LbmParameters : public OperatorNode {  // "lbm_parameters" (lbm_parameters.cpp:73-99)
 public:
  ADD_SLOT(Vec3d, Fext, INPUT, Vec3d{}, DocString{"external force, physical units"});
  ADD_SLOT(double, celerity, INPUT, 1.0);
  ADD_SLOT(double, nuth, INPUT, REQUIRED);
  ADD_SLOT(double, avg_rho, INPUT, 1.0);
  ADD_SLOT(double, tau, INPUT, OPTIONAL);
  ADD_SLOT(double, dt, INPUT, 0.0);
  ADD_SLOT(HlbmHandle, hlbm, INPUT_OUTPUT, REQUIRED);
  void execute() final {
    double F[3];
    vec3(*Fext, F);
    const bool has_tau = tau.has_value();
    HlbmHandle::check(
        hlbm_lbm_parameters(hlbm->ctx, F, *celerity, *nuth, *avg_rho, has_tau ? 1 : 0, has_tau ? *tau : 0.0, *dt));
  }
};

class SetDistribution : public OperatorNode {  // "set_distribution" (set_distribution.cu:69-109)
 public:
  ADD_SLOT(double, value, INPUT, 1.0);
  ADD_SLOT(AABB, bounds, INPUT, OPTIONAL);
  ADD_SLOT(bool, do_update, INPUT, false);
  ADD_SLOT(HlbmHandle, hlbm, INPUT_OUTPUT, REQUIRED);
  void execute() final {
    double b6[6];
    const bool boxed = bounds.has_value();
    if (boxed) {
      vec3(bounds->bmin, b6);
      vec3(bounds->bmax, b6 + 3);
    }
    if (!hlbm->in_loop) {  // initialize: applied now
      HlbmHandle::check(hlbm_set_distribution(hlbm->ctx, *value, boxed ? b6 : nullptr, *do_update ? 1 : 0));
    } else if (hlbm->recording) {  // start_iteration hook
      if (!boxed) onika::fatal_error() << "hippolbm: start_iteration set_distribution needs bounds" << std::endl;
      HlbmHandle::check(hlbm_start_set_distribution(hlbm->ctx, *value, b6));
    }
  }
};

class InitObstacles : public OperatorNode {  // "init_obstacles"
 public:
  ADD_SLOT(HlbmHandle, hlbm, INPUT_OUTPUT, REQUIRED);
  void execute() final { HlbmHandle::check(hlbm_init_obstacles(hlbm->ctx)); }
};

class RegisterSolidBall : public OperatorNode {  // "register_solid_ball"
 public:
  ADD_SLOT(int, id, INPUT, REQUIRED);
  ADD_SLOT(Vec3d, center, INPUT, REQUIRED);
  ADD_SLOT(double, radius, INPUT, REQUIRED);
  ADD_SLOT(HlbmHandle, hlbm, INPUT_OUTPUT, REQUIRED);
  void execute() final {
    double c[3];
    vec3(*center, c);
    HlbmHandle::check(hlbm_register_solid_ball(hlbm->ctx, *id, c, *radius));
  }
};

class RegisterSolidWall : public OperatorNode {  // "register_solid_wall"
 public:
  ADD_SLOT(int, id, INPUT, REQUIRED);
  ADD_SLOT(AABB, bounds, INPUT, REQUIRED);
  ADD_SLOT(HlbmHandle, hlbm, INPUT_OUTPUT, REQUIRED);
  void execute() final {
    double lo[3], hi[3];
    vec3(bounds->bmin, lo);
    vec3(bounds->bmax, hi);
    HlbmHandle::check(hlbm_register_solid_wall(hlbm->ctx, *id, lo, hi));
  }
};

class RegisterQuadrics : public OperatorNode {  // "register_quadrics": the transformed 4x4 matrix
 public:
  ADD_SLOT(int, id, INPUT, REQUIRED);
  ADD_SLOT(std::vector<double>, quadrics, INPUT, REQUIRED, DocString{"16 values, row-major"});
  ADD_SLOT(HlbmHandle, hlbm, INPUT_OUTPUT, REQUIRED);
  void execute() final {
    if (quadrics->size() != 16) onika::fatal_error() << "hippolbm: a quadric has 16 coefficients" << std::endl;
    HlbmHandle::check(hlbm_register_quadric(hlbm->ctx, *id, quadrics->data()));
  }
};

class UpdateObstacles : public OperatorNode {  // "update_obstacles" (update_obstacles.cu:106-119)
 public:
  ADD_SLOT(HlbmHandle, hlbm, INPUT_OUTPUT, REQUIRED);
  void execute() final { HlbmHandle::check(hlbm_update_obstacles(hlbm->ctx)); }
};

// ------------------------------------------------------------------ compute loop
class MacroVariables : public OperatorNode {  // "macro_variables": launches pending iterations
 public:
  ADD_SLOT(HlbmHandle, hlbm, INPUT_OUTPUT, REQUIRED);
  void execute() final {
    hlbm->in_loop = true;
    hlbm->flush();
  }
};

template <int KIND>
class Collision : public OperatorNode {  // "bgk" (bgk.cu:77-94) / "mrt" (mrt.cu:71-89)
 public:
  ADD_SLOT(std::vector<double>, rates, INPUT, OPTIONAL,
           DocString{"MRT s_e, s_eps, s_q, s_pi, s_m, w_eps, w_epsj, w_xx (default: the reference's)"});
  ADD_SLOT(HlbmHandle, hlbm, INPUT_OUTPUT, REQUIRED);
  void execute() final {
    if (!hlbm->recording) return;
    const double* r = (KIND == 1 && rates.has_value() && rates->size() == 8) ? rates->data() : nullptr;
    HlbmHandle::check(hlbm_collision(hlbm->ctx, KIND, r));
  }
};

class PreBounceBack : public OperatorNode {  // "pre_bounce_back"
 public:
  ADD_SLOT(HlbmHandle, hlbm, INPUT_OUTPUT, REQUIRED);
  void execute() final {
    if (hlbm->recording) HlbmHandle::check(hlbm_pre_bounce_back(hlbm->ctx));
  }
};

template <int SIDE>
class Cavity : public OperatorNode {  // "cavity_z_0" / "cavity_z_l" (cavity.cu:66-88)
 public:
  ADD_SLOT(Vec3d, U, INPUT, REQUIRED, DocString{"wall velocity, lattice units"});
  ADD_SLOT(HlbmHandle, hlbm, INPUT_OUTPUT, REQUIRED);
  void execute() final {
    if (!hlbm->recording) return;
    double u[3];
    vec3(*U, u);
    HlbmHandle::check(hlbm_cavity(hlbm->ctx, SIDE, u));
  }
};

class WallBounceBack : public OperatorNode {  // "wall_bounce_back"
 public:
  ADD_SLOT(HlbmHandle, hlbm, INPUT_OUTPUT, REQUIRED);
  void execute() final {
    if (hlbm->recording) HlbmHandle::check(hlbm_wall_bounce_back(hlbm->ctx));
  }
};

class Streaming : public OperatorNode {  // "streaming" (streaming.cu:68-118)
 public:
  ADD_SLOT(HlbmHandle, hlbm, INPUT_OUTPUT, REQUIRED);
  void execute() final { hlbm->pending++; }
};

class PostBounceBack : public OperatorNode {  // "post_bounce_back"
 public:
  ADD_SLOT(HlbmHandle, hlbm, INPUT_OUTPUT, REQUIRED);
  void execute() final {
    if (hlbm->recording) HlbmHandle::check(hlbm_post_bounce_back(hlbm->ctx, hlbm->post_hook()));
  }
};

template <int LID>
class PlaneVelocity : public OperatorNode {  // "neumann" (neuman.cu:69-122) / "lid_driven_cavity"
 public:
  ADD_SLOT(Vec3d, U, INPUT, REQUIRED, DocString{"velocity, physical units"});
  ADD_SLOT(std::vector<std::string>, regions, INPUT, REQUIRED);
  ADD_SLOT(HlbmHandle, hlbm, INPUT_OUTPUT, REQUIRED);
  void execute() final {
    if (!hlbm->recording) return;
    double u[3];
    vec3(*U, u);
    const std::vector<int32_t> r = plane_regions(*regions);
    if (LID)
      HlbmHandle::check(hlbm_lid_driven_cavity(hlbm->ctx, hlbm->post_hook(), u, r.data(), int32_t(r.size())));
    else
      HlbmHandle::check(hlbm_neumann(hlbm->ctx, hlbm->post_hook(), u, r.data(), int32_t(r.size())));
  }
};

class SimulationState : public OperatorNode {  // "simulation_state" (simulation_state.cu:73-98)
 public:
  ADD_SLOT(HlbmHandle, hlbm, INPUT_OUTPUT, REQUIRED);
  ADD_SLOT(State3, state, OUTPUT, OPTIONAL,
           DocString{"sum rho, min |u|, max |u|"});
  void execute() final {
    hlbm->flush();
    HlbmHandle::check(hlbm_simulation_state(hlbm->ctx, state->data()));
  }
};

}  // namespace hlbm_onika

ONIKA_AUTORUN_INIT(hippolbm_b200) {
  using onika::scg::make_simple_operator;
  using onika::scg::OperatorNodeFactory;
  using namespace hlbm_onika;
  OperatorNodeFactory* f = OperatorNodeFactory::instance();
  f->register_factory("domain", make_simple_operator<Domain>);
  f->register_factory("lbm_parameters", make_simple_operator<LbmParameters>);
  f->register_factory("set_distribution", make_simple_operator<SetDistribution>);
  f->register_factory("init_obstacles", make_simple_operator<InitObstacles>);
  f->register_factory("register_solid_ball", make_simple_operator<RegisterSolidBall>);
  f->register_factory("register_solid_wall", make_simple_operator<RegisterSolidWall>);
  f->register_factory("register_quadrics", make_simple_operator<RegisterQuadrics>);
  f->register_factory("update_obstacles", make_simple_operator<UpdateObstacles>);
  f->register_factory("macro_variables", make_simple_operator<MacroVariables>);
  f->register_factory("bgk", make_simple_operator<Collision<0>>);
  f->register_factory("mrt", make_simple_operator<Collision<1>>);
  f->register_factory("pre_bounce_back", make_simple_operator<PreBounceBack>);
  f->register_factory("cavity_z_0", make_simple_operator<Cavity<0>>);
  f->register_factory("cavity_z_l", make_simple_operator<Cavity<1>>);
  f->register_factory("wall_bounce_back", make_simple_operator<WallBounceBack>);
  f->register_factory("streaming", make_simple_operator<Streaming>);
  f->register_factory("post_bounce_back", make_simple_operator<PostBounceBack>);
  f->register_factory("neumann", make_simple_operator<PlaneVelocity<0>>);
  f->register_factory("lid_driven_cavity", make_simple_operator<PlaneVelocity<1>>);
  f->register_factory("simulation_state", make_simple_operator<SimulationState>);
}
