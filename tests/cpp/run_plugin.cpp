// run_plugin.cpp -- drives hippolbm_b200/host/onika_plugin.cpp the way an Onika graph runs
// regression_lbm_cavite.msp: the operators are made by name through the factory the plugin
// registers into, configured with the deck's slots, executed in the order of the deck's
// initialize list and compute loop (config_initialize.msp:14-32, config_compute_loop.msp:23-38),
// and the deck's check_macro_quantities pins are applied to simulation_state.
//   run_plugin <precision 0..4>   -> prints "sum_rho min_u max_u", exit 0 when the pins hold
#include <array>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <string>
#include <vector>

#include <onika/math/basic_types.h>
#include <onika/scg/operator.h>

using onika::math::AABB;
using onika::math::IJK;
using onika::math::Vec3d;
using onika::scg::OperatorNode;
using onika::scg::OperatorNodeFactory;

static std::shared_ptr<OperatorNode> op(const char* name) { return OperatorNodeFactory::instance()->make_operator(name); }

int main(int argc, char** argv) {
  const int precision = argc > 1 ? std::atoi(argv[1]) : 1;
  try {
    auto domain = op("domain");
    domain->configure("cell_dims", IJK{30, 30, 30});
    domain->configure("bounds", AABB{Vec3d{0, 0, 0}, Vec3d{0.1, 0.1, 0.1}});
    domain->configure("periodic", std::vector<bool>{false, false, false});
    domain->configure("precision", precision);
    auto params = op("lbm_parameters");
    params->configure("celerity", 1.0);
    params->configure("nuth", 1e-4);
    params->configure("avg_rho", 1000.0);
    auto init_obstacles = op("init_obstacles");
    auto update_obstacles = op("update_obstacles");
    for (auto& o : {domain, params, init_obstacles, update_obstacles}) o->execute();

    auto macro = op("macro_variables");
    auto collision = op("bgk");
    auto pre = op("pre_bounce_back");
    auto cavity = op("cavity_z_l");
    cavity->configure("U", Vec3d{0.0, 0.1, 0.0});
    auto streaming = op("streaming");
    auto post = op("post_bounce_back");
    for (int it = 0; it < 100; it++)
      for (auto& o : {macro, collision, pre, cavity, streaming, post}) o->execute();

    auto state = op("simulation_state");
    state->execute();
    const auto s = std::any_cast<std::array<double, 3>>(onika::scg::shared_slots().at("state"));
    std::printf("%.17g %.17g %.17g\n", s[0], s[1], s[2]);
    const bool ok = s[1] >= 1e-6 && s[2] <= 0.1 && s[0] - 29791.0 <= 0.1 && 29791.0 - s[0] <= 0.1;
    std::printf("%s\n", ok ? "Test Pass." : "Test Failed.");
    return ok ? 0 : 1;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 2;
  }
}
