// run_cavite.cpp -- a C++ host program that runs hippoLBM's regression deck
// regression_lbm_cavite.msp through include/hippolbm.h alone and applies the deck's own
// check_macro_quantities pins (check_marco_quantities.cpp:71-114).
//
// The deck: a 31^3-node cubic cavity (cell_dims 30, bounds [0, 0.1]^3, no periodic axis),
// lbm_parameters {celerity 1, nuth 1e-4, avg_rho 1000} (the time step follows from the
// celerity), BGK, pre_stream_bcs [pre_bounce_back, cavity_z_l {U: [0, 0.1, 0]}],
// post_stream_bcs [post_bounce_back], 100 iterations; pins density 29791 +/- 0.1, min |u| >= 1e-6,
// max |u| <= 0.1.
//
//   run_cavite <precision 0..4> <populations output file or ->
// prints "sum_rho min_u max_u" and exits 0 when the pins hold, 1 when they fail, 2 on a library
// error (with hlbm_last_error()).
#include <hippolbm.h>

#include <cstdio>
#include <cstdlib>
#include <vector>

namespace {

void check(int rc, const char* what) {
  if (rc != HLBM_OK) {
    std::fprintf(stderr, "%s failed (%d): %s\n", what, rc, hlbm_last_error());
    std::exit(2);
  }
}

}  // namespace

int main(int argc, char** argv) {
  const int precision = argc > 1 ? std::atoi(argv[1]) : HLBM_F64_STRICT;
  const char* dump = argc > 2 ? argv[2] : "-";

  // initialize (config_initialize.msp order): domain, lbm_parameters, collision, obstacles
  const int32_t cell_dims[3] = {30, 30, 30};
  const double bmin[3] = {0.0, 0.0, 0.0}, bmax[3] = {0.1, 0.1, 0.1};
  const int32_t periodic[3] = {0, 0, 0};
  hlbm_ctx* ctx = nullptr;
  check(hlbm_domain(cell_dims, bmin, bmax, periodic, precision, 0, &ctx), "domain");
  const double Fext[3] = {0.0, 0.0, 0.0};
  check(hlbm_lbm_parameters(ctx, Fext, /*celerity*/ 1.0, /*nuth*/ 1e-4, /*avg_rho*/ 1000.0, /*has_tau*/ 0, 0.0, 0.0),
        "lbm_parameters");
  check(hlbm_collision(ctx, 0, nullptr), "bgk");
  check(hlbm_init_obstacles(ctx), "init_obstacles");
  check(hlbm_update_obstacles(ctx), "update_obstacles");

  // compute_loop hooks, recorded in deck order
  check(hlbm_pre_bounce_back(ctx), "pre_bounce_back");
  const double U[3] = {0.0, 0.1, 0.0};
  check(hlbm_cavity(ctx, 1, U), "cavity_z_l");
  check(hlbm_post_bounce_back(ctx, HLBM_HOOK_POST_STREAM), "post_bounce_back");

  check(hlbm_step(ctx, 100), "compute_loop x 100");
  double state[3];
  check(hlbm_simulation_state(ctx, state), "simulation_state");
  std::printf("%.17g %.17g %.17g\n", state[0], state[1], state[2]);

  if (dump[0] != '-') {  // populations of the real nodes, FP64, the header's layout
    int64_t info[8];
    check(hlbm_info(ctx, info), "info");
    const size_t n = size_t(19) * size_t(info[0]) * size_t(info[1]) * size_t(info[2]);
    std::vector<double> f(n);
    check(hlbm_get_populations(ctx, f.data()), "get_populations");
    FILE* fh = std::fopen(dump, "wb");
    if (!fh || std::fwrite(f.data(), sizeof(double), n, fh) != n) {
      std::fprintf(stderr, "cannot write %s\n", dump);
      return 2;
    }
    std::fclose(fh);
  }
  check(hlbm_destroy(ctx), "destroy");

  // check_macro_quantities {density: 29791, tol: 0.1, vmin: 1e-6, vmax: 0.1}
  bool ok = true;
  if (state[1] < 1e-6) {
    std::printf("min vel (simulation): %f is below (user-defined check): %f\n", state[1], 1e-6);
    ok = false;
  }
  if (state[2] > 0.1) {
    std::printf("max vel (simulation): %f is upper (user-defined check): %f\n", state[2], 0.1);
    ok = false;
  }
  if (state[0] - 29791.0 > 0.1 || 29791.0 - state[0] > 0.1) {
    std::printf("Sum of densities (simulation): %f is not closed to (user-defined check): %f +/- %f\n", state[0],
                29791.0, 0.1);
    ok = false;
  }
  std::printf("%s\n", ok ? "Test Pass." : "Test Failed.");
  return ok ? 0 : 1;
}
