// ref_harness.cpp -- drives the reference's OWN kernel functors on the CPU.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile into oracle/_ref/libhlbm_ref.so
// from the reference headers where they lie (read-only include paths); no reference
// source is copied into this repository.  It exports the same orc_* symbols as the
// C restatement (hlbm_oracle.c), so tests can run both through identical calls and
// pin the restatement bit for bit.  Each entry restates only the operator's
// execute() sequencing (the Onika graph and MPI are not available here); the
// per-cell arithmetic is the reference functors'.  Single rank: every periodic
// neighbour is the rank itself, as in make_domain.hpp:213-255.
#include <onika/math/basic_types.h>
#include <onika/math/matrix4d.h>

#include <cstdio>
#include <cstdlib>
#include <memory>
#include <variant>

// core + grid
#include <hippoLBM/core/box3d.hpp>
#include <hippoLBM/core/enum.hpp>
#include <hippoLBM/core/point3d.hpp>
#include <hippoLBM/grid/field_view.hpp>
#include <hippoLBM/grid/grid.hpp>
#include <hippoLBM/grid/scheme.hpp>
#include <hippoLBM/grid/stencil.hpp>
#include <hippoLBM/grid/fields.hpp>
#include <hippoLBM/grid/grid_region.hpp>
#include <hippoLBM/grid/grid_helper.hpp>
#include <hippoLBM/grid/lbm_parameters.hpp>
#include <hippoLBM/grid/operator_ghost_manager.hpp>
#include <hippoLBM/grid/packers.hpp>
#include <hippoLBM/grid/set_distribution.hpp>
// collision + streaming
#include <hippoLBM/collision/bgk.hpp>
#include <hippoLBM/collision/macro_variables.hpp>
#include <hippoLBM/collision/mrt.hpp>
#include <hippoLBM/collision/streaming.hpp>
#include <hippoLBM/grid/init_obst.hpp>
// boundary conditions
#include <hippoLBM/bcs/bounce_back.hpp>
#include <hippoLBM/bcs/bounce_back_manager.hpp>
#include <hippoLBM/bcs/cavity.hpp>
#include <hippoLBM/bcs/lid_driven_cavity.hpp>
#include <hippoLBM/bcs/neumann.hpp>
#include <hippoLBM/prepro/double_couette.hpp>
// obstacles + io
#include <hippoLBM/io/simulation_state.hpp>
#include <hippoLBM/obstacle/obstacle.hpp>

using namespace hippoLBM;
using onika::math::Vec3d;
constexpr int Q = 19;

namespace {
struct RefLattice {
  LBMGrid G;
  LBMGridRegion R;
  LBMFields<Q> F;
  bounce_back_manager<Q> bb;
  LBMParameters P;
  int n[3];
  std::vector<bool> periodic;
  std::vector<std::unique_ptr<std::variant<Ball, Wall, Quadric>>> obstacles;
};

RefLattice* L(void* h) { return static_cast<RefLattice*>(h); }

// set_distribution (set_distribution.cu:73-108)
void set_distribution_impl(RefLattice* g, double value, const double* bounds6, int do_update);
// update_ghost on one rank (update_ghost.hpp:57-70 with ghost_manager.hpp:101-137)
void update_ghost_impl(RefLattice* g) {
  constexpr Area Lc = Area::Local;
  Box3D mesh_box = g->G.build_box<Lc, Traversal::All>();
  FieldView<Q> pf = g->F.distributions();
  std::array<bool, 3> per = {bool(g->periodic[0]), bool(g->periodic[1]), bool(g->periodic[2])};
  int coord[3] = {0, 0, 0}, ndims[3] = {1, 1, 1};
  struct Pair {
    Box3D send, recv;
    std::vector<double> buf;
  };
  std::vector<Pair> comms;
  for (int i = 0; i < 27; i++) {  // make_domain.hpp:213-255
    int idx = i;
    int3d rel;
    for (int dim = 0; dim < 3; dim++) {
      int d = idx % 3;
      rel[dim] = d - 1;
      idx = (idx - d) / 3;
    }
    if (rel == int3d{0, 0, 0}) continue;
    bool per_b[3] = {per[0], per[1], per[2]};
    auto [exists, coord_neig] = build_comm(rel, std::span<int>(coord, 3), std::span<bool>(per_b, 3),
                                           std::span<int>(ndims, 3));
    if (!exists) continue;
    auto [send_box, recv_box] = build_boxes(rel, g->G);
    send_box = fix_box_with_periodicity(rel, g->G);
    comms.push_back({send_box, recv_box, std::vector<double>(size_t(send_box.number_of_points()) * Q)});
  }
  for (auto& c : comms) {  // do_pack_send
    FieldView<Q> wsend = {c.buf.data(), uint64_t(c.send.number_of_points())};
    packer<Q> pack = {wsend, pf, c.send, mesh_box};
    for (int z = c.send.start(2); z <= c.send.end(2); z++)
      for (int y = c.send.start(1); y <= c.send.end(1); y++)
        for (int x = c.send.start(0); x <= c.send.end(0); x++) pack(onikaInt3_t{x, y, z});
  }
  for (auto& c : comms) {  // do_unpack (the self-message buffer is the send buffer)
    FieldView<Q> wrecv = {c.buf.data(), uint64_t(c.recv.number_of_points())};
    unpacker<Q> unpack = {pf, wrecv, c.recv, mesh_box};
    for (int z = c.recv.start(2); z <= c.recv.end(2); z++)
      for (int y = c.recv.start(1); y <= c.recv.end(1); y++)
        for (int x = c.recv.start(0); x <= c.recv.end(0); x++) unpack(onikaInt3_t{x, y, z});
  }
}

void set_distribution_impl(RefLattice* g, double value, const double* bounds6, int do_update) {
  GridIJKtoIdx ijk_to_idx(g->G);
  FieldView<Q> pf = g->F.distributions();
  init_distributions<Q> func = {value, ijk_to_idx};
  if (bounds6) {
    double Dx = g->G.dx_;
    Point3D _min = {int(bounds6[0] / Dx), int(bounds6[1] / Dx), int(bounds6[2] / Dx)};
    Point3D _max = {int(bounds6[3] / Dx), int(bounds6[4] / Dx), int(bounds6[5] / Dx)};
    Box3D global_wall_box = {_min, _max};
    auto [inside, box] = g->G.restrict_box_to_grid<Area::Local, Traversal::Extend>(global_wall_box);
    if (!inside) return;
#pragma omp parallel for schedule(static)
    for (int z = box.start(2); z <= box.end(2); z++)
      for (int y = box.start(1); y <= box.end(1); y++)
        for (int x = box.start(0); x <= box.end(0); x++) func(x, y, z, pf);
  } else if (do_update) {
    auto [ptr, size_sb] = g->R.get_data<Traversal::Real>();
  const size_t size = size_sb;
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < size; i++) func(ptr[i], pf);
    update_ghost_impl(g);
  } else {
    auto [ptr, size_sb] = g->R.get_data<Traversal::All>();
  const size_t size = size_sb;
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < size; i++) func(ptr[i], pf);
  }
}

void lbm_parameters_impl(RefLattice* g, const double Fext[3], double celerity, double nuth, double avg_rho,
                         int has_tau, double tau, double dt) {  // lbm_parameters.cpp:73-99
  double Dx = g->G.dx_;
  LBMParameters params;
  params.nuth_ = nuth;
  params.avg_rho_ = avg_rho;
  if (dt > 0.0)
    params.define_by_dt(dt, Dx);
  else if (has_tau)
    params.define_by_tau(tau, Dx);
  else
    params.define_by_c(celerity, Dx);
  params.Fext_ = convert_force<LBM_UNITS>(Vec3d{Fext[0], Fext[1], Fext[2]}, params);
  g->P = params;
}
template <int dim, Side dir, bool pre>
void bb_launch(RefLattice* g) {  // pre_bounce_back.cu:70-86, post_bounce_back.cu:81-98
  int idx = helper_dim_idx<dim, dir>();
  FieldView<5> pfi = g->bb.get_data(idx);
  if (pfi.num_elements_ == 0) return;
  constexpr Traversal Tr = get_traversal<dim, dir>();
  auto [ptr, size_sb] = g->R.get_data<Tr>();
  const size_t size = size_sb;
  FieldView<Q> pf = g->F.distributions();
  if constexpr (pre) {
    pre_bounce_back<dim, dir, Q> kernel = {ptr};
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < size; i++) kernel(int(i), pf, pfi);
  } else {
    post_bounce_back<dim, dir, Q> kernel = {ptr};
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < size; i++) kernel(int(i), pf, pfi);
  }
}

template <Side S>
void cavity_launch(RefLattice* g, const double U[3]) {  // cavity.cu:66-88
  cavity<DIMZ, S, Q> bcs = {};
  constexpr int idx = helper_dim_idx<DIMZ, S>();
  FieldView<5> pfi = g->bb.get_data(idx);
  int* const pobst = g->F.obstacles();
  bcs.compute_coeff(U[0], U[1], U[2], g->n[0], g->n[1], g->n[2]);
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < pfi.num_elements_; i++) bcs(int(i), pobst, pfi);
}

template <class Functor>
void plane_apply(RefLattice* g, Traversal tr, const Vec3d& u) {
  traversal_data t = get_traversal(g->R, tr);
  Functor fn = {};
  int* pobst = g->F.obstacles();
  FieldView<Q> pf = g->F.distributions();
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < t.size_; i++) fn(t.ptr_[i], pobst, pf, u.x, u.y, u.z);
}

}  // namespace

extern "C" {

void* orc_create(const int32_t cell_dims[3], const double bmin[3], const double bmax[3], const int32_t periodic[3],
                 int32_t* err) {
  *err = 0;
  // domain (domain_lbm.cpp:66-110)
  onika::math::IJK grid_size = {cell_dims[0] + 1, cell_dims[1] + 1, cell_dims[2] + 1};
  Vec3d inf = {bmin[0], bmin[1], bmin[2]}, sup = {bmax[0], bmax[1], bmax[2]};
  Vec3d reso = {(sup.x - inf.x) / double(grid_size.i - 1), (sup.y - inf.y) / double(grid_size.j - 1),
                (sup.z - inf.z) / double(grid_size.k - 1)};
  if (reso.x != reso.y || reso.x != reso.z) {
    *err = -2;
    return nullptr;
  }
  double r = reso.x;
  if (inf.x + (grid_size.i - 1) * r != sup.x || inf.y + (grid_size.j - 1) * r != sup.y ||
      inf.z + (grid_size.k - 1) * r != sup.z) {
    *err = -3;
    return nullptr;
  }
  auto* g = new RefLattice();
  g->periodic = {periodic[0] != 0, periodic[1] != 0, periodic[2] != 0};
  g->n[0] = int(grid_size.i);
  g->n[1] = int(grid_size.j);
  g->n[2] = int(grid_size.k);
  // load_balancing on one rank (make_domain.hpp:278-349) + make_domain (make_domain.hpp:158-200)
  double GridDx = double(sup.x - inf.x) / double(grid_size.i - 1);
  constexpr int ghost_layer = 2;
  int3d size_with_ghost = {g->n[0] + 2 * ghost_layer - 1, g->n[1] + 2 * ghost_layer - 1,
                           g->n[2] + 2 * ghost_layer - 1};
  Box3D local_box = {{0, 0, 0}, size_with_ghost};
  Box3D ext = local_box;
  for (int dim = 0; dim < 3; dim++)
    if (!periodic[dim]) {
      ext.inf_[dim] += ghost_layer;
      ext.sup_[dim] -= ghost_layer;
    }
  g->G.set_box(local_box);
  g->G.set_ext(ext);
  g->G.set_offset(Point3D{-ghost_layer, -ghost_layer, -ghost_layer});
  g->G.set_ghost_layer(ghost_layer);
  g->G.set_dx(GridDx);
  g->G.set_origin(inf);
  // build_traversal (build_traversal.cpp:52-56)
  g->R.build_traversal(g->G, onika::math::IJK{0, 0, 0}, onika::math::IJK{1, 1, 1});
  // define_grid_3dq19 (define_lbm_fields.cpp:58-86)
  const size_t np = local_box.number_of_points();
  g->F.grid_size_ = np;
  g->F.f_.resize(np * Q, 0);
  g->F.obst_.resize(np);
  g->F.m0_.resize(np, 0);
  g->F.m1_.resize(np * 3, 0);
  // bounce-back buffers (pre_bounce_back.cu:101-107)
  auto ba = g->G.build_box<Area::Local, Traversal::All>();
  onika::math::IJK lgs = {ba.get_length(0), ba.get_length(1), ba.get_length(2)};
  g->bb.resize_data(g->periodic, lgs, onika::math::IJK{0, 0, 0}, onika::math::IJK{1, 1, 1});
  // init_obst (init_obst.cu)
  init_obst io = {g->F.obstacles()};
  for (size_t i = 0; i < np; i++) io(int(i));
  // set_distribution default (config_initialize.msp:22-23)
  set_distribution_impl(g, 1.0, nullptr, 0);
  double F0[3] = {0, 0, 0};
  lbm_parameters_impl(g, F0, 1.0, 1e-4, 1000.0, 0, 0.0, 0.0);
  return g;
}

void orc_destroy(void* h) { delete L(h); }

void orc_lbm_parameters(void* h, const double Fext[3], double celerity, double nuth, double avg_rho, int32_t has_tau,
                        double tau, double dt) {
  lbm_parameters_impl(L(h), Fext, celerity, nuth, avg_rho, has_tau, tau, dt);
}

void orc_get_parameters(void* h, double out[9]) {
  auto& p = L(h)->P;
  out[0] = p.Fext_.x;
  out[1] = p.Fext_.y;
  out[2] = p.Fext_.z;
  out[3] = p.celerity_;
  out[4] = p.dtLB_;
  out[5] = p.nuth_;
  out[6] = p.nu_;
  out[7] = p.tau_;
  out[8] = p.avg_rho_;
}

void orc_set_distribution(void* h, double value, const double* bounds6, int32_t do_update) {
  set_distribution_impl(L(h), value, bounds6, do_update);
}

void orc_init_obstacles(void* h) { L(h)->obstacles.clear(); }

static void put_obstacle(RefLattice* g, int id, std::variant<Ball, Wall, Quadric> v) {
  if (size_t(id) >= g->obstacles.size()) g->obstacles.resize(id + 1);
  g->obstacles[id] = std::make_unique<std::variant<Ball, Wall, Quadric>>(v);
}

void orc_register_ball(void* h, int32_t id, const double c[3], double radius) {
  put_obstacle(L(h), id, Ball(Vec3d{c[0], c[1], c[2]}, radius));
}
void orc_register_wall(void* h, int32_t id, const double bmin[3], const double bmax[3]) {
  put_obstacle(L(h), id, Wall(onika::math::AABB{{bmin[0], bmin[1], bmin[2]}, {bmax[0], bmax[1], bmax[2]}}));
}
void orc_register_quadric(void* h, int32_t id, const double q[16]) {
  onika::math::Mat4d m;
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) m.m[i][j] = q[i * 4 + j];
  put_obstacle(L(h), id, Quadric(m));
}

void orc_update_obstacles(void* h) {  // update_obstacles.cu:48-72 and :106-119
  RefLattice* g = L(h);
  LBMGrid grid = g->G;
  int* obst = g->F.obstacles();
  double dx_ = g->G.dx_;
  for (auto& slot : g->obstacles) {
    if (!slot) continue;
    std::visit(
        [&](auto& obj) {
          onika::math::AABB bounds = obj.covered();
          Vec3d mn = bounds.bmin, mx = bounds.bmax;
          Point3D _min = {int(mn.x / dx_), int(mn.y / dx_), int(mn.z / dx_)};
          Point3D _max = {int(mx.x / dx_), int(mx.y / dx_), int(mx.z / dx_)};
          Box3D global_box = {_min, _max};
          auto [inside, box] = grid.restrict_box_to_grid<Area::Local, Traversal::Extend>(global_box);
          if (!inside) return;
#pragma omp parallel for schedule(static)
          for (int k = box.start(2); k <= box.end(2); k++)
            for (int j = box.start(1); j <= box.end(1); j++)
              for (int i = box.start(0); i <= box.end(0); i++)
                if (obj.solid(grid.compute_position<Area::Global>(i, j, k))) obst[grid(i, j, k)] = WALL_;
        },
        *slot);
  }
}

void orc_macro_variables(void* h) {  // macro_variables.cu:71-90
  RefLattice* g = L(h);
  macro_variables<Q> func = {g->P.Fext_ / 2};
  FieldView<3> pm1 = g->F.flux();
  int* const pobst = g->F.obstacles();
  FieldView<Q> pf = g->F.distributions();
  double* const pm0 = g->F.densities();
  auto [ptr, size_sb] = g->R.get_data<Traversal::All>();
  const size_t size = size_sb;
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < size; i++) func(ptr[i], pm1, pobst, pf, pm0);
}

void orc_bgk(void* h) {  // bgk.cu:77-94
  RefLattice* g = L(h);
  auto [ptr, size_sb] = g->R.get_levels();
  const size_t size = size_sb;
  bgk<Q, Traversal::Real> func = {ptr, g->P.Fext_, g->F.flux(), g->F.obstacles(), g->F.distributions(),
                                  g->F.densities(), g->P.tau_};
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < size; i++) func(int(i));
}

void orc_mrt(void* h, const double* rates8) {  // mrt.cu:71-89
  if (rates8) {
    std::fprintf(stderr, "reference MRT rates are fixed (mrt.hpp:43-47)\n");
    std::abort();
  }
  RefLattice* g = L(h);
  mrt<Q> func = {g->P.Fext_};
  int* const pobst = g->F.obstacles();
  FieldView<Q> pf = g->F.distributions();
  double* const pm0 = g->F.densities();
  auto [ptr, size_sb] = g->R.get_data<Traversal::Real>();
  const size_t size = size_sb;
  const double tau = g->P.tau_;
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < size; i++) func(ptr[i], pobst, pf, pm0, tau);
}


void orc_pre_bounce_back(void* h) {
  RefLattice* g = L(h);
  bb_launch<0, Side::Left, true>(g);
  bb_launch<0, Side::Right, true>(g);
  bb_launch<1, Side::Left, true>(g);
  bb_launch<1, Side::Right, true>(g);
  bb_launch<2, Side::Left, true>(g);
  bb_launch<2, Side::Right, true>(g);
}

void orc_post_bounce_back(void* h) {
  RefLattice* g = L(h);
  bb_launch<0, Side::Left, false>(g);
  bb_launch<0, Side::Right, false>(g);
  bb_launch<1, Side::Left, false>(g);
  bb_launch<1, Side::Right, false>(g);
  bb_launch<2, Side::Left, false>(g);
  bb_launch<2, Side::Right, false>(g);
}


void orc_cavity(void* h, int32_t side, const double U[3]) {
  if (side)
    cavity_launch<Side::Right>(L(h), U);
  else
    cavity_launch<Side::Left>(L(h), U);
}

void orc_wall_bounce_back(void* h) {  // wall_bounce_back.cu:58-73
  RefLattice* g = L(h);
  wall_bounce_back<Q> func = {g->G, g->F.obstacles(), g->F.distributions()};
  Box3D extend = g->G.build_box<Area::Local, Traversal::Extend>();
#pragma omp parallel for schedule(static)
  for (int z = extend.start(2); z <= extend.end(2); z++)
    for (int y = extend.start(1); y <= extend.end(1); y++)
      for (int x = extend.start(0); x <= extend.end(0); x++) func(onikaInt3_t{x, y, z});
}

void orc_update_ghost(void* h) { update_ghost_impl(L(h)); }

void orc_streaming(void* h) {  // streaming.cu:68-118, asynchrone: false
  RefLattice* g = L(h);
  auto [ptr, size_sb] = g->R.get_levels();
  const size_t size = size_sb;
  FieldView<Q> pf = g->F.distributions();
  streaming_step1<Q, Traversal::Real> step1 = {ptr, pf};
  streaming_step2<Q, Traversal::Extend> step2 = {ptr, g->G, pf};
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < size; i++) step1(int(i));
  update_ghost_impl(g);
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < size; i++) step2(int(i));
}


int32_t orc_neumann(void* h, int32_t face, const double U[3]) {  // neuman.cu:69-122
  RefLattice* g = L(h);
  Vec3d u = convert_velocity<LBM_UNITS>(Vec3d{U[0], U[1], U[2]}, g->P);
  switch (face) {
    case 0: plane_apply<neumann_x_0<Q>>(g, Traversal::Plan_yz_0, u); break;
    case 1: plane_apply<neumann_x_l<Q>>(g, Traversal::Plan_yz_l, u); break;
    case 2: plane_apply<neumann_y_0<Q>>(g, Traversal::Plan_xz_0, u); break;
    case 3: plane_apply<neumann_y_l<Q>>(g, Traversal::Plan_xz_l, u); break;
    case 4: plane_apply<neumann_z_0<Q>>(g, Traversal::Plan_xy_0, u); break;
    case 5: plane_apply<neumann_z_l<Q>>(g, Traversal::Plan_xy_l, u); break;
    default: return -1;
  }
  return 0;
}

int32_t orc_lid_driven_cavity(void* h, int32_t face, const double U[3]) {  // lid_driven_cavity.cu:69-93
  RefLattice* g = L(h);
  if (face < 0 || face > 5) return -1;
  static const Traversal T[6] = {Traversal::Plan_yz_0, Traversal::Plan_yz_l, Traversal::Plan_xz_0,
                                 Traversal::Plan_xz_l, Traversal::Plan_xy_0, Traversal::Plan_xy_l};
  Vec3d uLB = convert_velocity<LBM_UNITS>(Vec3d{U[0], U[1], U[2]}, g->P);
  LidDrivenCavityBCsFunctor<Q> bcs = {uLB, g->F.distributions(), g->F.obstacles()};
  traversal_data t = get_traversal(g->R, T[face]);
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < t.size_; i++) bcs(t.ptr_[i]);
  return 0;
}

// init_double_couette (init_double_couette.cu:74-100): the reference functor over the Real box
void orc_init_double_couette(void* h, const double U[3], int32_t dim) {
  RefLattice* g = L(h);
  const Vec3d Uc = Vec3d{U[0], U[1], U[2]} / g->P.celerity_;
  FieldView<Q> pf = g->F.distributions();
  Box3D real = g->G.build_box<Area::Local, Traversal::Real>();
  auto run = [&](auto func) {
    for (int z = real.start(2); z <= real.end(2); z++)
      for (int y = real.start(1); y <= real.end(1); y++)
        for (int x = real.start(0); x <= real.end(0); x++) func(onikaInt3_t{x, y, z});
  };
  const Vec3d dU = Uc / (0.5 * (g->n[dim] - 1));
  if (dim == 0) run(InitDoubleCouetteFunc<Q, DIMX>{g->G, pf, dU, Uc});
  if (dim == 1) run(InitDoubleCouetteFunc<Q, DIMY>{g->G, pf, dU, Uc});
  if (dim == 2) run(InitDoubleCouetteFunc<Q, DIMZ>{g->G, pf, dU, Uc});
}

void orc_simulation_state(void* h, double out[3]) {  // simulation_state.cu:73-98, serial order
  RefLattice* g = L(h);
  ComputeSimulationStateFunc func = {g->F.densities(), g->F.flux()};
  SimulationStatistics s;
  auto [ptr, size_sb] = g->R.get_data<Traversal::Real>();
  const size_t size = size_sb;
  for (size_t i = 0; i < size; i++) func(s, uint64_t(ptr[i]), reduce_thread_local_t{});
  out[0] = s.sum_density_;
  out[1] = s.min_velocity_norm_;
  out[2] = s.max_velocity_norm_;
}

void orc_info(void* h, int64_t info[13]) {
  RefLattice* g = L(h);
  auto ba = g->G.build_box<Area::Local, Traversal::All>();
  for (int d = 0; d < 3; d++) {
    info[d] = ba.get_length(d);
    info[3 + d] = g->n[d];
  }
  info[6] = int64_t(g->F.grid_size_);
  static const Traversal T[6] = {Traversal::Plan_yz_0, Traversal::Plan_yz_l, Traversal::Plan_xz_0,
                                 Traversal::Plan_xz_l, Traversal::Plan_xy_0, Traversal::Plan_xy_l};
  for (int p = 0; p < 6; p++) info[7 + p] = int64_t(get_traversal(g->R, T[p]).size_);
}
double* orc_f(void* h) { return L(h)->F.f_.data(); }
double* orc_m0(void* h) { return L(h)->F.m0_.data(); }
double* orc_m1(void* h) { return L(h)->F.m1_.data(); }
int32_t* orc_obst(void* h) { return L(h)->F.obst_.data(); }
int32_t* orc_level(void* h) { return L(h)->R.level_.data(); }
}
