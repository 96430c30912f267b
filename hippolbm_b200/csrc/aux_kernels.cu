// aux_kernels.cu -- initialisation, obstacle rasterisation, macroscopic fields, FP64
// statistics and FP64 <-> storage conversion.  Compiled with --fmad=false so that the
// obstacle tests and the initial populations round exactly like the reference's.
#include <cuda_runtime.h>

#include <algorithm>

#include "aux_kernels.cuh"
#include "lbm_step_tma.cuh"

namespace hlbm {

// ------------------------------------------------------------------ set_distribution
// init_distributions (set_distribution.hpp:39-42): f_i = value * w_i on a box of nodes.
template <typename S, typename R>
__global__ void k_set_distribution(S* f, int64_t stride, int nx, int ny, int lo0, int lo1, int lo2, int hx,
                                   int hy, int hz, double value, const StepPlan p) {
  const int x = lo0 + blockIdx.x * blockDim.x + threadIdx.x;
  const int y = lo1 + blockIdx.y;
  const int z = lo2 + blockIdx.z;
  if (x > hx || y > hy || z > hz) return;
  const int64_t idx = ((int64_t)z * ny + y) * nx + x;
  Unroll<0, Q>::run([&]<int I>() {
    const double v = value * (1.0 / D3Q19::wden[I]);
    f[I * stride + idx] = Codec<S, R>::template enc<I>(R(v), p);
  });
}

// init_double_couette (double_couette.hpp:25-49, init_double_couette.cu:74-100): equilibrium of
// u = Uc - dU * g at every real node, g its global index along `dim`; FP64 in the reference's
// operation order, then stored.
template <typename S, typename R>
__global__ void k_double_couette(S* f, const StepPlan p, int dim, double ucx, double ucy, double ucz, double dux,
                                 double duy, double duz) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  const int z = blockIdx.z;
  if (x >= p.nx) return;
  const int64_t idx = ((int64_t)z * p.ny + y) * p.nx + x;
  const double g = dim == 0 ? double(x) : (dim == 1 ? double(y) : double(z));
  const double ux = ucx - dux * g, uy = ucy - duy * g, uz = ucz - duz * g;
  const double u_squ = ux * ux + uy * uy + uz * uz;
  Unroll<0, Q>::run([&]<int I>() {
    const double eu = ux * double(D3Q19::ex[I]) + uy * double(D3Q19::ey[I]) + uz * double(D3Q19::ez[I]);
    const double w = 1.0 / D3Q19::wden[I];
    const double v = 1. * w * (1. + 3. * eu + 4.5 * eu * eu - 1.5 * u_squ);
    f[I * p.stride + idx] = Codec<S, R>::template enc<I>(R(v), p);
  });
}

cudaError_t launch_double_couette(int prec, void* f, const StepPlan& p, int dim, const double uc[3],
                                  const double du[3], cudaStream_t s) {
  dim3 block(128), grid((p.nx + 127) / 128, p.ny, p.nz);
  switch (prec) {
    case 2:
      k_double_couette<float, float><<<grid, block, 0, s>>>(static_cast<float*>(f), p, dim, uc[0], uc[1], uc[2],
                                                            du[0], du[1], du[2]);
      break;
    case 3:
      k_double_couette<__half, float><<<grid, block, 0, s>>>(static_cast<__half*>(f), p, dim, uc[0], uc[1], uc[2],
                                                             du[0], du[1], du[2]);
      break;
    case 4:
      k_double_couette<__nv_bfloat16, float><<<grid, block, 0, s>>>(static_cast<__nv_bfloat16*>(f), p, dim, uc[0],
                                                                    uc[1], uc[2], du[0], du[1], du[2]);
      break;
    default:
      k_double_couette<double, double><<<grid, block, 0, s>>>(static_cast<double*>(f), p, dim, uc[0], uc[1], uc[2],
                                                              du[0], du[1], du[2]);
  }
  return cudaGetLastError();
}

// ------------------------------------------------------------------ zero-gradient outlet pass
// The pass over one face of lattice m of a descriptor array (lbm_step.cuh: zero_gradient_node),
// run before each step that pulls from f[cur ^ parity].
template <typename S, typename R>
__global__ void __launch_bounds__(256) k_zero_gradient(const LatticeDesc* __restrict__ lats, int m, int face,
                                                       int parity) {
  __shared__ StepPlan sp;
  const LatticeDesc L = lats[m];
  const uint32_t* src = reinterpret_cast<const uint32_t*>(L.plan);
  uint32_t* dst = reinterpret_cast<uint32_t*>(&sp);
  for (int w = threadIdx.x; w < int(sizeof(StepPlan) / 4); w += blockDim.x) dst[w] = src[w];
  __syncthreads();
  const StepPlan& p = sp;
  S* fin = static_cast<S*>(L.f[L.cur ^ parity]);
  const int axis = face / 2;
  const int na = axis == 0 ? p.ny : p.nx, nb = axis == 2 ? p.ny : p.nz;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < int64_t(na) * nb;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int a = int(k % na), b = int(k / na);
    switch (face) {
      case 0: zero_gradient_node<S, R, 0>(fin, L.flags, p, a, b); break;
      case 1: zero_gradient_node<S, R, 1>(fin, L.flags, p, a, b); break;
      case 2: zero_gradient_node<S, R, 2>(fin, L.flags, p, a, b); break;
      case 3: zero_gradient_node<S, R, 3>(fin, L.flags, p, a, b); break;
      case 4: zero_gradient_node<S, R, 4>(fin, L.flags, p, a, b); break;
      default: zero_gradient_node<S, R, 5>(fin, L.flags, p, a, b); break;
    }
  }
}

cudaError_t launch_zero_gradient(int prec, const LatticeDesc* lats, int m, int face, int parity, const int n[3],
                                 cudaStream_t s) {
  const int axis = face / 2;
  const int64_t nodes = int64_t(axis == 0 ? n[1] : n[0]) * (axis == 2 ? n[1] : n[2]);
  const int blocks = int(std::min<int64_t>((nodes + 255) / 256, 4 * 148));
  switch (prec) {
    case 2: k_zero_gradient<float, float><<<blocks, 256, 0, s>>>(lats, m, face, parity); break;
    case 3: k_zero_gradient<__half, float><<<blocks, 256, 0, s>>>(lats, m, face, parity); break;
    case 4: k_zero_gradient<__nv_bfloat16, float><<<blocks, 256, 0, s>>>(lats, m, face, parity); break;
    default: k_zero_gradient<double, double><<<blocks, 256, 0, s>>>(lats, m, face, parity); break;
  }
  return cudaGetLastError();
}

// ------------------------------------------------------------------ obstacles
// SetObstacleFunc (update_obstacles.cu:32-45): the node at real (x, y, z) sits at
// ((x + 2) - 2) * dx (compute_position<Global>, grid.hpp:355-361: the origin is not added).
__global__ void k_rasterize(int8_t* flags, int nx, int ny, int lo0, int lo1, int lo2, int hx, int hy, int hz,
                            double dx, ObstacleDesc o) {
  const int x = lo0 + blockIdx.x * blockDim.x + threadIdx.x;
  const int y = lo1 + blockIdx.y;
  const int z = lo2 + blockIdx.z;
  if (x > hx || y > hy || z > hz) return;
  const double px = ((double)(x + 2) + (double)(-2)) * dx;
  const double py = ((double)(y + 2) + (double)(-2)) * dx;
  const double pz = ((double)(z + 2) + (double)(-2)) * dx;
  bool solid = false;
  if (o.type == OBS_BALL) {  // Ball::solid (obstacle.hpp:59-62)
    const double rx = px - o.a[0], ry = py - o.a[1], rz = pz - o.a[2];
    solid = rx * rx + ry * ry + rz * rz <= o.a[4];
  } else if (o.type == OBS_WALL) {  // intersect (obstacle.hpp:13-17): strict interior
    solid = o.a[0] < px && px < o.a[3] && o.a[1] < py && py < o.a[4] && o.a[2] < pz && pz < o.a[5];
  } else if (o.type == OBS_QUADRIC) {  // p^T Q p <= 0 with p = (x, y, z, 1)
    const double pv[4] = {px, py, pz, 1.0};
    double acc = 0.0;
#pragma unroll
    for (int i = 0; i < 4; i++) {
      double row = 0.0;
#pragma unroll
      for (int j = 0; j < 4; j++) row = row + o.a[i * 4 + j] * pv[j];
      acc = acc + pv[i] * row;
    }
    solid = acc <= 0.0;
  }
  if (solid) flags[((int64_t)z * ny + y) * nx + x] = FLAG_WALL;
}

// ------------------------------------------------------------------ macro + statistics
// macro_variables (macro_variables.hpp:48-79) on a state S_k, in FP64, plus the per-block
// partials of simulation_state (simulation_state.hpp:47-54): sum rho, min |u|, max |u|.
// Walls keep rho = 0 and u = 0 (macro_variables never writes their m0).
template <typename S, typename R>
__global__ void __launch_bounds__(256) k_macro_stats(const S* __restrict__ f, const int8_t* __restrict__ flags,
                                                     int64_t ncell, double* __restrict__ rho_out,
                                                     double* __restrict__ u_out, double* __restrict__ partials,
                                                     const StepPlan p) {
  double s = 0.0, vmin = 1.79769313486231570815e+308, vmax = -1.79769313486231570815e+308;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < ncell;
       idx += (int64_t)gridDim.x * blockDim.x) {
    double rho = 0.0, ux = 0.0, uy = 0.0, uz = 0.0;
    if (flags[idx] >= FLAG_FLUID) {
      double v[Q];
      Unroll<0, Q>::run([&]<int I>() { v[I] = double(Codec<S, R>::template dec<I>(f[I * p.stride + idx], p)); });
      macro<double, true>(v, rho, ux, uy, uz);
    }
    if (rho_out) rho_out[idx] = rho;
    if (u_out) {
      u_out[idx] = ux;
      u_out[ncell + idx] = uy;
      u_out[2 * ncell + idx] = uz;
    }
    s += rho;
    const double n = sqrt(ux * ux + uy * uy + uz * uz);
    vmin = n < vmin ? n : vmin;
    vmax = n > vmax ? n : vmax;
  }
  // warp then block reduction (fixed order: deterministic for a fixed launch shape)
  for (int off = 16; off > 0; off >>= 1) {
    s += __shfl_down_sync(0xffffffffu, s, off);
    const double a = __shfl_down_sync(0xffffffffu, vmin, off);
    const double b = __shfl_down_sync(0xffffffffu, vmax, off);
    vmin = a < vmin ? a : vmin;
    vmax = b > vmax ? b : vmax;
  }
  __shared__ double sh[3][8];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    sh[0][warp] = s;
    sh[1][warp] = vmin;
    sh[2][warp] = vmax;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = blockDim.x >> 5;
    double a = sh[0][0], b = sh[1][0], c = sh[2][0];
    for (int w = 1; w < nw; w++) {
      a += sh[0][w];
      b = sh[1][w] < b ? sh[1][w] : b;
      c = sh[2][w] > c ? sh[2][w] : c;
    }
    partials[3 * blockIdx.x + 0] = a;
    partials[3 * blockIdx.x + 1] = b;
    partials[3 * blockIdx.x + 2] = c;
  }
}

// second pass: one block folds the per-block partials in block order
__global__ void k_reduce_partials(const double* __restrict__ partials, int nparts, double* __restrict__ out) {
  __shared__ double sh[3][256];
  double s = 0.0, vmin = 1.79769313486231570815e+308, vmax = -1.79769313486231570815e+308;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
    s += partials[3 * i];
    vmin = partials[3 * i + 1] < vmin ? partials[3 * i + 1] : vmin;
    vmax = partials[3 * i + 2] > vmax ? partials[3 * i + 2] : vmax;
  }
  sh[0][threadIdx.x] = s;
  sh[1][threadIdx.x] = vmin;
  sh[2][threadIdx.x] = vmax;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) {
      sh[0][threadIdx.x] += sh[0][threadIdx.x + h];
      sh[1][threadIdx.x] = sh[1][threadIdx.x + h] < sh[1][threadIdx.x] ? sh[1][threadIdx.x + h] : sh[1][threadIdx.x];
      sh[2][threadIdx.x] = sh[2][threadIdx.x + h] > sh[2][threadIdx.x] ? sh[2][threadIdx.x + h] : sh[2][threadIdx.x];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = sh[0][0];
    out[1] = sh[1][0];
    out[2] = sh[2][0];
  }
}

// ------------------------------------------------------------------ sums over the lattice
// Per-block FP64 partial sums of up to 4 quantities, folded by k_fold_sums in block order.
template <int NS>
__device__ __forceinline__ void block_sums(double (&acc)[NS], double* partials) {
  for (int off = 16; off > 0; off >>= 1)
#pragma unroll
    for (int k = 0; k < NS; k++) acc[k] += __shfl_down_sync(0xffffffffu, acc[k], off);
  __shared__ double sh[NS][8];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NS; k++) sh[k][warp] = acc[k];
  __syncthreads();
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < NS; k++) {
      double a = sh[k][0];
      for (int w = 1; w < int(blockDim.x >> 5); w++) a += sh[k][w];
      partials[4 * blockIdx.x + k] = a;
    }
}

__global__ void k_fold_sums(const double* __restrict__ partials, int nparts, double* __restrict__ out) {
  __shared__ double sh[4][256];
  double a[4] = {0, 0, 0, 0};
  for (int i = threadIdx.x; i < nparts; i += blockDim.x)
#pragma unroll
    for (int k = 0; k < 4; k++) a[k] += partials[4 * i + k];
#pragma unroll
  for (int k = 0; k < 4; k++) sh[k][threadIdx.x] = a[k];
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h)
#pragma unroll
      for (int k = 0; k < 4; k++) sh[k][threadIdx.x] += sh[k][threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < 4; k++) out[k] = sh[k][0];
}

// steady-state residual: sum |u - u_prev|^2 and sum |u|^2 (FP64), then u_prev <- u (FP32 copy)
template <typename S, typename R>
__global__ void __launch_bounds__(256) k_residual(const S* __restrict__ f, const int8_t* __restrict__ flags,
                                                  int64_t ncell, float* __restrict__ uprev, int first,
                                                  double* __restrict__ partials, const StepPlan p) {
  double acc[4] = {0, 0, 0, 0};
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < ncell;
       idx += (int64_t)gridDim.x * blockDim.x) {
    if (flags[idx] < FLAG_FLUID) continue;
    double v[Q], rho, ux, uy, uz;
    Unroll<0, Q>::run([&]<int I>() { v[I] = double(Codec<S, R>::template dec<I>(f[I * p.stride + idx], p)); });
    macro<double, true>(v, rho, ux, uy, uz);
    const double px = uprev[idx], py = uprev[ncell + idx], pz = uprev[2 * ncell + idx];
    if (!first) acc[0] += (ux - px) * (ux - px) + (uy - py) * (uy - py) + (uz - pz) * (uz - pz);
    acc[1] += ux * ux + uy * uy + uz * uz;
    uprev[idx] = float(ux);
    uprev[ncell + idx] = float(uy);
    uprev[2 * ncell + idx] = float(uz);
  }
  block_sums<4>(acc, partials);
}

// total mass and momentum: sum rho, sum rho u over fluid and passive nodes (FP64)
template <typename S, typename R>
__global__ void __launch_bounds__(256) k_moments(const S* __restrict__ f, const int8_t* __restrict__ flags,
                                                 int64_t ncell, double* __restrict__ partials, const StepPlan p) {
  double acc[4] = {0, 0, 0, 0};
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < ncell;
       idx += (int64_t)gridDim.x * blockDim.x) {
    if (flags[idx] < FLAG_FLUID) continue;
    double v[Q];
    Unroll<0, Q>::run([&]<int I>() { v[I] = double(Codec<S, R>::template dec<I>(f[I * p.stride + idx], p)); });
    double rho = v[0];
    for (int i = 1; i < Q; i++) rho += v[i];
    acc[0] += rho;
    acc[1] += ((((((((v[1] - v[2]) + v[7]) - v[8]) + v[9]) - v[10]) + v[11]) - v[12]) + v[13]) - v[14];
    acc[2] += ((((((((v[3] - v[4]) + v[7]) - v[8]) - v[9]) + v[10]) + v[15]) - v[16]) + v[17]) - v[18];
    acc[3] += ((((((((v[5] - v[6]) + v[11]) - v[12]) - v[13]) + v[14]) + v[15]) - v[16]) - v[17]) + v[18];
  }
  block_sums<4>(acc, partials);
}

// Force on the walls by momentum exchange (no reference counterpart): for every fluid node x and
// direction i whose neighbour x + e_i is a wall, the post-collision population f*_i(x) hits the
// wall and comes back reversed, transferring 2 f*_i(x) e_i.  Reads the post-collision state.
template <typename S, typename R>
__global__ void __launch_bounds__(256) k_wall_force(const S* __restrict__ fpost, const int8_t* __restrict__ flags,
                                                    double* __restrict__ partials, const StepPlan p) {
  double acc[4] = {0, 0, 0, 0};
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < p.ncell;
       idx += (int64_t)gridDim.x * blockDim.x) {
    if (flags[idx] != FLAG_FLUID) continue;
    const int x = int(idx % p.nx), y = int((idx / p.nx) % p.ny), z = int(idx / (int64_t(p.nx) * p.ny));
    Unroll<1, Q>::run([&]<int I>() {
      int xn = x + D3Q19::ex[I], yn = y + D3Q19::ey[I], zn = z + D3Q19::ez[I];
      if (xn < 0 || xn >= p.nx) { if (!p.periodic[0]) return; xn = xn < 0 ? xn + p.nx : xn - p.nx; }
      if (yn < 0 || yn >= p.ny) { if (!p.periodic[1]) return; yn = yn < 0 ? yn + p.ny : yn - p.ny; }
      if (zn < 0 || zn >= p.nz) { if (!p.periodic[2]) return; zn = zn < 0 ? zn + p.nz : zn - p.nz; }
      if (flags[(int64_t(zn) * p.ny + yn) * p.nx + xn] != FLAG_WALL) return;
      const double fi = double(Codec<S, R>::template dec<I>(fpost[I * p.stride + idx], p));
      acc[0] += 2.0 * fi * D3Q19::ex[I];
      acc[1] += 2.0 * fi * D3Q19::ey[I];
      acc[2] += 2.0 * fi * D3Q19::ez[I];
    });
  }
  block_sums<4>(acc, partials);
}

// ------------------------------------------------------------------ FP64 <-> storage
template <typename S, typename R, int I>
__device__ __forceinline__ void dec_plane(const S* f, double* out, int64_t n, const StepPlan& p) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = double(Codec<S, R>::template dec<I>(f[I * p.stride + i], p));
}
template <typename S, typename R>
__global__ void k_decode(const S* __restrict__ f, double* __restrict__ out, int dir, int64_t n, const StepPlan p) {
  Unroll<0, Q>::run([&]<int I>() {
    if (I == dir) dec_plane<S, R, I>(f, out, n, p);
  });
}
template <typename S, typename R>
__global__ void k_encode(S* __restrict__ f, const double* __restrict__ in, int dir, int64_t n, const StepPlan p) {
  Unroll<0, Q>::run([&]<int I>() {
    if (I != dir) return;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      f[I * p.stride + i] = Codec<S, R>::template enc<I>(R(in[i]), p);
  });
}

// ------------------------------------------------------------------ host launchers
template <typename S, typename R>
static cudaError_t set_dist_t(void* f, const StepPlan& p, const int lo[3], const int hi[3], double value,
                              cudaStream_t s) {
  const int w = hi[0] - lo[0] + 1;
  dim3 block(w >= 128 ? 128 : ((w + 31) / 32) * 32), grid((w + block.x - 1) / block.x, hi[1] - lo[1] + 1,
                                                             hi[2] - lo[2] + 1);
  k_set_distribution<S, R><<<grid, block, 0, s>>>(static_cast<S*>(f), p.stride, p.nx, p.ny, lo[0], lo[1], lo[2],
                                                  hi[0], hi[1], hi[2], value, p);
  return cudaGetLastError();
}

cudaError_t launch_set_distribution(int prec, void* f, const StepPlan& p, const int lo[3], const int hi[3],
                                    double value, cudaStream_t s) {
  switch (prec) {
    case 0:
    case 1: return set_dist_t<double, double>(f, p, lo, hi, value, s);
    case 2: return set_dist_t<float, float>(f, p, lo, hi, value, s);
    case 3: return set_dist_t<__half, float>(f, p, lo, hi, value, s);
    default: return set_dist_t<__nv_bfloat16, float>(f, p, lo, hi, value, s);
  }
}

cudaError_t launch_rasterize(int8_t* flags, const StepPlan& p, const int lo[3], const int hi[3], double dx,
                             const ObstacleDesc& o, cudaStream_t s) {
  const int w = hi[0] - lo[0] + 1;
  dim3 block(w >= 128 ? 128 : ((w + 31) / 32) * 32), grid((w + block.x - 1) / block.x, hi[1] - lo[1] + 1,
                                                             hi[2] - lo[2] + 1);
  k_rasterize<<<grid, block, 0, s>>>(flags, p.nx, p.ny, lo[0], lo[1], lo[2], hi[0], hi[1], hi[2], dx, o);
  return cudaGetLastError();
}

// near[idx] = 1 when a direction of node idx pulls from a wall node (the pull the step kernels
// replace by on-node bounce-back under wall_bounce_back), with the gather's periodic wrap; pulls
// from outside a non-periodic face bounce anyway and are not counted.
__global__ void k_near_wall(const int8_t* __restrict__ flags, int8_t* __restrict__ near, int nx, int ny, int nz,
                            int px, int py, int pz) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, z = blockIdx.z;
  if (x >= nx) return;
  int8_t any = 0;
  for (int dz = -1; dz <= 1; dz++)
    for (int dy = -1; dy <= 1; dy++)
      for (int dx = -1; dx <= 1; dx++) {
        const int m = (dx != 0) + (dy != 0) + (dz != 0);
        if (m == 0 || m == 3) continue;  // D3Q19: the 6 axis and 12 edge neighbours
        int sx = x + dx, sy = y + dy, sz = z + dz;
        if (sx < 0 || sx >= nx) { if (!px) continue; sx = sx < 0 ? sx + nx : sx - nx; }
        if (sy < 0 || sy >= ny) { if (!py) continue; sy = sy < 0 ? sy + ny : sy - ny; }
        if (sz < 0 || sz >= nz) { if (!pz) continue; sz = sz < 0 ? sz + nz : sz - nz; }
        if (flags[(int64_t(sz) * ny + sy) * nx + sx] == FLAG_WALL) any = 1;
      }
  near[(int64_t(z) * ny + y) * nx + x] = any;
}

cudaError_t launch_near_wall(const int8_t* flags, int8_t* near, const int n[3], const int periodic[3],
                             cudaStream_t s) {
  const dim3 block(n[0] >= 128 ? 128 : ((n[0] + 31) / 32) * 32);
  const dim3 grid((n[0] + block.x - 1) / block.x, n[1], n[2]);
  k_near_wall<<<grid, block, 0, s>>>(flags, near, n[0], n[1], n[2], periodic[0], periodic[1], periodic[2]);
  return cudaGetLastError();
}

int stats_blocks(int64_t ncell) {
  int64_t b = (ncell + 255) / 256;
  return int(b < 148 * 8 ? b : 148 * 8);
}

template <typename S, typename R>
static cudaError_t macro_stats_t(const void* f, const int8_t* flags, const StepPlan& p, double* rho, double* u,
                                 double* partials, double* out3, cudaStream_t s) {
  const int nb = stats_blocks(p.ncell);
  k_macro_stats<S, R><<<nb, 256, 0, s>>>(static_cast<const S*>(f), flags, p.ncell, rho, u, partials, p);
  k_reduce_partials<<<1, 256, 0, s>>>(partials, nb, out3);
  return cudaGetLastError();
}

cudaError_t launch_macro_stats(int prec, const void* f, const int8_t* flags, const StepPlan& p, double* rho,
                               double* u, double* partials, double* out3, cudaStream_t s) {
  switch (prec) {
    case 0:
    case 1: return macro_stats_t<double, double>(f, flags, p, rho, u, partials, out3, s);
    case 2: return macro_stats_t<float, float>(f, flags, p, rho, u, partials, out3, s);
    case 3: return macro_stats_t<__half, float>(f, flags, p, rho, u, partials, out3, s);
    default: return macro_stats_t<__nv_bfloat16, float>(f, flags, p, rho, u, partials, out3, s);
  }
}

#define HLBM_PREC_DISPATCH(prec, CALL)                          \
  switch (prec) {                                               \
    case 2: { using S = float; using R = float; CALL; break; }  \
    case 3: { using S = __half; using R = float; CALL; break; } \
    case 4: { using S = __nv_bfloat16; using R = float; CALL; break; } \
    default: { using S = double; using R = double; CALL; break; } \
  }

cudaError_t launch_residual(int prec, const void* f, const int8_t* flags, const StepPlan& p, float* uprev, int first,
                            double* partials, double* out4, cudaStream_t s) {
  const int nb = stats_blocks(p.ncell);
  HLBM_PREC_DISPATCH(prec, (k_residual<S, R><<<nb, 256, 0, s>>>(static_cast<const S*>(f), flags, p.ncell, uprev,
                                                                    first, partials, p)));
  k_fold_sums<<<1, 256, 0, s>>>(partials, nb, out4);
  return cudaGetLastError();
}

cudaError_t launch_moments(int prec, const void* f, const int8_t* flags, const StepPlan& p, double* partials,
                           double* out4, cudaStream_t s) {
  const int nb = stats_blocks(p.ncell);
  HLBM_PREC_DISPATCH(prec, (k_moments<S, R><<<nb, 256, 0, s>>>(static_cast<const S*>(f), flags, p.ncell, partials, p)));
  k_fold_sums<<<1, 256, 0, s>>>(partials, nb, out4);
  return cudaGetLastError();
}

cudaError_t launch_wall_force(int prec, const void* fpost, const int8_t* flags, const StepPlan& p, double* partials,
                              double* out4, cudaStream_t s) {
  const int nb = stats_blocks(p.ncell);
  HLBM_PREC_DISPATCH(prec, (k_wall_force<S, R><<<nb, 256, 0, s>>>(static_cast<const S*>(fpost), flags, partials, p)));
  k_fold_sums<<<1, 256, 0, s>>>(partials, nb, out4);
  return cudaGetLastError();
}

// plane_velocity_profile (plane_velocity_profile.cu:64-90, 179-260): per plane normal to `dim`,
// the sum, count, minimum and maximum over fluid nodes of |ratio * u| (FP64, u from the same
// macro arithmetic as the statistics).  One block per plane, fixed thread-to-node assignment and a
// fixed-order reduction: deterministic.
template <typename S, typename R>
__global__ void __launch_bounds__(256) k_plane_profile(const S* __restrict__ f, const int8_t* __restrict__ flags,
                                                       const StepPlan p, int dim, double ratio,
                                                       double* __restrict__ out) {
  const int plane = blockIdx.x;
  const int64_t nplane = dim == 0 ? int64_t(p.ny) * p.nz : (dim == 1 ? int64_t(p.nx) * p.nz : int64_t(p.nx) * p.ny);
  double sum = 0.0, cnt = 0.0, vmin = 1.79769313486231570815e+308, vmax = -1.79769313486231570815e+308;
  for (int64_t k = threadIdx.x; k < nplane; k += blockDim.x) {
    int64_t idx;
    if (dim == 2) {
      idx = int64_t(plane) * p.nx * p.ny + k;
    } else if (dim == 1) {
      const int64_t z = k / p.nx, x = k - z * p.nx;
      idx = (z * p.ny + plane) * p.nx + x;
    } else {
      idx = k * p.nx + plane;
    }
    if (flags[idx] != FLAG_FLUID) continue;
    double v[Q];
    Unroll<0, Q>::run([&]<int I>() { v[I] = double(Codec<S, R>::template dec<I>(f[I * p.stride + idx], p)); });
    double rho, ux, uy, uz;
    macro<double, true>(v, rho, ux, uy, uz);
    const double ax = ratio * ux, ay = ratio * uy, az = ratio * uz;
    const double n = sqrt(ax * ax + ay * ay + az * az);
    sum += n;
    cnt += 1.0;
    vmin = n < vmin ? n : vmin;
    vmax = n > vmax ? n : vmax;
  }
  for (int off = 16; off > 0; off >>= 1) {
    sum += __shfl_down_sync(0xffffffffu, sum, off);
    cnt += __shfl_down_sync(0xffffffffu, cnt, off);
    const double a = __shfl_down_sync(0xffffffffu, vmin, off);
    const double b = __shfl_down_sync(0xffffffffu, vmax, off);
    vmin = a < vmin ? a : vmin;
    vmax = b > vmax ? b : vmax;
  }
  __shared__ double sh[4][8];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    sh[0][warp] = sum;
    sh[1][warp] = cnt;
    sh[2][warp] = vmin;
    sh[3][warp] = vmax;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = sh[0][0], c = sh[1][0], lo = sh[2][0], hi = sh[3][0];
    for (int w = 1; w < int(blockDim.x >> 5); w++) {
      a += sh[0][w];
      c += sh[1][w];
      lo = sh[2][w] < lo ? sh[2][w] : lo;
      hi = sh[3][w] > hi ? sh[3][w] : hi;
    }
    out[4 * plane + 0] = a;
    out[4 * plane + 1] = c;
    out[4 * plane + 2] = lo;
    out[4 * plane + 3] = hi;
  }
}

cudaError_t launch_plane_profile(int prec, const void* f, const int8_t* flags, const StepPlan& p, int dim,
                                 double ratio, double* out4n, cudaStream_t s) {
  const int n = dim == 0 ? p.nx : (dim == 1 ? p.ny : p.nz);
  HLBM_PREC_DISPATCH(prec, (k_plane_profile<S, R><<<n, 256, 0, s>>>(static_cast<const S*>(f), flags, p, dim, ratio,
                                                                     out4n)));
  return cudaGetLastError();
}

// 16-bit storage re-encoding: decode under the old storage parameters, encode under the new
template <typename S, typename R>
__global__ void k_reencode(S* __restrict__ f, const StepPlan po, const StepPlan pn) {
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < pn.ncell;
       idx += (int64_t)gridDim.x * blockDim.x)
    Unroll<0, Q>::run([&]<int I>() {
      S* a = f + I * pn.stride + idx;
      *a = Codec<S, R>::template enc<I>(Codec<S, R>::template dec<I>(*a, po), pn);
    });
}

cudaError_t launch_reencode(int prec, void* f, const StepPlan& old_plan, const StepPlan& new_plan, cudaStream_t s) {
  const int nb = stats_blocks(new_plan.ncell);
  if (prec == 3)
    k_reencode<__half, float><<<nb, 256, 0, s>>>(static_cast<__half*>(f), old_plan, new_plan);
  else if (prec == 4)
    k_reencode<__nv_bfloat16, float><<<nb, 256, 0, s>>>(static_cast<__nv_bfloat16*>(f), old_plan, new_plan);
  return cudaGetLastError();
}

cudaError_t launch_decode(int prec, const void* f, double* out, int dir, const StepPlan& p, cudaStream_t s) {
  const int nb = stats_blocks(p.ncell);
  switch (prec) {
    case 2: k_decode<float, float><<<nb, 256, 0, s>>>(static_cast<const float*>(f), out, dir, p.ncell, p); break;
    case 3: k_decode<__half, float><<<nb, 256, 0, s>>>(static_cast<const __half*>(f), out, dir, p.ncell, p); break;
    case 4:
      k_decode<__nv_bfloat16, float><<<nb, 256, 0, s>>>(static_cast<const __nv_bfloat16*>(f), out, dir, p.ncell, p);
      break;
    default: k_decode<double, double><<<nb, 256, 0, s>>>(static_cast<const double*>(f), out, dir, p.ncell, p); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_encode(int prec, void* f, const double* in, int dir, const StepPlan& p, cudaStream_t s) {
  const int nb = stats_blocks(p.ncell);
  switch (prec) {
    case 2: k_encode<float, float><<<nb, 256, 0, s>>>(static_cast<float*>(f), in, dir, p.ncell, p); break;
    case 3: k_encode<__half, float><<<nb, 256, 0, s>>>(static_cast<__half*>(f), in, dir, p.ncell, p); break;
    case 4:
      k_encode<__nv_bfloat16, float><<<nb, 256, 0, s>>>(static_cast<__nv_bfloat16*>(f), in, dir, p.ncell, p);
      break;
    default: k_encode<double, double><<<nb, 256, 0, s>>>(static_cast<double*>(f), in, dir, p.ncell, p); break;
  }
  return cudaGetLastError();
}

}  // namespace hlbm
