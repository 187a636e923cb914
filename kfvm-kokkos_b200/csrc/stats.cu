// stats.cu -- flow statistics of the state (FlowStats<Eq>: src/physics/hydro/Hydro_K.H:103-178,
// src/physics/navierstokes/NavierStokes_K.H:102-175, src/physics/mhd_glm/MHD_GLM_K.H:108-211;
// driven by Solver::evalFlowStats, src/Solver.cpp:153-185, of slug-cfd/kfvm-kokkos):
// volume averages of the kinetic energy |m|^2 / (2 rho), the enstrophy rho |curl v|^2 / 2
// with the velocity gradients by central differences, and for GLM-MHD the current
// helicity B . curl B.  SRHydro reports one statistic that stays 0, as the reference's.
// One partial triple per block of kStatBlock cells, then a fixed-order sum.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/kfvm_b200.h"
#include "kernels.cuh"
#include "launch.h"

namespace kfvm {

constexpr int kStatBlock = 256;

template <int DIM, bool GLM>
__global__ void __launch_bounds__(kStatBlock)
    stats_kernel(const double *__restrict__ U, Grid g, double ifac, double *__restrict__ part) {
  const int64_t c = blockIdx.x * (int64_t)kStatBlock + threadIdx.x;
  double ek = 0.0, et = 0.0, hl = 0.0;
  if (c < g.n) {
    const int64_t i = c % g.nx, j = (c / g.nx) % g.ny, k = c / (g.nx * g.ny);
    const double *Uc = U + pidx(g, i, j, k);
    const int64_t sy = g.px, sz = g.px * g.py;
    auto u = [&](int64_t o, int v) { return Uc[v * g.pvol + o]; };
    // velocity component v (MOMX..MOMZ) at offset o
    auto vel = [&](int64_t o, int v) { return u(o, v) / u(o, DENS); };
    const double rho = u(0, DENS);
    ek = 0.5 * (u(0, MOMX) * u(0, MOMX) + u(0, MOMY) * u(0, MOMY) + u(0, MOMZ) * u(0, MOMZ)) / rho;
    const double dyu = 0.5 * (vel(sy, MOMX) - vel(-sy, MOMX)) / g.dy;
    const double dxv = 0.5 * (vel(1, MOMY) - vel(-1, MOMY)) / g.dx;
    double dzu = 0.0, dzv = 0.0, dxw = 0.0, dyw = 0.0;
    if (DIM == 3) {
      dzu = 0.5 * (vel(sz, MOMX) - vel(-sz, MOMX)) / g.dz;
      dzv = 0.5 * (vel(sz, MOMY) - vel(-sz, MOMY)) / g.dz;
      dxw = 0.5 * (vel(1, MOMZ) - vel(-1, MOMZ)) / g.dx;
      dyw = 0.5 * (vel(sy, MOMZ) - vel(-sy, MOMZ)) / g.dy;
    }
    const double omx = dyw - dzv, omy = dzu - dxw, omz = dxv - dyu;
    et = 0.5 * rho * (omx * omx + omy * omy + omz * omz);
    if (GLM) {
      const double dybx = 0.5 * (u(sy, MAGX) - u(-sy, MAGX)) / g.dy;
      const double dxby = 0.5 * (u(1, MAGY) - u(-1, MAGY)) / g.dx;
      double dzbx = 0.0, dzby = 0.0, dxbz = 0.0, dybz = 0.0;
      if (DIM == 3) {
        dzbx = 0.5 * (u(sz, MAGX) - u(-sz, MAGX)) / g.dz;
        dzby = 0.5 * (u(sz, MAGY) - u(-sz, MAGY)) / g.dz;
        dxbz = 0.5 * (u(1, MAGZ) - u(-1, MAGZ)) / g.dx;
        dybz = 0.5 * (u(sy, MAGZ) - u(-sy, MAGZ)) / g.dy;
      }
      const double cbx = dybz - dzby, cby = dzbx - dxbz, cbz = dxby - dybx;
      hl = u(0, MAGX) * cbx + u(0, MAGY) * cby + u(0, MAGZ) * cbz;
    }
    ek *= ifac;
    et *= ifac;
    hl *= ifac;
  }
  __shared__ double s[3][kStatBlock];
  s[0][threadIdx.x] = ek;
  s[1][threadIdx.x] = et;
  s[2][threadIdx.x] = hl;
  __syncthreads();
  for (int h = kStatBlock / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h)
      for (int q = 0; q < 3; q++) s[q][threadIdx.x] += s[q][threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x < 3) part[3 * blockIdx.x + threadIdx.x] = s[threadIdx.x][0];
}

__global__ void __launch_bounds__(1024) stats_sum_kernel(const double *__restrict__ part, int64_t nblk,
                                                         double *__restrict__ out) {
  __shared__ double s[3][1024];
  double a[3] = {0.0, 0.0, 0.0};
  for (int64_t t = threadIdx.x; t < nblk; t += 1024)
    for (int q = 0; q < 3; q++) a[q] += part[3 * t + q];
  for (int q = 0; q < 3; q++) s[q][threadIdx.x] = a[q];
  __syncthreads();
  for (int h = 512; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h)
      for (int q = 0; q < 3; q++) s[q][threadIdx.x] += s[q][threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x < 3) out[threadIdx.x] = s[threadIdx.x][0];
}

int64_t stats_blocks(const Grid &g) { return (g.n + kStatBlock - 1) / kStatBlock; }

int stats_count(int eq) { return eq == KFVM_EQ_MHD_GLM ? 3 : (eq == KFVM_EQ_SRHYDRO ? 1 : 2); }

cudaError_t launch_stats(int dim, int eq, const double *U, const Grid &g, double ifac, double *part, double *out,
                         cudaStream_t s) {
  const int64_t nblk = stats_blocks(g);
  if (eq == KFVM_EQ_SRHYDRO) return cudaMemsetAsync(out, 0, 3 * sizeof(double), s);
  const bool glm = eq == KFVM_EQ_MHD_GLM;
  if (dim == 2 && !glm) stats_kernel<2, false><<<(unsigned)nblk, kStatBlock, 0, s>>>(U, g, ifac, part);
  else if (dim == 3 && !glm) stats_kernel<3, false><<<(unsigned)nblk, kStatBlock, 0, s>>>(U, g, ifac, part);
  else if (dim == 2) stats_kernel<2, true><<<(unsigned)nblk, kStatBlock, 0, s>>>(U, g, ifac, part);
  else stats_kernel<3, true><<<(unsigned)nblk, kStatBlock, 0, s>>>(U, g, ifac, part);
  stats_sum_kernel<<<1, 1024, 0, s>>>(part, nblk, out);
  return cudaGetLastError();
}

} // namespace kfvm
