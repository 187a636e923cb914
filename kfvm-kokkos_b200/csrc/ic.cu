// ic.cu -- initial conditions as cell averages by Q^d Gauss quadrature (Q = 2 or 3)
// (IntegrateIC_K, src/numeric/Numeric_K.H:31-107 of slug-cfd/kfvm-kokkos) for
// the built-in problems.  The pointwise formulas are the problem library's
// InitialCondition.H functions with the benchmark problems' parameters:
//   isentropic vortex   exec/Hydro/IsenVort/InitialCondition.H (Shu's vortex, beta=5,
//                       freestream rho=u=v=p=1)
//   spherical Sod       rho,p = 1,1 inside r<0.2 around the box centre, 0.125,0.1 outside
//   Kelvin-Helmholtz    exec/Hydro/KelvinHelmholtz (slab |y-1/2|<1/4, seeded noise on v)
//   Taylor-Green        exec/NavierStokes/TaylorGreen/InitialCondition.H:9-31, Mach 0.1
//   Orszag-Tang         exec/MHD/OrszagTang/InitialCondition.H:9-36 at z=0
#include <cuda_runtime.h>

#include <cstdint>

#include "geometry.h"
#include "kernels.cuh"
#include "launch.h"

namespace kfvm {

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

struct IcParams {
  int kind, dim, eq;
  double gamma, xlo, xup, ylo, yup, zlo, zup;  // the whole domain
  double x0, y0, z0;                            // this block's first face per axis
};

__device__ void ic_point(const IcParams &p, double x, double y, double z, double noise,
                         double *s) {
  const double g = p.gamma, gm = g - 1.0;
  const double pi = 3.14159265358979323846;
#pragma unroll
  for (int v = 0; v < 9; v++) s[v] = 0.0;
  switch (p.kind) {
  case KFVM_IC_ISENTROPIC_VORTEX: {
    const double beta = 5.0, r2 = x * x + y * y;
    const double f = beta / (2.0 * pi) * exp(0.5 * (1.0 - r2));
    const double u = 1.0 - y * f, v = 1.0 + x * f;
    const double T = 1.0 - gm * beta * beta / (8.0 * g * pi * pi) * exp(1.0 - r2);
    const double rho = pow(T, 1.0 / gm), pr = rho * T;
    s[DENS] = rho;
    s[MOMX] = rho * u;
    s[MOMY] = rho * v;
    s[ETOT] = pr / gm + 0.5 * rho * (u * u + v * v);
    break;
  }
  case KFVM_IC_SPHERICAL_SOD: {
    const double dx = x - 0.5, dy = y - 0.5, dz = z - 0.5;
    const bool in = sqrt(dx * dx + dy * dy + dz * dz) < 0.2;
    const double rho = in ? 1.0 : 0.125, pr = in ? 1.0 : 0.1;
    s[DENS] = rho;
    s[ETOT] = pr / gm;
    break;
  }
  case KFVM_IC_KELVIN_HELMHOLTZ: {
    const bool in = fabs(y - 0.5) < 0.25;
    const double rho = in ? 2.0 : 1.0, u = in ? 0.5 : -0.5, pr = 2.5;
    const double v = 0.01 * sin(4.0 * pi * x) + noise;
    s[DENS] = rho;
    s[MOMX] = rho * u;
    s[MOMY] = rho * v;
    s[ETOT] = pr / gm + 0.5 * rho * (u * u + v * v);
    break;
  }
  case KFVM_IC_TAYLOR_GREEN: {
    const double mach = (double)0.1f; // user:mach 0.1 parsed through std::stof
    const double gMasq = g * mach * mach;
    const double u = sin(x) * cos(y) * cos(z), v = -cos(x) * sin(y) * cos(z), w = 0.0;
    const double q = (cos(2.0 * x) + cos(2.0 * y)) * (cos(2.0 * z) + 2.0);
    const double rho = 1.0 + gMasq * q / 16.0, pr = 1.0 / gMasq + q / 16.0;
    s[DENS] = rho;
    s[MOMX] = rho * u;
    s[MOMY] = rho * v;
    s[MOMZ] = rho * w;
    s[ETOT] = pr / gm + 0.5 * rho * (u * u + v * v + w * w);
    break;
  }
  case KFVM_IC_ORSZAG_TANG: {
    const double rho = g * g, pr = g;
    const double u = -sin(2.0 * pi * y), v = sin(2.0 * pi * x), w = 0.0;
    const double bx = -sin(2.0 * pi * y), by = sin(4.0 * pi * x), bz = 0.0;
    s[DENS] = rho;
    s[MOMX] = rho * u;
    s[MOMY] = rho * v;
    s[MOMZ] = rho * w;
    s[MAGX] = bx;
    s[MAGY] = by;
    s[MAGZ] = bz;
    s[ETOT] = pr / gm + rho * (u * u + v * v + w * w) / 2.0 + (bx * bx + by * by + bz * bz) / 2.0;
    break;
  }
  case KFVM_IC_SR_SHOCK_TUBE: {
    // exec/SRHydro/SRShockTube: at rest, rho, p = 10, 40/3 for |x| < 1/2, else 1, 1e-6
    const double gR = g / gm, ax = fabs(x);
    const double rho = ax < 0.5 ? 10.0 : 1.0, pr = ax < 0.5 ? 40.0 / 3.0 : 1.e-6;
    const double h = 1.0 + pr * gR / rho;
    s[DENS] = rho;
    s[ETOT] = rho * h - pr;
    break;
  }
  case KFVM_IC_SR_RIEMANN_2D: {
    // exec/SRHydro/SRRiem2d: four quadrants, two of them moving at 0.99 c
    const double gR = g / gm, v0 = 0.99;
    double rho = 0.5, vx = 0.0, vy = 0.0, pr = 1.0;
    if (x > 0.0) {
      rho = 0.1;
      if (y > 0.0) pr = 0.01;
      else vy = v0;
    } else if (y > 0.0) {
      rho = 0.1;
      vx = v0;
    }
    const double W = 1.0 / sqrt(1.0 - vx * vx - vy * vy), h = 1.0 + pr * gR / rho;
    s[DENS] = rho * W;
    s[MOMX] = rho * W * W * h * vx;
    s[MOMY] = rho * W * W * h * vy;
    s[ETOT] = rho * W * W * h - pr;
    break;
  }
  case KFVM_IC_STIR_TURB: {
    // exec/{Hydro,NavierStokes,MHD}/StirTurb: at rest with unit sound speed; GLM-MHD
    // adds a uniform bx of plasma beta 0.1 (user:beta, read through std::stof)
    const double pr = 1.0 / g;
    s[DENS] = 1.0;
    s[ETOT] = pr / gm;
    if (p.eq == KFVM_EQ_MHD_GLM) {
      const double bx = sqrt(2.0 * pr / (double)0.1f);
      s[ETOT] += 0.5 * bx * bx;
      s[MAGX] = bx;
    }
    break;
  }
  default: { // KFVM_IC_SMOOTH_WAVE: periodic smooth flow on the box
    const double X = 2.0 * pi * (x - p.xlo) / (p.xup - p.xlo);
    const double Y = 2.0 * pi * (y - p.ylo) / (p.yup - p.ylo);
    const double Z = p.dim == 3 ? 2.0 * pi * (z - p.zlo) / (p.zup - p.zlo) : 0.0;
    const double rho = 1.0 + 0.2 * sin(X) * cos(Y) * cos(Z);
    const double u = 0.5 + 0.1 * sin(Y), v = 0.3 * cos(X), w = 0.1 * sin(X + Y);
    const double pr = 1.0 + 0.1 * cos(X - Y + Z);
    if (p.eq == KFVM_EQ_SRHYDRO) {
      // the same primitives as a special-relativistic state
      const double W = 1.0 / sqrt(1.0 - (u * u + v * v + w * w)), h = 1.0 + pr * g / (gm * rho);
      s[DENS] = rho * W;
      s[MOMX] = rho * W * W * h * u;
      s[MOMY] = rho * W * W * h * v;
      s[MOMZ] = rho * W * W * h * w;
      s[ETOT] = rho * W * W * h - pr;
      break;
    }
    s[DENS] = rho;
    s[MOMX] = rho * u;
    s[MOMY] = rho * v;
    s[MOMZ] = rho * w;
    s[ETOT] = pr / gm + 0.5 * rho * (u * u + v * v + w * w);
    if (p.eq == KFVM_EQ_MHD_GLM) {
      const double bx = 0.3 * sin(Y), by = 0.2 * cos(X), bz = 0.1, psi = 0.01 * sin(X);
      s[MAGX] = bx;
      s[MAGY] = by;
      s[MAGZ] = bz;
      s[PSI] = psi;
      s[ETOT] += 0.5 * (bx * bx + by * by + bz * bz) + 0.5 * psi * psi;
    }
    break;
  }
  }
}

template <int DIM, int NV>
__global__ void __launch_bounds__(128) ic_kernel(IcParams p, uint64_t seed, double *__restrict__ U,
                                                 Grid g) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t j = blockIdx.y * (int64_t)blockDim.y + threadIdx.y;
  const int64_t k = blockIdx.z;
  if (i >= g.nx || j >= g.ny) return;
  // Gauss-Legendre rule on (-1/2, 1/2) in the reference's point order
  // (src/numeric/Numeric.cpp:14-27), g.nq = 2 or 3 points per direction
  const int nq = g.nq;
  double ab[3], wt[3];
  if (nq == 3) {
    ab[0] = 0.0;
    ab[1] = -0.7745966692414833770358530 / 2.0;
    ab[2] = 0.7745966692414833770358530 / 2.0;
    wt[0] = 0.8888888888888888888888888 / 2.0;
    wt[1] = wt[2] = 0.5555555555555555555555555 / 2.0;
  } else {
    ab[0] = -0.577350269189625764509148 / 2.0;
    ab[1] = 0.577350269189625764509148 / 2.0;
    ab[2] = 0.0;
    wt[0] = wt[1] = 1.0 / 2.0;
    wt[2] = 0.0;
  }
  const double xc = g.dx * (double(i) + 0.5) + p.x0, yc = g.dy * (double(j) + 0.5) + p.y0;
  const double zc = g.dz * (double(k) + 0.5) + p.z0;
  double noise = 0.0;
  if (p.kind == KFVM_IC_KELVIN_HELMHOLTZ) {
    // the cell's index in the whole domain (this block's offset added)
    const uint64_t gi = (uint64_t)(((k + g.off[2]) * g.gn[1] + (j + g.off[1])) * g.gn[0] + (i + g.off[0]));
    const double u01 = (double)(splitmix64(seed ^ gi) >> 11) * (1.0 / 9007199254740992.0);
    noise = 1.0e-3 * (2.0 * u01 - 1.0);
  }
  double acc[NV];
#pragma unroll
  for (int v = 0; v < NV; v++) acc[v] = 0.0;
  const int nzq = DIM == 3 ? nq : 1;
  for (int a = 0; a < nq; a++)
    for (int b = 0; b < nq; b++)
      for (int e = 0; e < nzq; e++) {
        const double x = ab[a] * g.dx + xc, y = ab[b] * g.dy + yc;
        const double z = DIM == 3 ? ab[e] * g.dz + zc : p.zlo;
        double s[9];
        ic_point(p, x, y, z, noise, s);
#pragma unroll
        for (int v = 0; v < NV; v++) {
          if (DIM == 2) acc[v] += wt[a] * wt[b] * s[v];
          else acc[v] += wt[a] * wt[b] * wt[e] * s[v];
        }
      }
  const int64_t pp = pidx(g, i, j, k);
#pragma unroll
  for (int v = 0; v < NV; v++) U[v * g.pvol + pp] = acc[v];
}

cudaError_t launch_ic(int dim, int eq, int ic_kind, uint64_t seed, const kfvm_config &cfg,
                      double *U, const Grid &g, cudaStream_t s) {
  IcParams p{ic_kind, dim, eq, cfg.gamma, cfg.xlo, cfg.xup, cfg.ylo, cfg.yup, cfg.zlo, cfg.zup,
             cfg_lo(&cfg, 0), cfg_lo(&cfg, 1), cfg_lo(&cfg, 2)};
  const dim3 grid((unsigned)((g.nx + kBlockX - 1) / kBlockX), (unsigned)((g.ny + kBlockY - 1) / kBlockY),
                  (unsigned)g.nz);
  const dim3 blk(kBlockX, kBlockY);
  const bool glm = eq == KFVM_EQ_MHD_GLM;
  if (dim == 2 && !glm) ic_kernel<2, 5><<<grid, blk, 0, s>>>(p, seed, U, g);
  else if (dim == 3 && !glm) ic_kernel<3, 5><<<grid, blk, 0, s>>>(p, seed, U, g);
  else if (dim == 2) ic_kernel<2, 9><<<grid, blk, 0, s>>>(p, seed, U, g);
  else ic_kernel<3, 9><<<grid, blk, 0, s>>>(p, seed, U, g);
  return cudaGetLastError();
}

} // namespace kfvm
