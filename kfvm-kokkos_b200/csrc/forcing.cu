// forcing.cu -- random forcing of the stirred-turbulence problems: the mode table on
// the host (EosParameters' constructor and updateForcing, src/ParameterStructs.H:45-73,
// src/ParameterStructs.cpp:41-88 of slug-cfd/kfvm-kokkos) and, on the device, the
// two domain integrals that fix the strength and the kick itself
// (RandForcingIntegrate_K / RandForcingApply_K, src/physics/Common_K.H:645-784).
//
// Mode n has wavevector k = (k1, k2, k3) and per direction d a complex amplitude
// a_d = (re, im); at x the mode gives g_d = re cos(2 pi k.x) - im sin(2 pi k.x), and
// the kick is the Helmholtz mix f = sum_n [r g + (1 - 2r) k (k.g) / |k|^2] with r the
// compressive-to-solenoidal ratio, summed mode by mode in the reference's order.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <random>

#include "../../include/kfvm_b200.h"
#include "kernels.cuh"
#include "launch.h"

namespace kfvm {

constexpr int kForceBlock = 256;
constexpr int kForceKMax = 3; // MAX_FORCING_MODE (src/Types.H:105)

// wavevectors of the forcing band in the reference's loop order; returns the count
static int forcing_wavevectors(int dim, double *modes) {
  const int kMax = kForceKMax, kMaxSq = kMax * kMax, kMaxZ = dim == 2 ? 0 : kMax;
  int nm = 0;
  for (int i = 0; i <= kMax; i++)
    for (int j = -kMax; j <= kMax; j++)
      for (int k = -kMaxZ; k <= kMaxZ; k++) {
        const int ksq = i * i + j * j + k * k;
        if (ksq == 0 || ksq > kMaxSq) continue;    // outside the band
        if (i == 0 && (j < 0 || k < 0)) continue;  // one of each +-k pair on the i = 0 plane
        if (modes) {
          const int kv[3] = {i, j, k};
          for (int d = 0; d < dim; d++) {
            double *m = modes + ((size_t)nm * dim + d) * 3;
            m[0] = (double)kv[d];
            m[1] = m[2] = 0.0;
          }
        }
        nm++;
      }
  return nm;
}

int forcing_num_modes(int dim) { return (dim == 2 || dim == 3) ? forcing_wavevectors(dim, nullptr) : -1; }

void forcing_draw(int dim, uint32_t seed32, double *modes) {
  const int nm = forcing_wavevectors(dim, modes);
  std::mt19937 gen{seed32};
  std::normal_distribution<double> sn{0.0, 1.0};
  for (int n = 0; n < nm; n++) {
    const double *kv = modes + (size_t)n * dim * 3;
    const double k1 = kv[0], k2 = kv[3], k3 = dim == 3 ? kv[6] : 0.0;
    const double kMag = std::sqrt(k1 * k1 + k2 * k2 + k3 * k3);
    const double sig = std::sqrt(kMag * (4.0 - kMag));
    for (int d = 0; d < dim; d++) {
      double *m = modes + ((size_t)n * dim + d) * 3;
      m[1] = sig * sn(gen); // real
      m[2] = sig * sn(gen); // imaginary
    }
  }
}

struct ForceArgs {
  const double *modes; // [n][DIM][3] on the device
  int nm;
  double ratio, str;
  double xlo, ylo, zlo;
};

// kick direction at (x, y, z); with str != 1 each mode's contribution is scaled
// as the reference's apply kernel scales it
template <int DIM, bool SCALED>
__device__ __forceinline__ void force_at(const ForceArgs &a, double x, double y, double z, double &fu,
                                         double &fv, double &fw) {
  constexpr double kTwoPi = 2.0 * 3.14159265358979323846;
  const double fr = a.ratio, mfr = 1.0 - 2.0 * fr;
  fu = fv = fw = 0.0;
  for (int n = 0; n < a.nm; n++) {
    const double *m = a.modes + n * DIM * 3;
    const double k1 = m[0], k2 = m[3], k3 = DIM == 3 ? m[6] : 0.0;
    const double kdx = k1 * x + k2 * y + k3 * (DIM == 3 ? z : 0.0);
    double sn, cs;
    sincos(kTwoPi * kdx, &sn, &cs);
    const double fun = m[1] * cs - m[2] * sn;
    const double fvn = m[4] * cs - m[5] * sn;
    const double fwn = DIM == 3 ? m[7] * cs - m[8] * sn : 0.0;
    const double ksq = k1 * k1 + k2 * k2 + k3 * k3, iksq = 1.0 / ksq;
    const double du = (fr + mfr * iksq * k1 * k1) * fun + mfr * iksq * (k1 * k2 * fvn + k1 * k3 * fwn);
    const double dv = (fr + mfr * iksq * k2 * k2) * fvn + mfr * iksq * (k1 * k2 * fun + k2 * k3 * fwn);
    const double dw = (fr + mfr * iksq * k3 * k3) * fwn + mfr * iksq * (k1 * k3 * fun + k2 * k3 * fvn);
    if (SCALED) {
      fu += a.str * du;
      fv += a.str * dv;
      fw += a.str * dw;
    } else {
      fu += du;
      fv += dv;
      fw += dw;
    }
  }
}

__device__ __forceinline__ void cell_of(const Grid &g, int64_t c, int64_t &i, int64_t &j, int64_t &k) {
  i = c % g.nx;
  j = (c / g.nx) % g.ny;
  k = c / (g.nx * g.ny);
}

// intA = sum rho |f|^2 / 2, intB = sum m . f over the interior; one partial pair per block
template <int DIM>
__global__ void __launch_bounds__(kForceBlock)
    forcing_integrate_kernel(const double *__restrict__ U, Grid g, ForceArgs a, double *__restrict__ part) {
  const int64_t c = blockIdx.x * (int64_t)kForceBlock + threadIdx.x;
  double ia = 0.0, ib = 0.0;
  if (c < g.n) {
    int64_t i, j, k;
    cell_of(g, c, i, j, k);
    const double x = g.dx * ((double)i + 0.5) + a.xlo, y = g.dy * ((double)j + 0.5) + a.ylo;
    const double z = g.dz * ((double)k + 0.5) + a.zlo;
    double fu, fv, fw;
    force_at<DIM, false>(a, x, y, z, fu, fv, fw);
    const double *Uc = U + pidx(g, i, j, k);
    const double rho = Uc[DENS * g.pvol];
    ia = 0.5 * rho * (fu * fu + fv * fv + fw * fw);
    ib = Uc[MOMX * g.pvol] * fu + Uc[MOMY * g.pvol] * fv + Uc[MOMZ * g.pvol] * fw;
  }
  __shared__ double sa[kForceBlock], sb[kForceBlock];
  sa[threadIdx.x] = ia;
  sb[threadIdx.x] = ib;
  __syncthreads();
  for (int h = kForceBlock / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) {
      sa[threadIdx.x] += sa[threadIdx.x + h];
      sb[threadIdx.x] += sb[threadIdx.x + h];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = sa[0];
    part[2 * blockIdx.x + 1] = sb[0];
  }
}

// fixed-order sum of the block partials (one block)
__global__ void __launch_bounds__(1024) forcing_sum_kernel(const double *__restrict__ part, int64_t nblk,
                                                           double *__restrict__ out) {
  __shared__ double sa[1024], sb[1024];
  double a = 0.0, b = 0.0;
  for (int64_t t = threadIdx.x; t < nblk; t += 1024) {
    a += part[2 * t];
    b += part[2 * t + 1];
  }
  sa[threadIdx.x] = a;
  sb[threadIdx.x] = b;
  __syncthreads();
  for (int h = 512; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) {
      sa[threadIdx.x] += sa[threadIdx.x + h];
      sb[threadIdx.x] += sb[threadIdx.x + h];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = sa[0];
    out[1] = sb[0];
  }
}

// momenta += rho f, total energy += rho |f|^2 / 2 + m . f (f at strength str)
template <int DIM>
__global__ void __launch_bounds__(kForceBlock) forcing_apply_kernel(double *__restrict__ U, Grid g, ForceArgs a) {
  const int64_t c = blockIdx.x * (int64_t)kForceBlock + threadIdx.x;
  if (c >= g.n) return;
  int64_t i, j, k;
  cell_of(g, c, i, j, k);
  const double x = g.dx * ((double)i + 0.5) + a.xlo, y = g.dy * ((double)j + 0.5) + a.ylo;
  const double z = g.dz * ((double)k + 0.5) + a.zlo;
  double fu, fv, fw;
  force_at<DIM, true>(a, x, y, z, fu, fv, fw);
  double *Uc = U + pidx(g, i, j, k);
  const double rho = Uc[DENS * g.pvol];
  double ePert = 0.5 * rho * (fu * fu + fv * fv + fw * fw);
  ePert += Uc[MOMX * g.pvol] * fu + Uc[MOMY * g.pvol] * fv + Uc[MOMZ * g.pvol] * fw;
  Uc[MOMX * g.pvol] += rho * fu;
  Uc[MOMY * g.pvol] += rho * fv;
  Uc[MOMZ * g.pvol] += rho * fw;
  Uc[ETOT * g.pvol] += ePert;
}

int64_t forcing_blocks(const Grid &g) { return (g.n + kForceBlock - 1) / kForceBlock; }

cudaError_t launch_forcing_integrate(int dim, const double *U, const Grid &g, const double *modes, int nm,
                                     double ratio, const double lo[3], double *part, double *sums,
                                     cudaStream_t s) {
  const ForceArgs a{modes, nm, ratio, 1.0, lo[0], lo[1], lo[2]};
  const int64_t nblk = forcing_blocks(g);
  if (dim == 2) forcing_integrate_kernel<2><<<(unsigned)nblk, kForceBlock, 0, s>>>(U, g, a, part);
  else forcing_integrate_kernel<3><<<(unsigned)nblk, kForceBlock, 0, s>>>(U, g, a, part);
  forcing_sum_kernel<<<1, 1024, 0, s>>>(part, nblk, sums);
  return cudaGetLastError();
}

cudaError_t launch_forcing_apply(int dim, double *U, const Grid &g, const double *modes, int nm, double ratio,
                                 double str, const double lo[3], cudaStream_t s) {
  const ForceArgs a{modes, nm, ratio, str, lo[0], lo[1], lo[2]};
  const int64_t nblk = forcing_blocks(g);
  if (dim == 2) forcing_apply_kernel<2><<<(unsigned)nblk, kForceBlock, 0, s>>>(U, g, a);
  else forcing_apply_kernel<3><<<(unsigned)nblk, kForceBlock, 0, s>>>(U, g, a);
  return cudaGetLastError();
}

} // namespace kfvm
