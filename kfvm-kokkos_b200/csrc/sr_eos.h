// sr_eos.h -- equation of state of special-relativistic hydrodynamics, usable
// from device code (physics.cuh) and from the host (plotfile.cpp's auxiliary
// variables).  Conserved variables U = (D, Sx, Sy, Sz, E) with D = rho W,
// S = rho h W^2 v, E = rho h W^2 - p, ideal gas h = 1 + gamma p / ((gamma - 1) rho).
//
// Restates src/physics/srhydro/SRHydro_EOS.H:30-260 (slug-cfd/kfvm-kokkos): the
// pressure is recovered by Newton iteration on the quartic of algorithm 2.1 of
// arXiv:2305.14805, switching to the better conditioned psi(p) iteration of its
// algorithm 2.3 when D^2 / (E^2 - S^2) < 1e-4 or the Lorentz factor of an iterate
// drops below 1.01; the initial guess is its eqs (2.21) / (2.16).  Both iterations
// stop at a relative step below 1e-9 or after 200 iterations.
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define KFVM_SR_HD __host__ __device__ __forceinline__
#else
#define KFVM_SR_HD inline
#endif

namespace kfvm {
namespace sr {

constexpr int kMaxIter = 200;
constexpr double kRtol = 1.e-9;

KFVM_SR_HD double ssq(const double *U) { return U[1] * U[1] + U[2] * U[2] + U[3] * U[3]; }

// Lorentz factor of the state at pressure p: S / (E + p) is the velocity
KFVM_SR_HD double lorenz(double p, const double *U) {
  const double DhW = U[4] + p;
  return 1.0 / sqrt(1.0 - ssq(U) / (DhW * DhW));
}

KFVM_SR_HD double pres_guess(double gam, const double *U) {
  const double ESsq = U[4] * U[4] - ssq(U);
  if (U[0] >= ESsq / U[4]) return 0.0;
  const double gm2E = (gam - 2.0) * U[4], gm = gam - 1.0;
  return (gm2E + sqrt(gm2E * gm2E - 4.0 * gm * (U[0] * sqrt(ESsq) - ESsq))) / 2.0;
}

KFVM_SR_HD double pres_stable(double gam, const double *U, double p) {
  const double gm = gam - 1.0, gm2 = gam - 2.0, D = U[0], E = U[4], Ssq = ssq(U);
  for (int n = 0; n < kMaxIter; n++) {
    const double EP = E + p, rt = sqrt(EP * EP - Ssq);
    const double psi = Ssq + EP * (p / gm - E) + D * rt;
    const double dpsi = (2.0 * p - gm2 * E) / gm + D * EP / rt;
    const double dp = -psi / dpsi;
    if (fabs(dp) / p < kRtol) break;
    p += dp;
  }
  return p;
}

KFVM_SR_HD double pres(double gam, const double *U) {
  double p = pres_guess(gam, U);
  const double Dsq = U[0] * U[0], Esq = U[4] * U[4], Ssq = ssq(U), ESsq = Esq - Ssq;
  if (Dsq / ESsq < 1.e-4) return pres_stable(gam, U, p);
  const double gm = gam - 1.0, gm2 = gam - 2.0;
  const double c0 = -ESsq * (Dsq - ESsq) * gm * gm;
  const double c1 = 2.0 * U[4] * (gm2 * ESsq * gm - Dsq * gm * gm);
  const double c2 = Esq * (gam * gam - 6.0 * gm) + 2.0 * Ssq * gm - Dsq * gm * gm;
  const double c3 = -2.0 * U[4] * gm2;
  for (int n = 0; n < kMaxIter; n++) {
    if (lorenz(p, U) < 1.0 + 0.01) return pres_stable(gam, U, p);
    const double phi = c0 + p * (c1 + p * (c2 + p * (c3 + p)));
    const double dphi = c1 + p * (2.0 * c2 + p * (3.0 * c3 + p));
    const double dp = -phi / dphi;
    if (fabs(dp) / p < kRtol) break;
    p += dp;
  }
  return p;
}

// primitives V = (rho, vx, vy, vz, p, W): the pressure at V[4] as for the other
// systems, the Lorentz factor after it
KFVM_SR_HD void cons2prim(double gam, const double *U, double *V) {
  const double p = pres(gam, U);
  const double W = lorenz(p, U);
  const double rho = U[0] / W;
  const double h = 1.0 + gam * (p / ((gam - 1.0) * rho));
  const double m = rho * W * W * h;
  V[0] = rho;
  V[1] = U[1] / m;
  V[2] = U[2] / m;
  V[3] = U[3] / m;
  V[4] = p;
  V[5] = W;
}

KFVM_SR_HD double soundspeed(double gam, const double *V) {
  const double h = 1.0 + gam * V[4] / ((gam - 1.0) * V[0]);
  return sqrt(gam * V[4] / (V[0] * h));
}

// E - sqrt(D^2 + S^2), which the limiter keeps above its neighbourhood minimum
// (SRHydro_K.H:440-450)
KFVM_SR_HD double ediff(const double *U) { return U[4] - sqrt(U[0] * U[0] + ssq(U)); }

// admissibility: D > 0 and E^2 > D^2 + S^2 (positive pressure, |v| < 1)
KFVM_SR_HD double positivity(const double *U) {
  const double etotDiff = U[4] * U[4] - (U[0] * U[0] + ssq(U));
  return U[0] < etotDiff ? U[0] : etotDiff;
}

} // namespace sr
} // namespace kfvm
