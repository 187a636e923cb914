// physics.cuh -- device-side equation-of-state, flux and Riemann-solver
// functions for the Euler, Navier-Stokes and GLM-MHD systems, FP64.
//
// Restates (slug-cfd/kfvm-kokkos):
//   src/physics/hydro/Hydro_EOS.H:22-92          EOS<Hydro>
//   src/physics/navierstokes/NavierStokes_EOS.H   EOS<NavierStokes> (same algebra)
//   src/physics/mhd_glm/MHD_GLM_EOS.H:22-128      EOS<MHD_GLM>
//   src/physics/hydro/Hydro_Riemann.H:26-187      Euler flux, Batten/Roe speeds, HLLC
//   src/physics/mhd_glm/MHD_GLM_Riemann.H:25-99   GLM flux, Davis + Wu-Shu speeds
//   src/physics/Common_K.H:23-63                  HLL / LLF in Batten's form
//   src/physics/Riemann.H:15-45                   HLLC star-state helpers
//   src/physics/*/_K.H VarConvert                 linearised primitive variables
//   src/physics/srhydro/SRHydro_{EOS,Riemann}.H  special-relativistic EOS (sr_eos.h),
//                                                 flux and wave speeds (HLL / LLF)
// The arithmetic follows the reference expression by expression; nvcc may fuse
// multiply-adds, so results agree with the CPU oracle to rounding, not bitwise.
#pragma once

#include <cstdint>

#include "sr_eos.h"

namespace kfvm {

enum { DENS = 0, MOMX = 1, MOMY = 2, MOMZ = 3, ETOT = 4, MAGX = 5, MAGY = 6, MAGZ = 7, PSI = 8 };
enum { EQ_HYDRO = 0, EQ_NS = 1, EQ_GLM = 2, EQ_SR = 3 };
enum { RS_LLF = 0, RS_HLL = 1, RS_HLLC = 2 };

// bound on the relative error of Eos::weno_approx.  For |log2 rho| <= 20 and
// gamma <= 3 the exponent -gamma lg2(rho) is off by at most gamma x 2 ulp(20)
// = 1.2e-5 (lg2.approx) plus the FP32 roundings of gamma and of the product
// (<= 5.5e-6), i.e. <= 1.8e-5 x ln 2 = 1.2e-5 relative after ex2; ex2.approx
// (2^-22) and the FP32 roundings of p and rho add < 4e-7.
constexpr double kWenoApproxEps = 2e-5;
// Two face states whose components differ by at most kSameTol x their largest
// component are treated as one state by the Riemann kernel (Eos::same_state): every
// solver here is consistent, F(u, u) = F(u), and differs from F(u) by about
// (wave speed) x |uR - uL| for nearby states, so the flux changes by less than
// 1e-14 of its scale.  The reconstruction of a uniform region leaves such
// rounding-level differences between the two sides of a face.
constexpr double kSameTol = 1e-14;
// bound on the relative error of Eos::weno_round: one rounding to FP32 (2^-24)
// plus a few FP64 ulps of the pressure, the power and the quotient
constexpr double kWenoRoundEps = 6.0e-8;

// Reciprocal by Newton-Raphson refinement (Flynn 1970; Markstein 1990) of the
// hardware's approximate FP64 reciprocal (PTX rcp.approx.ftz.f64): each step
// e = 1 - y r, r = r + r e squares the relative error, and two steps bring the
// seed to within about one ulp of 1/y for normal y (tests compare it with the
// IEEE quotient).  It has no special-case branches: y = 0, infinite or subnormal
// gives NaN or infinity, which only states that are already unphysical reach.
__device__ __forceinline__ double rcp_nr(double y) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(y));
  double e = fma(-y, r, 1.0);
  r = fma(r, e, r);
  e = fma(-y, r, 1.0);
  return fma(r, e, r);
}

template <int EQ>
struct Eos {
  static constexpr int NV = EQ == EQ_GLM ? 9 : 5;
  // primitives: SR keeps the Lorentz factor after the pressure
  static constexpr int NVP = EQ == EQ_SR ? 6 : NV;

  // kinetic energy; gas at rest (all momenta exactly 0, common in undisturbed
  // regions) skips the division, whose zero-dividend case leaves the hardware's
  // fast path: the value is the same +0 the quotient gives for a positive density
  __device__ __forceinline__ static double ekin(const double *U) {
    const double m2 = 0.5 * (U[MOMX] * U[MOMX] + U[MOMY] * U[MOMY] + U[MOMZ] * U[MOMZ]);
    if (m2 == 0.0 && U[DENS] > 0.0) return 0.0;
    return m2 / U[DENS];
  }
  __device__ __forceinline__ static double prsb(const double *U) {
    return 0.5 * (U[MAGX] * U[MAGX] + U[MAGY] * U[MAGY] + U[MAGZ] * U[MAGZ]);
  }
  __device__ __forceinline__ static double eint(const double *U) {
    if constexpr (EQ == EQ_GLM) {
      return (U[ETOT] - prsb(U) - ekin(U) - 0.5 * U[PSI] * U[PSI]);
    } else {
      return (U[ETOT] - ekin(U));
    }
  }
  // Internal energy for a comparison with the bound b: the kinetic energy by the
  // Newton-refined reciprocal (within 2 ulp of the quotient), and the exact
  // expression wherever the approximate value lies within 2^-50 (|ke| + |eint|)
  // of b, so that eint > b is decided as the exact expression decides it.
  // Non-finite or non-positive densities fall through to the exact expression.
  __device__ __forceinline__ static double eint_vs(const double *U, double b) {
    const double m2 = 0.5 * (U[MOMX] * U[MOMX] + U[MOMY] * U[MOMY] + U[MOMZ] * U[MOMZ]);
    const double ke = m2 * rcp_nr(U[DENS]);
    double ei;
    if constexpr (EQ == EQ_GLM) ei = U[ETOT] - prsb(U) - ke - 0.5 * U[PSI] * U[PSI];
    else ei = U[ETOT] - ke;
    if (!(fabs(ei - b) > 8.9e-16 * (fabs(ke) + fabs(ei)) + 1e-300) || !(U[DENS] > 0.0)) ei = eint(U);
    return ei;
  }
  // internal energy with the reciprocal density given (one division shared by
  // the quantities of a state)
  __device__ __forceinline__ static double eint_r(const double *U, double ir) {
    const double ke = 0.5 * (U[MOMX] * U[MOMX] + U[MOMY] * U[MOMY] + U[MOMZ] * U[MOMZ]) * ir;
    if constexpr (EQ == EQ_GLM) {
      return (U[ETOT] - prsb(U) - ke - 0.5 * U[PSI] * U[PSI]);
    } else {
      return (U[ETOT] - ke);
    }
  }
  __device__ __forceinline__ static double pres(double g, const double *U) {
    return (g - 1.0) * eint(U);
  }
  __device__ __forceinline__ static double soundspeed(double g, const double *U) {
    return sqrt(g * pres(g, U) / U[DENS]);
  }
  // KXRCF indicator variable p / rho^gamma (SR: the density D, SRHydro_EOS.H:225-228)
  __device__ __forceinline__ static double weno(double g, const double *U) {
    if constexpr (EQ == EQ_SR) return U[DENS];
    else return pres(g, U) / pow(U[DENS], g);
  }
  // The same indicator with the power taken in FP32 by the hardware lg2 / ex2
  // approximations (the pressure stays FP64): relative error below
  // kWenoApproxEps for densities in [2^-20, 2^20] and 1 < gamma <= 3.  Outside
  // that range, or for a non-finite pressure, it returns NaN, which tells the
  // reader to recompute the exact value.
  __device__ __forceinline__ static float weno_approx(double g, const double *U) {
    return weno_approx_rp(g, U[DENS], pres(g, U));
  }
  // the same from density and pressure
  __device__ __forceinline__ static float weno_approx_rp(double g, double rho, double p) {
    if (!(rho >= 9.5367431640625e-07 && rho <= 1048576.0) || !(g <= 3.0) || !isfinite(p))
      return __int_as_float(0x7fc00000);
    float l2, r;
    asm("lg2.approx.f32 %0, %1;" : "=f"(l2) : "f"((float)rho));
    asm("ex2.approx.f32 %0, %1;" : "=f"(r) : "f"(-(float)g * l2));
    const float w = (float)p * r;
    // an FP32 underflow (or overflow) of the product voids the bound
    return fabsf(w) >= 1.17549435e-38f ? w : __int_as_float(0x7fc00000);
  }
  // The indicator computed in FP64 as the reference does and rounded once to FP32
  // (relative error below kWenoRoundEps), or NaN where FP32 cannot hold it
  __device__ __forceinline__ static float weno_round_rp(double g, double rho, double p) {
    const float w = __double2float_rn(p / pow(rho, g));
    return fabsf(w) >= 1.17549435e-38f && fabsf(w) <= 3.0e38f ? w : __int_as_float(0x7fc00000);
  }
  // the FP32 form the reconstruction stores: in 2D (8 face points per cell, where
  // the power is cheap next to the rest and fine grids put smooth cells' jumps
  // close to the threshold) the rounded FP64 value; in 3D (24 points) the
  // hardware approximation
  template <int DIM>
  __device__ __forceinline__ static float weno_store(double g, double rho, double p) {
    if constexpr (DIM == 2) return weno_round_rp(g, rho, p);
    else return weno_approx_rp(g, rho, p);
  }
  __device__ __forceinline__ static double positivity(const double *U) {
    if constexpr (EQ == EQ_SR) return sr::positivity(U);
    if constexpr (EQ == EQ_GLM) {
#pragma unroll
      for (int v = 0; v < NV; v++)
        if (isnan(U[v])) return -1.0;
    }
    return fmin(U[DENS], eint(U));
  }
  __device__ __forceinline__ static void cons2prim(double g, const double *U, double *V) {
    if constexpr (EQ == EQ_SR) {
      sr::cons2prim(g, U, V);
      return;
    }
    V[0] = U[DENS];
    V[1] = U[MOMX] / U[DENS];
    V[2] = U[MOMY] / U[DENS];
    V[3] = U[MOMZ] / U[DENS];
    V[4] = pres(g, U);
    if constexpr (EQ == EQ_GLM) {
      V[5] = U[MAGX];
      V[6] = U[MAGY];
      V[7] = U[MAGZ];
      V[8] = U[PSI];
    }
  }
  __device__ __forceinline__ static double fastMagSonic(double g, const double *U, double bl) {
    const double asq = g * pres(g, U) / U[DENS];
    const double bsq = 2.0 * prsb(U) / U[DENS];
    const double blsq = bl * bl / U[DENS];
    const double absq = asq + bsq;
    return sqrt(0.5 * (absq + sqrt(absq * absq - 4.0 * asq * blsq)));
  }

  // physical flux in direction ord[0]
  __device__ __forceinline__ static void flux(double ch, const int *vo, const int *bo,
                                              const double *U, const double *V, double *F) {
    if constexpr (EQ == EQ_SR) {
      // SRHydro_Riemann.H:24-37
      (void)ch;
      (void)bo;
      F[DENS] = U[DENS] * V[vo[0]];
      F[vo[0]] = U[vo[0]] * V[vo[0]] + V[4];
      F[vo[1]] = U[vo[1]] * V[vo[0]];
      F[vo[2]] = U[vo[2]] * V[vo[0]];
      F[ETOT] = U[vo[0]];
    } else if constexpr (EQ != EQ_GLM) {
      (void)ch;
      (void)bo;
      F[DENS] = U[vo[0]];
      F[vo[0]] = U[vo[0]] * V[vo[0]] + V[4];
      F[vo[1]] = U[vo[0]] * V[vo[1]];
      F[vo[2]] = U[vo[0]] * V[vo[2]];
      F[ETOT] = V[vo[0]] * (U[ETOT] + V[4]);
    } else {
      const double mx = U[vo[0]];
      const double vx = V[vo[0]], vy = V[vo[1]], vz = V[vo[2]];
      const double bx = U[bo[0]], by = U[bo[1]], bz = U[bo[2]];
      const double et = U[ETOT], pg = V[4];
      const double chpsi = ch * U[PSI], hpsisq = 0.5 * U[PSI] * U[PSI];
      const double uDb = vx * bx + vy * by + vz * bz, bsq = bx * bx + by * by + bz * bz;
      const double pt = pg + 0.5 * bsq;
      F[DENS] = mx;
      F[vo[0]] = mx * vx + pt - bx * bx;
      F[vo[1]] = mx * vy - bx * by;
      F[vo[2]] = mx * vz - bx * bz;
      F[ETOT] = vx * (et + pt - hpsisq) + bx * (chpsi - uDb);
      F[bo[0]] = chpsi;
      F[bo[1]] = vx * by - vy * bx;
      F[bo[2]] = vx * bz - vz * bx;
      F[PSI] = ch * bx;
    }
  }

  __device__ __forceinline__ static double roeAvg(double rL, double rR, double qL, double qR) {
    return (qL * sqrt(rL) + qR * sqrt(rR)) / (sqrt(rL) + sqrt(rR));
  }

  // GLM-MHD wave-speed estimates (Davis with the cleaning speed, and the Wu-Shu
  // bound; MHD_GLM_Riemann.H:25-99)
  __device__ __forceinline__ static double speeds(double g, double ch, const int *vo,
                                                  const int *bo, const double *uL,
                                                  const double *uR, const double *vL,
                                                  const double *vR, double &sL, double &sR) {
    const double cfL = fastMagSonic(g, uL, uL[bo[0]]);
    const double cfR = fastMagSonic(g, uR, uR[bo[0]]);
    const double sdL = fmin(vL[vo[0]] - fmax(ch, cfL), vR[vo[0]] - fmax(ch, cfR));
    const double sdR = fmax(vL[vo[0]] + fmax(ch, cfL), vR[vo[0]] + fmax(ch, cfR));
    const double rtL = sqrt(uL[DENS]), rtR = sqrt(uR[DENS]);
    const double rtSum = rtL + rtR, vSum = (rtL * vL[vo[0]] + rtR * vR[vo[0]]) / rtSum;
    const double b0 = uL[bo[0]] - uR[bo[0]], b1 = uL[bo[1]] - uR[bo[1]],
                 b2 = uL[bo[2]] - uR[bo[2]];
    const double bnDiff = sqrt(b0 * b0 + b1 * b1 + b2 * b2) / rtSum;
    const double aL = fmin(vL[vo[0]], vSum) - cfL - bnDiff;
    const double aR = fmin(vR[vo[0]], vSum) + cfR + bnDiff;
    sL = fmin(sdL, aL);
    sR = fmax(sdR, aR);
    return fmax(fabs(sL), fabs(sR));
  }

  // Euler / Navier-Stokes primitives with the density reciprocal taken once
  // (the reference divides by rho at every use; the values differ by rounding only)
  __device__ __forceinline__ static void cons2prim_r(double g, const double *U, double ir, double *V) {
    V[0] = U[DENS];
    V[1] = U[MOMX] * ir;
    V[2] = U[MOMY] * ir;
    V[3] = U[MOMZ] * ir;
    V[4] = (g - 1.0) * (U[ETOT] - 0.5 * (U[MOMX] * U[MOMX] + U[MOMY] * U[MOMY] + U[MOMZ] * U[MOMZ]) * ir);
  }

  // uL, uR equal to kSameTol (false when either holds a NaN)
  __device__ __forceinline__ static bool same_state(const double *uL, const double *uR) {
    double s = 0.0;
#pragma unroll
    for (int v = 0; v < NV; v++) s = fmax(s, fabs(uL[v]));
    bool same = true;
#pragma unroll
    for (int v = 0; v < NV; v++) same = same && fabs(uR[v] - uL[v]) <= kSameTol * s;
    return same;
  }

  // Face with equal states (kSameTol): the physical flux, and the speed bound
  // max(|sL|, |sR|) that the estimates give for equal states.  Euler / Navier-Stokes:
  // |u_n| + a (Hydro_Riemann.H:41-81 with uTil = u, aTil = a); SRHydro: the larger
  // magnitude of the state's two characteristic bounds (SRHydro_Riemann.H:39-77),
  // with one pressure recovery instead of two; GLM-MHD: |u_n| + max(ch, cf), what
  // the Davis and Wu-Shu bounds (MHD_GLM_Riemann.H:55-99) give with no jump in B
  __device__ __forceinline__ static double solve_same(double g, double ch, int dir, const double *u, double *F) {
    const int ord[3] = {dir, (dir + 1) % 3, (dir + 2) % 3};
    const int vo[3] = {MOMX + ord[0], MOMX + ord[1], MOMX + ord[2]};
    const int bo[3] = {MAGX + ord[0], MAGX + ord[1], MAGX + ord[2]};
    if constexpr (EQ == EQ_GLM) {
      double V[NV];
      cons2prim(g, u, V);
      flux(ch, vo, bo, u, V, F);
      return fabs(V[vo[0]]) + fmax(ch, fastMagSonic(g, u, u[bo[0]]));
    }
    if constexpr (EQ == EQ_SR) {
      double V[NVP];
      sr::cons2prim(g, u, V);
      flux(0.0, vo, bo, u, V, F);
      const double a = sr::soundspeed(g, V), asq = a * a;
      const double w = V[5], sig = asq / (w * w * (1.0 - asq));
      const double rt = sqrt(sig * (1.0 + sig - V[vo[0]] * V[vo[0]]));
      const double sm = (V[vo[0]] - rt) / (1.0 + sig), sp = (V[vo[0]] + rt) / (1.0 + sig);
      return fmax(fabs(sm), fabs(sp));
    }
    const double ir = 1.0 / u[DENS];
    double V[NV];
    cons2prim_r(g, u, ir, V);
    flux(0.0, vo, bo, u, V, F);
    return fabs(V[vo[0]]) + sqrt(g * V[4] * ir);
  }

  // Riemann solve at one face point in direction dir; returns max(|sL|,|sR|).
  // Euler / Navier-Stokes: Batten/Roe speed estimates (Hydro_Riemann.H:26-80) and,
  // for HLLC, the low-Mach / shear-corrected star fluxes (Hydro_Riemann.H:82-187),
  // with each repeated divisor (rho, the Roe weight sum, sL - sS, sR - sS, psL - psR)
  // inverted once by rcp_nr, the Roe weights from one root of rR / rL and the Mach
  // estimate from one root: 7 reciprocals and 6 roots where the literal form
  // divides about 30 times.
  __device__ __forceinline__ static double solve(int rs, double g, double ch, int dir,
                                                 const double *uL, const double *uR,
                                                 double *F) {
    const int ord[3] = {dir, (dir + 1) % 3, (dir + 2) % 3};
    const int vo[3] = {MOMX + ord[0], MOMX + ord[1], MOMX + ord[2]};
    const int bo[3] = {MAGX + ord[0], MAGX + ord[1], MAGX + ord[2]};
    double vL[NVP], vR[NVP];
    double sL, sR, sMax;
    if constexpr (EQ == EQ_SR) {
      // SRHydro_Riemann.H:39-77: bounds of the relativistic characteristic speeds
      sr::cons2prim(g, uL, vL);
      sr::cons2prim(g, uR, vR);
      const double aL = sr::soundspeed(g, vL), aLsq = aL * aL;
      const double aR = sr::soundspeed(g, vR), aRsq = aR * aR;
      const double wL = vL[5], sigL = aLsq / (wL * wL * (1.0 - aLsq));
      const double sqrtL = sqrt(sigL * (1.0 + sigL - vL[vo[0]] * vL[vo[0]]));
      const double wR = vR[5], sigR = aRsq / (wR * wR * (1.0 - aRsq));
      const double sqrtR = sqrt(sigR * (1.0 + sigR - vR[vo[0]] * vR[vo[0]]));
      const double sLm = (vL[vo[0]] - sqrtL) / (1.0 + sigL), sRm = (vR[vo[0]] - sqrtR) / (1.0 + sigR);
      const double sLp = (vL[vo[0]] + sqrtL) / (1.0 + sigL), sRp = (vR[vo[0]] + sqrtR) / (1.0 + sigR);
      sL = fmin(sLm, sRm);
      sR = fmax(sLp, sRp);
      sMax = fmax(fabs(sL), fabs(sR));
    } else if constexpr (EQ != EQ_GLM) {
      const double rL = uL[DENS], rR = uR[DENS];
      const double iLR = rcp_nr(rL * rR), iL = rR * iLR, iR = rL * iLR;
      cons2prim_r(g, uL, iL, vL);
      cons2prim_r(g, uR, iR, vR);
      const double pL = vL[4], pR = vR[4];
      const double a2L = g * pL * iL, a2R = g * pR * iR;
      const double aL = sqrt(a2L), aR = sqrt(a2R);

      const double hL = (uL[ETOT] + pL) * iL, hR = (uR[ETOT] + pR) * iR;
      // Roe weights sqrt(rL) / (sqrt(rL) + sqrt(rR)) = 1 / (1 + sqrt(rR / rL)) and
      // sqrt(rR) / (...) = sqrt(rR / rL) / (1 + sqrt(rR / rL)): one root, one reciprocal
      const double tq = sqrt(rR * iL), wL = rcp_nr(1.0 + tq), wR = tq * wL;
      const double uTil = vL[vo[0]] * wL + vR[vo[0]] * wR, vTil = vL[vo[1]] * wL + vR[vo[1]] * wR,
                   wTil = vL[vo[2]] * wL + vR[vo[2]] * wR, hTil = hL * wL + hR * wR;
      const double vsqTil = uTil * uTil + vTil * vTil + wTil * wTil;
      const double aTil = sqrt((g - 1.0) * (hTil - 0.5 * vsqTil));
      sL = fmin(vL[vo[0]] - aL, uTil - aTil);
      sR = fmax(vR[vo[0]] + aR, uTil + aTil);
      sMax = fmax(fabs(sL), fabs(sR));
      if (rs == RS_HLLC) {
        const double vsqL = vL[1] * vL[1] + vL[2] * vL[2] + vL[3] * vL[3];
        const double vsqR = vR[1] * vR[1] + vR[2] * vR[2] + vR[3] * vR[3];
        // max of the two Mach numbers max(|v|^2 / a^2) = max(vsqL a2R, vsqR a2L) / (a2L a2R):
        // one root and one reciprocal of aL aR
        double M = sqrt(fmax(vsqL * a2R, vsqR * a2L)) * rcp_nr(aL * aR);
        const double uLn = vL[vo[0]], uRn = vR[vo[0]];
        const double psL = rL * (sL - uLn), psR = rR * (sR - uRn);
        // sS and psR psL / (psR - psL) share the reciprocal of psL - psR
        const double iD = rcp_nr(psL - psR);
        const double sS = ((pR - pL) + (psL * uLn - psR * uRn)) * iD;
        const double pS = 0.5 * ((pL + pR) + psL * (sS - uLn) + psR * (sS - uRn));
        const double dLR = rcp_nr((sL - sS) * (sR - sS)), dL = (sR - sS) * dLR, dR = (sL - sS) * dLR;
        const double sFacL = sS * dL, sFacR = sS * dR;
        const double uJump = uRn - uLn, vJump = vR[vo[1]] - vL[vo[1]], wJump = vR[vo[2]] - vL[vo[2]];
        const double psiFac = -(psR * psL) * iD;
        const double presRat = fmin(1.0, fmin(pL, pR) * rcp_nr(fmax(pL, pR)));
        // presRat^M (pressure ratio in (0, 1]) as exp(M log presRat); exactly 0 for equal pressures
        const double gFac = pL == pR ? 0.0 : 1.0 - exp(M * log(presRat));
        const double shFacL = psiFac * gFac * sL * dL, shFacR = psiFac * gFac * sR * dR;
        M = fmin(M, 1.0);
        const double omm = 1.0 - M * M;
        const double fM = M * sqrt(4.0 + omm * omm) * rcp_nr(1.0 + M * M);
        const double pFacL = psiFac * (fM - 1.0) * uJump + sL * pS * dL;
        const double pFacR = psiFac * (fM - 1.0) * uJump + sR * pS * dR;
        if (0 <= sL) {
          flux(ch, vo, bo, uL, vL, F);
        } else if (0 <= sS) {
          flux(ch, vo, bo, uL, vL, F);
          F[DENS] = sFacL * (sL * uL[DENS] - F[DENS]);
          F[vo[0]] = sFacL * (sL * uL[vo[0]] - F[vo[0]]) + pFacL;
          F[vo[1]] = sFacL * (sL * uL[vo[1]] - F[vo[1]]) + shFacL * vJump;
          F[vo[2]] = sFacL * (sL * uL[vo[2]] - F[vo[2]]) + shFacL * wJump;
          F[ETOT] = sFacL * (sL * uL[ETOT] - F[ETOT]) + sS * pFacL;
        } else if (0 < sR) {
          flux(ch, vo, bo, uR, vR, F);
          F[DENS] = sFacR * (sR * uR[DENS] - F[DENS]);
          F[vo[0]] = sFacR * (sR * uR[vo[0]] - F[vo[0]]) + pFacR;
          F[vo[1]] = sFacR * (sR * uR[vo[1]] - F[vo[1]]) + shFacR * vJump;
          F[vo[2]] = sFacR * (sR * uR[vo[2]] - F[vo[2]]) + shFacR * wJump;
          F[ETOT] = sFacR * (sR * uR[ETOT] - F[ETOT]) + sS * pFacR;
        } else {
          flux(ch, vo, bo, uR, vR, F);
        }
        return sMax;
      }
    } else {
      cons2prim(g, uL, vL);
      cons2prim(g, uR, vR);
      sMax = speeds(g, ch, vo, bo, uL, uR, vL, vR, sL, sR);
    }
    if (rs == RS_LLF) {
      sL = -sMax;
      sR = sMax;
    }
    const double iS = rcp_nr(sR - sL);
    const double tR = (fmin(0.0, sR) - fmin(0.0, sL)) * iS, tL = 1.0 - tR;
    const double tD = 0.5 * (sR * fabs(sL) - sL * fabs(sR)) * iS;
    double FR[NV];
    flux(ch, vo, bo, uL, vL, F);
    flux(ch, vo, bo, uR, vR, FR);
#pragma unroll
    for (int v = 0; v < NV; v++) F[v] = tL * F[v] + tR * FR[v] - tD * (uR[v] - uL[v]);
    return sMax;
  }
};

// Linearisation of the conserved variables about a reference state
template <int EQ>
struct VarConv {
  double gamm, rho, irho, u, v, w, bx, by, bz, rPsi, vsq;
  __device__ __forceinline__ VarConv(const double *ref, double gam) {
    if constexpr (EQ == EQ_SR) {
      // SRHydro_K.H:22-56: the momenta over D, linearised about (D, S) of the cell;
      // (rho, u, v, w) hold (D, Sx, Sy, Sz)
      gamm = gam - 1.0;
      rho = ref[DENS];
      irho = 1.0 / rho;
      u = ref[MOMX];
      v = ref[MOMY];
      w = ref[MOMZ];
      bx = by = bz = rPsi = vsq = 0.0;
      return;
    }
    gamm = gam - 1.0;
    rho = ref[DENS];
    irho = 1.0 / rho;
    u = ref[MOMX] / rho;
    v = ref[MOMY] / rho;
    w = ref[MOMZ] / rho;
    if constexpr (EQ == EQ_GLM) {
      bx = ref[MAGX];
      by = ref[MAGY];
      bz = ref[MAGZ];
      rPsi = ref[PSI];
      vsq = (u * u + v * v + w * w) / 2.0;
    } else {
      bx = by = bz = rPsi = 0.0;
      vsq = 0.5 * (u * u + v * v + w * w);
    }
  }
  __device__ __forceinline__ void cons2LinPrim(double *s) const {
    if constexpr (EQ == EQ_SR) {
      s[MOMX] = s[MOMX] / rho - s[DENS] * u / (rho * rho);
      s[MOMY] = s[MOMY] / rho - s[DENS] * v / (rho * rho);
      s[MOMZ] = s[MOMZ] / rho - s[DENS] * w / (rho * rho);
      return;
    }
    if constexpr (EQ == EQ_GLM) {
      s[ETOT] = gamm * (vsq * s[DENS] + s[ETOT] - u * s[MOMX] - v * s[MOMY] - w * s[MOMZ] -
                        bx * s[MAGX] - by * s[MAGY] - bz * s[MAGZ] - rPsi * s[PSI]);
    } else {
      s[ETOT] = gamm * (vsq * s[DENS] - u * s[MOMX] - v * s[MOMY] - w * s[MOMZ] + s[ETOT]);
    }
    s[MOMX] = (s[MOMX] - u * s[DENS]) / rho;
    s[MOMY] = (s[MOMY] - v * s[DENS]) / rho;
    s[MOMZ] = (s[MOMZ] - w * s[DENS]) / rho;
  }
  // component c of cons2LinPrim(s), the momenta scaled by the reciprocal density
  __device__ __forceinline__ double lin1(const double *s, int c) const {
    if constexpr (EQ == EQ_SR) {
      if (c == MOMX) return s[MOMX] / rho - s[DENS] * u / (rho * rho);
      if (c == MOMY) return s[MOMY] / rho - s[DENS] * v / (rho * rho);
      if (c == MOMZ) return s[MOMZ] / rho - s[DENS] * w / (rho * rho);
      return s[c];
    }
    if (c == DENS) return s[DENS];
    if (c == MOMX) return (s[MOMX] - u * s[DENS]) * irho;
    if (c == MOMY) return (s[MOMY] - v * s[DENS]) * irho;
    if (c == MOMZ) return (s[MOMZ] - w * s[DENS]) * irho;
    if (c == ETOT) {
      if constexpr (EQ == EQ_GLM) {
        return gamm * (vsq * s[DENS] + s[ETOT] - u * s[MOMX] - v * s[MOMY] - w * s[MOMZ] - bx * s[MAGX] -
                       by * s[MAGY] - bz * s[MAGZ] - rPsi * s[PSI]);
      } else {
        return gamm * (vsq * s[DENS] - u * s[MOMX] - v * s[MOMY] - w * s[MOMZ] + s[ETOT]);
      }
    }
    return s[c];
  }
  __device__ __forceinline__ void linPrim2Cons(double *s) const {
    if constexpr (EQ == EQ_SR) {
      s[MOMX] = s[DENS] * u / rho + rho * s[MOMX];
      s[MOMY] = s[DENS] * v / rho + rho * s[MOMY];
      s[MOMZ] = s[DENS] * w / rho + rho * s[MOMZ];
      return;
    }
    if constexpr (EQ == EQ_GLM) {
      s[ETOT] = (vsq * s[DENS] + rho * u * s[MOMX] + rho * v * s[MOMY] + rho * w * s[MOMZ] +
                 bx * s[MAGX] + by * s[MAGY] + bz * s[MAGZ] + s[ETOT] / gamm + rPsi * s[PSI]);
    } else {
      s[ETOT] = (vsq * s[DENS] + rho * u * s[MOMX] + rho * v * s[MOMY] + rho * w * s[MOMZ] +
                 s[ETOT] / gamm);
    }
    s[MOMX] = (rho * s[MOMX] + u * s[DENS]);
    s[MOMY] = (rho * s[MOMY] + v * s[DENS]);
    s[MOMZ] = (rho * s[MOMZ] + w * s[DENS]);
  }
};

} // namespace kfvm
