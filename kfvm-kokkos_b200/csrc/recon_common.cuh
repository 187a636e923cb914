// recon_common.cuh -- pieces shared by the FP64 and the tensor-core (3xTF32)
// linear reconstruction kernels: the weight-row layout, the face-slot addressing
// of the face arrays and the positivity limiter's per-block footprint tile.
#pragma once

#include "kernels.cuh"

namespace kfvm {

// ---------------------------------------------------------------------------
// Rows of the linear reconstruction: face points f*NQF+q, then (GLM sources)
// the interior points; the full-stencil weights are [cell][row] on the host
// and reach the kernels as MMA operand tables.
template <int DIM, int EQ, int NQ = 2>
struct LinRows {
  using T = Cfg<DIM, EQ, NQ>;
  static constexpr int NROWS = T::NF * T::NQF + (T::SRC ? T::NQC : 0);
  static constexpr int SIZE = T::C * NROWS;
};

// face-slot address of point q, variable v of face f of cell (i,j,k) in a
// [slot][q][v][face] array with nvv variables
__device__ __forceinline__ int64_t face_slot_addr(const Grid &g, int f, int64_t i, int64_t j, int64_t k,
                                                  int q, int v, int nqf, int nvv) {
  const int d = f >> 1, hi = f & 1;
  const int64_t fi = i + (d == 0 && hi), fj = j + (d == 1 && hi), fk = k + (d == 2 && hi);
  const int64_t fidx = (fk * g.fdim[d][1] + fj) * g.fdim[d][0] + fi;
  const int slot = hi ? 0 : 1;
  return ((int64_t)(slot * nqf + q) * nvv + v) * g.nface[d] + fidx;
}

// Per-block footprint (block cells plus a one-cell ring) of the cell quantities the
// limiter's bounds read from the 3^d neighbourhood: rho, eint, sound speed and the
// three velocities.  Each is computed once per cell instead of once per neighbour.
template <int DIM>
struct PosTile {
  static constexpr int TX = kBlockX + 2, TY = kBlockY + 2, TZ = DIM == 3 ? 3 : 1;
  static constexpr int N = TX * TY * TZ;
};

// the footprint quantities of a cell state st into entry t of sm
template <int EQ, int NT>
__device__ __forceinline__ void pos_quantities(const double (&st)[Eos<EQ>::NV], const Grid &g, double (*sm)[NT],
                                               int t) {
  using E = Eos<EQ>;
  if constexpr (EQ == EQ_SR) {
    // density and E - sqrt(D^2 + S^2); SR bounds need nothing else
    sm[0][t] = st[DENS];
    sm[1][t] = sr::ediff(st);
    return;
  }
  const double ir = 1.0 / st[DENS];
  const double ei = E::eint_r(st, ir);
  sm[0][t] = st[DENS];
  sm[1][t] = ei;
  sm[2][t] = sqrt(g.gamma * ((g.gamma - 1.0) * ei) * ir);
  // velocities as the reference's divergence estimate takes them (m / rho,
  // Common_K.H:363-378)
  sm[3][t] = st[MOMX] / st[DENS];
  sm[4][t] = st[MOMY] / st[DENS];
  sm[5][t] = st[MOMZ] / st[DENS];
}

// the footprint quantities of padded cell (gi, gj, gk) into entry t of sm
template <int EQ, int NT>
__device__ __forceinline__ void pos_cell(const double *__restrict__ U, const Grid &g, int64_t gi, int64_t gj,
                                         int64_t gk, double (*sm)[NT], int t) {
  using E = Eos<EQ>;
  const double *Uc = U + pidx(g, gi, gj, gk);
  double st[E::NV];
#pragma unroll
  for (int v = 0; v < E::NV; v++) st[v] = Uc[v * g.pvol];
  pos_quantities<EQ>(st, g, sm, t);
}

template <int DIM, int EQ>
__device__ __forceinline__ void pos_tile_fill(const double *__restrict__ U, const Grid &g, int64_t i0,
                                              int64_t j0, int64_t k, double (*sm)[PosTile<DIM>::N]) {
  using P = PosTile<DIM>;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  for (int t = tid; t < P::N; t += blockDim.x * blockDim.y) {
    const int a = t % P::TX, b = (t / P::TX) % P::TY, cz = t / (P::TX * P::TY);
    const int64_t gi = i0 - 1 + a, gj = j0 - 1 + b, gk = k - (DIM == 3 ? 1 : 0) + cz;
    if (gi > g.nx || gj > g.ny) continue; // beyond the ring of any live cell
    pos_cell<EQ>(U, g, gi, gj, gk, sm, t);
  }
}

// PositivityPreserve_K bounds (Common_K.H:331-380; SR: SRHydro_K.H:224-246, no
// flattening) from the footprint tile
// (at(xo, yo, zo) gives the entry of the neighbour at that offset)
template <int DIM, int EQ, int NT, class At>
__device__ __forceinline__ PosBounds pos_bounds_at(const double (*sm)[NT], At at) {
  double maxDens = -1.7976931348623157e308, minDens = 1.7976931348623157e308;
  double minEint = 1.7976931348623157e308, minSdSp = 1.7976931348623157e308;
  constexpr int zr = DIM == 3 ? 1 : 0;
  if constexpr (EQ == EQ_SR) {
#pragma unroll
    for (int xo = -1; xo <= 1; xo++)
#pragma unroll
      for (int yo = -1; yo <= 1; yo++)
#pragma unroll
        for (int zo = -zr; zo <= zr; zo++) {
          const int t = at(xo, yo, zo);
          maxDens = fmax(maxDens, sm[0][t]);
          minDens = fmin(minDens, sm[0][t]);
          minEint = fmin(minEint, sm[1][t]);
        }
    return PosBounds{sm[0][at(0, 0, 0)], minDens, maxDens, minEint};
  } else {
#pragma unroll
  for (int xo = -1; xo <= 1; xo++)
#pragma unroll
    for (int yo = -1; yo <= 1; yo++)
#pragma unroll
      for (int zo = -zr; zo <= zr; zo++) {
        const int t = at(xo, yo, zo);
        maxDens = fmax(maxDens, sm[0][t]);
        minDens = fmin(minDens, sm[0][t]);
        minEint = fmin(minEint, sm[1][t]);
        minSdSp = fmin(minSdSp, sm[2][t]);
      }
  const double dxU = sm[3][at(1, 0, 0)] - sm[3][at(-1, 0, 0)];
  const double dyV = sm[4][at(0, 1, 0)] - sm[4][at(0, -1, 0)];
  const double dzW = sm[5][at(0, 0, zr)] - sm[5][at(0, 0, -zr)];
  const double divV = (dxU + dyV + dzW) / 2.0;
  double kappa = 0.2;
  const double eta = fmin(1.0, fmax(0.0, -(kappa * minSdSp + divV) / (kappa * minSdSp)));
  kappa *= (1.0 - eta);
  PosBounds b;
  b.rDens = sm[0][at(0, 0, 0)];
  b.maxDens = maxDens * (1.0 + kappa);
  b.minDens = minDens * (1.0 - kappa);
  b.minEint = minEint * (1.0 - kappa);
  return b;
  }
}

template <int DIM, int EQ>
__device__ __forceinline__ PosBounds pos_bounds_tile(const double (*sm)[PosTile<DIM>::N], int tx, int ty) {
  using P = PosTile<DIM>;
  constexpr int zr = DIM == 3 ? 1 : 0;
  return pos_bounds_at<DIM, EQ>(sm, [&](int xo, int yo, int zo) {
    return ((zr + zo) * P::TY + (ty + 1 + yo)) * P::TX + (tx + 1 + xo);
  });
}

} // namespace kfvm
