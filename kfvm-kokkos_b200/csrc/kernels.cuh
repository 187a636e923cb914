// kernels.cuh -- sm_100a kernels of one RHS evaluation + RK stage update.
//
// One stage is these launches on the solver's stream:
//   bc_fill      periodic / outflow halo of the stage state   (Solver::setCellBCs)
//   recon        linear face states of every cell written to the face arrays, the
//                KXRCF indicator at each own face point and whether every state lies
//                inside the positivity bounds (KernelLinearRecon_K); FP64 FMAs, or
//                the 3xTF32 tcgen05 contraction of recon_tc.cu
//   flag         KXRCF flags from the indicators               (WenoSelect_K)
//   compact      the flag-set semantics of WenoSelector::update, theta = 1 for
//                in-bounds linear cells, the compacted list of heavy cells
//   heavy        WENO-AO and/or the full positivity limiter on the listed cells
//                (KernelWenoRecon_K, PositivityPreserve_K)
//   riemann<d>   one thread per face point: HLLC/HLL/LLF, quadrature weighted flux
//                sum per face, max wave speed                 (RiemannSolver*_K)
//   stage        flux divergence (+ viscous terms, + GLM sources), fused with the
//                low-storage FSAL register update and the error estimate
//                (IntegrateRHS_K, Viscosity_K, SourceTerms_K, RKFSAL_*_K)
// Reference: slug-cfd/kfvm-kokkos src/Solver.cpp:188-530 and the functors named above.
//
// Layouts in HBM (all FP64):
//   U      [v][nz+2r][ny+2r][nx+2r]   padded SoA, r = 2 (2D: one z plane, no z halo)
//   faces  [slot][q][v][face]         per direction, face = (k*fy + j)*fx + i
//   flux   [v][face]                  quadrature-weighted flux per face
//   K, Uhat, Utmp [v][cell]           interior SoA, cell = (k*ny + j)*nx + i
#pragma once

#include <cstdint>

#include "../../include/kfvm_b200.h"
#include "physics.cuh"

namespace kfvm {

constexpr int kRad = 2;
constexpr int kBlockX = 32, kBlockY = 4;

// geometry and pointers of one solver, passed by value
struct Grid {
  int64_t nx, ny, nz, n;     // interior cells (nz = 1 in 2D)
  int64_t px, py, pvol;      // padded pitch in x, rows per plane, values per variable
  int64_t rz;                // z halo (0 in 2D)
  int64_t fdim[3][3];        // face grid extents per direction
  int64_t nface[3];
  double dx, dy, dz;
  double rdx, rdy, rdz;      // 1 / dx, 1 / dy, 1 / dz
  int nq;                    // Gauss points per direction
  int bc[6];
  // variables whose sign the wall mirror flips, bit v per face (reflecting and
  // no-slip coefficient tables of <Eq>_BCCoeffs.H; 0 for periodic / outflow)
  unsigned bflip[6];
  double gamma, ch_init;
  int rs;
  int64_t loff[KFVM_MAX_CELLS]; // stencil offsets in the padded array
  int64_t off[3], gn[3];        // this block's first cell and the domain's cells per axis
};

// a boundary face whose outer face state is held in the face array itself (received
// from the neighbouring block, or written by a user boundary condition) instead of
// being derived from the inner state on read
__host__ __device__ inline bool outer_in_face(int bc) { return bc == KFVM_BC_EXCHANGE || bc == KFVM_BC_USER; }

// stencil on the device: weights plus linear offsets in the padded array, and the
// full-stencil linear weights packed as [cell][row] (rows: face points f*NQF+q, then
// interior points q) for the light reconstruction pass
constexpr int kMaxLinRows = 6 * 9 + 27; // 3D, 3 Gauss points: 6 faces x 9 points (+ 27 interior, GLM-MHD)
// The same weights for the tensor-core form: W = hi + lo, both TF32 values in FP32
// containers, stored as the tcgen05 B operand (K-major, no swizzle): K = stencil
// cells padded to 40, N = rows padded to 32, [cell/4][row][cell%4].
constexpr int kTcMaxK = 40, kTcMaxN = 32;
// And as B fragments of the FP64 MMA m8n8k4 (4 stencil cells x 8 rows per
// fragment, one double per lane): [k step][8-row tile][lane], lane -> (cell
// 4 ks + lane % 4, row 8 nt + lane / 4), zero beyond the stencil or the rows.
constexpr int kDmmaMaxB = 8 * 7 * 32; // 8 K-steps x 7 row tiles (54 rows)
struct DevStencil {
  kfvm_stencil w;
  int64_t loff[KFVM_MAX_CELLS];
  double lin[KFVM_MAX_CELLS * kMaxLinRows];
  alignas(16) float tcw[2][kTcMaxK * kTcMaxN];
  alignas(16) double dmma_b[kDmmaMaxB];
};

// device-side scalars written by reductions
struct DevScalars {
  unsigned long long maxvel_bits; // max wave speed of the current step attempt
  unsigned long long glm_lam_bits, glm_vel_bits;
  unsigned int nflag;             // KXRCF flags of the current evaluation
  unsigned int napplied;          // cells reconstructed with WENO
  unsigned int nheavy;            // cells in the heavy (WENO / limiter) list
  unsigned int fault;              // a bounded wait in a kernel gave up (sticky)
  double err, posmin;             // error estimate outputs (finalize kernel)
  // learned indicator's judge, cumulative: judged cells, of them labelled
  // troubled, troubled but not predicted (missed), predicted but not troubled
  unsigned long long mlp_judged, mlp_pos, mlp_missed, mlp_false;
  // Riemann faces with equal states in the sampled blocks of the equal-state
  // variant, and the faces sampled, cumulative
  unsigned long long nsame, nsamp;
};

// heavy-list entries carry the cell index in the low 29 bits (grids of at most 2^29
// cells: 180 GB holds about 1.4e8 cells of the 3D path's arrays)
constexpr uint32_t kHeavyCellMax = 0x1fffffffu;

// variations below this fraction of a cell's density / pressure count as smooth for
// the learned indicator (labels and the normalisation of its features)
constexpr double kMlpFloor = 1e-4;

// the learned indicator's judge: a hashed fraction of the cells runs full WENO
// and has its label compared with the network's prediction
struct JudgeArgs {
  double frac;           // 0: no judge
  uint64_t seed;         // changes every evaluation
  double tau;            // label threshold on the WENO weight departure
  const uint8_t *pred;   // the network's per-cell prediction
};

enum ReconMode { RECON_LINEAR = 0, RECON_SPARSE = 1, RECON_FULL = 2 };
enum StageMode { STAGE_EVAL = 0, STAGE_UPDATE = 1, STAGE_FSAL = 2 };

struct StageCoef {
  double delta, g1, g2, g3, betaDt, bhatDt;
  int use_tmp; // delta or g2 nonzero somewhere in the scheme
};

__device__ __forceinline__ int64_t pidx(const Grid &g, int64_t i, int64_t j, int64_t k) {
  return ((k + g.rz) * g.py + (j + kRad)) * g.px + (i + kRad);
}

__device__ __forceinline__ void atomic_max_pos(unsigned long long *a, double v) {
  // non-negative doubles order like their bit patterns; NaN is ignored as in the
  // reference's "vq > maxVel ? vq : maxVel".  The maximum only grows during a
  // launch, so a value not above a plain read of it cannot raise it: skipping
  // those spares the same-address atomics that serialise in L2 (one per warp over
  // millions of warps doubled the Riemann kernel's time once the wave speeds
  // varied from warp to warp).
  if (v >= 0.0) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    if (b > *(volatile const unsigned long long *)a) atomicMax(a, b);
  }
}

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  // splitmix64 finaliser
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

// uniform in [0, 1) from two keys
__device__ __forceinline__ double unit_hash(uint64_t a, uint64_t b) {
  return (double)(mix64(a ^ mix64(b)) >> 11) * (1.0 / 9007199254740992.0);
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// NQ_: Gauss points per direction (NUM_QUAD_PTS of the reference's Definitions.H)
template <int DIM, int EQ, int NQ_ = 2>
struct Cfg {
  static constexpr int NV = Eos<EQ>::NV;
  static constexpr int NQ = NQ_;
  static constexpr int NQF = DIM == 2 ? NQ_ : NQ_ * NQ_;
  static constexpr int NQC = DIM == 2 ? NQ_ * NQ_ : NQ_ * NQ_ * NQ_;
  static constexpr int NF = 2 * DIM;
  static constexpr int C = DIM == 2 ? 13 : 33;
  static constexpr int CC = DIM == 2 ? 5 : 7;
  static constexpr int CB = DIM == 2 ? 5 : 11;
  static constexpr int NSUB = DIM == 2 ? 6 : 8;
  static constexpr int NB = DIM == 2 ? 4 : 6;
  static constexpr int NI = DIM == 2 ? 5 : 19;
  static constexpr bool SRC = EQ == EQ_GLM;
};

// Gauss-Legendre weights on (-1/2,1/2) in the reference's point order
// (src/numeric/Numeric.cpp:14-27: 2 points (1/2, 1/2); 3 points, centre first)
template <int NQ>
__device__ __forceinline__ double gl_wt(int q) {
  if constexpr (NQ == 3) return q == 0 ? 0.8888888888888888888888888 / 2.0 : 0.5555555555555555555555555 / 2.0;
  else return 1.0 / 2.0;
}

// Label of the learned troubled-cell indicator: the largest departure of the
// normalised WENO-JS weights (createOmegas, Stencil_K.H:556-580, before the
// adaptive-order transform) from the linear weights gamma_s, over the substencils
// and over density and pressure (linearised primitives 0 and 4) where their
// variation over the stencil exceeds kMlpFloor = 1e-4 of the cell value (below
// that the weights of noise-level variations are arbitrary, and the linear
// reconstruction of such variations is harmless).  The
// smoothness indicators are those of heavy_var_kernel (findSmoothness, 506-554).
template <int DIM, int EQ>
__device__ double weno_departure(const double *__restrict__ Uc, const Grid &g,
                                 const DevStencil *__restrict__ S) {
  using T = Cfg<DIM, EQ>;
  constexpr int NV = T::NV;
  const kfvm_stencil &st = S->w;
  double ref[NV];
#pragma unroll
  for (int v = 0; v < NV; v++) ref[v] = Uc[v * g.pvol];
  VarConv<EQ> vc(ref, g.gamma);
  double lin[NV];
#pragma unroll
  for (int v = 0; v < NV; v++) lin[v] = ref[v];
  vc.cons2LinPrim(lin);
  double Vf[T::C][2];
  for (int c = 0; c < T::C; c++) {
    const int64_t o = S->loff[c];
    double u[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) u[v] = Uc[v * g.pvol + o];
    vc.cons2LinPrim(u);
    Vf[c][0] = u[DENS];
    Vf[c][1] = u[ETOT];
  }
  double om[T::NSUB][2];
  for (int s = 0; s < T::NSUB; s++) {
    const int n = s == 0 ? T::C : (s == 1 ? T::CC : T::CB);
    om[s][0] = om[s][1] = 0.0;
    for (int i = 0; i < T::NI; i++) {
      double b0 = 0.0, b1 = 0.0;
      for (int q = 0; q < n; q++) {
        const int c = s < 2 ? q : (int)st.sub_idx[s - 2][q];
        const double w = st.deriv_w[s][i][q];
        b0 += w * Vf[c][0];
        b1 += w * Vf[c][1];
      }
      om[s][0] += b0 * b0;
      om[s][1] += b1 * b1;
    }
  }
  constexpr double gHi = 0.7, gLo = 0.7;
  double gam[T::NSUB];
  gam[0] = gHi;
  gam[1] = (1.0 - gHi) * gLo;
#pragma unroll
  for (int s = 2; s < T::NSUB; s++) gam[s] = (1.0 - gHi) * (1.0 - gLo) / (DIM == 2 ? 4.0 : 6.0);
  double dep = 0.0;
#pragma unroll
  for (int a = 0; a < 2; a++) {
    const double r = a == 0 ? lin[DENS] : lin[ETOT];
    if (!(sqrt(om[0][a]) > kMlpFloor * fabs(r))) continue;
    double tot = 0.0;
#pragma unroll
    for (int s = 0; s < T::NSUB; s++) {
      om[s][a] = gam[s] / (om[s][a] * om[s][a] + 1.e-40);
      tot += om[s][a];
    }
#pragma unroll
    for (int s = 0; s < T::NSUB; s++) dep = fmax(dep, fabs(om[s][a] / tot - gam[s]));
  }
  return dep;
}

// limiter bounds of a cell; minEint holds the bound on E - sqrt(D^2 + S^2) for SR
struct PosBounds {
  double rDens, minDens, maxDens, minEint;
};

template <int DIM, int EQ>
__device__ __forceinline__ PosBounds pos_bounds(const double *__restrict__ Uc, const Grid &g) {
  using E = Eos<EQ>;
  constexpr int NV = Eos<EQ>::NV;
  const double gm = g.gamma;
  double maxDens = -1.7976931348623157e308, minDens = 1.7976931348623157e308;
  double minEint = 1.7976931348623157e308, minSdSp = 1.7976931348623157e308;
  constexpr int zr = DIM == 3 ? 1 : 0;
  const int64_t sy = g.px, sz = g.px * g.py;
  if constexpr (EQ == EQ_SR) {
    // PositivityPreserve_K<SRHydro> (SRHydro_K.H:224-246): no flattening
#pragma unroll
    for (int xo = -1; xo <= 1; xo++)
#pragma unroll
      for (int yo = -1; yo <= 1; yo++)
#pragma unroll
        for (int zo = -zr; zo <= zr; zo++) {
          double s[NV];
          const int64_t o = xo + yo * sy + zo * sz;
#pragma unroll
          for (int v = 0; v < NV; v++) s[v] = Uc[v * g.pvol + o];
          maxDens = fmax(maxDens, s[DENS]);
          minDens = fmin(minDens, s[DENS]);
          minEint = fmin(minEint, sr::ediff(s));
        }
    return PosBounds{Uc[DENS * g.pvol], minDens, maxDens, minEint};
  } else {
#pragma unroll
  for (int xo = -1; xo <= 1; xo++)
#pragma unroll
    for (int yo = -1; yo <= 1; yo++)
#pragma unroll
      for (int zo = -zr; zo <= zr; zo++) {
        double s[NV];
        const int64_t o = xo + yo * sy + zo * sz;
#pragma unroll
        for (int v = 0; v < NV; v++) s[v] = Uc[v * g.pvol + o];
        const double ir = 1.0 / s[DENS];
        const double ei = E::eint_r(s, ir);
        maxDens = fmax(maxDens, s[DENS]);
        minDens = fmin(minDens, s[DENS]);
        minEint = fmin(minEint, ei);
        minSdSp = fmin(minSdSp, sqrt(gm * ((gm - 1.0) * ei) * ir));
      }
  auto U = [&](int64_t o, int v) { return Uc[v * g.pvol + o]; };
  const double dxU = U(1, MOMX) / U(1, DENS) - U(-1, MOMX) / U(-1, DENS);
  const double dyV = U(sy, MOMY) / U(sy, DENS) - U(-sy, MOMY) / U(-sy, DENS);
  const double dzW = DIM == 3 ? U(sz, MOMZ) / U(sz, DENS) - U(-sz, MOMZ) / U(-sz, DENS) : 0.0;
  const double divV = (dxU + dyV + dzW) / 2.0;
  double kappa = 0.2;
  const double eta = fmin(1.0, fmax(0.0, -(kappa * minSdSp + divV) / (kappa * minSdSp)));
  kappa *= (1.0 - eta);
  PosBounds b;
  b.rDens = Uc[DENS * g.pvol];
  b.maxDens = maxDens * (1.0 + kappa);
  b.minDens = minDens * (1.0 - kappa);
  b.minEint = minEint * (1.0 - kappa);
  return b;
  }
}

// true when a state leaves theta at 1 in both passes of the limiter
// (SR: the comparisons are strict the other way, SRHydro_K.H:256-257, 372)
template <int EQ>
__device__ __forceinline__ bool pos_inside(const PosBounds &b, const double *s) {
  const double rho = s[DENS];
  if constexpr (EQ == EQ_SR) return rho >= b.minDens && rho <= b.maxDens && sr::ediff(s) >= b.minEint;
  else return rho > b.minDens && rho < b.maxDens && Eos<EQ>::eint(s) > b.minEint;
}

} // namespace kfvm
