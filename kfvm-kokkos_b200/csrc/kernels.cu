// kernels.cu -- kernel bodies and host launchers of the per-stage hot path.
// See kernels.cuh for the stage structure and the HBM layouts.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <type_traits>

#include "kernels.cuh"
#include "launch.h"
#include "recon_common.cuh"
#include "tma.cuh"

namespace kfvm {

// ---------------------------------------------------------------------------
// halo fill: every halo cell copies the interior cell given by per-axis maps
// (periodic wrap or outflow mirror).  Applying the axis maps independently is
// the same as the reference's sequential x, y, z fills with their corner ranges
// (Solver.cpp:744-783, 826-930; BoundaryConditions_K.H:53-72).
__device__ __forceinline__ int64_t axis_map(int64_t i, int64_t n, int bcLo, int bcHi) {
  if (i < 0) return bcLo == KFVM_BC_PERIODIC ? i + n : -i - 1;
  if (i >= n) return bcHi == KFVM_BC_PERIODIC ? i - n : 2 * n - i - 1;
  return i;
}

template <int DIM, int NV>
__global__ void __launch_bounds__(256) bc_fill_kernel(double *__restrict__ U, Grid g) {
  const int64_t r = kRad;
  const int64_t hx = g.nx + 2 * r, hy = g.ny + 2 * r;
  const int64_t nxs = 2 * r * g.ny * g.nz;                 // x slabs (interior y,z)
  const int64_t nys = hx * 2 * r * g.nz;                   // y slabs (all x, interior z)
  const int64_t nzs = DIM == 3 ? hx * hy * 2 * r : 0;      // z slabs (all x, y)
  const int64_t total = nxs + nys + nzs;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t i, j, k;
    if (t < nxs) {
      const int64_t a = t % (2 * r), b = t / (2 * r);
      i = a < r ? a - r : g.nx + (a - r);
      j = b % g.ny;
      k = b / g.ny;
    } else if (t < nxs + nys) {
      const int64_t u = t - nxs, a = u % hx, b = u / hx;
      i = a - r;
      const int64_t jj = b % (2 * r);
      j = jj < r ? jj - r : g.ny + (jj - r);
      k = b / (2 * r);
    } else {
      const int64_t u = t - nxs - nys, a = u % hx, b = u / hx;
      i = a - r;
      j = b % hy - r;
      const int64_t kk = b / hy;
      k = kk < r ? kk - r : g.nz + (kk - r);
    }
    const int64_t si = axis_map(i, g.nx, g.bc[0], g.bc[1]);
    const int64_t sj = axis_map(j, g.ny, g.bc[2], g.bc[3]);
    const int64_t sk = DIM == 3 ? axis_map(k, g.nz, g.bc[4], g.bc[5]) : k;
    const int64_t dst = pidx(g, i, j, k), src = pidx(g, si, sj, sk);
    // wall mirrors flip signs; the sequential x, y, z fills of the reference
    // multiply a corner by the coefficients of every wall it lies beyond
    unsigned flip = (i < 0 ? g.bflip[0] : (i >= g.nx ? g.bflip[1] : 0u)) ^
                    (j < 0 ? g.bflip[2] : (j >= g.ny ? g.bflip[3] : 0u));
    if (DIM == 3) flip ^= k < 0 ? g.bflip[4] : (k >= g.nz ? g.bflip[5] : 0u);
#pragma unroll
    for (int v = 0; v < NV; v++) {
      const double x = U[v * g.pvol + src];
      U[v * g.pvol + dst] = (flip >> v) & 1u ? -x : x;
    }
  }
}

// ---------------------------------------------------------------------------
// Stage front end, four kernels:
//   recon    linear face states of every cell (FP64 MMA) written to the face
//            arrays, the KXRCF indicator p/rho^gamma (FP32 approximation) at each
//            own face point written to W, and whether every state lies strictly
//            inside the positivity limiter's bounds (then theta = 1 exactly as in
//            the reference)
//   flag     KXRCF flags from W, exact near the threshold (WenoSelect_K)
//   compact  the reference's flag-set semantics, theta = 1 for in-bounds linear
//            cells, and the compacted heavy list (WENO cells, cells to limit)
//   heavy    WENO-AO and/or the full limiter on the listed cells
// theta of the previous evaluation feeds the flags, so it is rewritten only after
// flag_kernel has read it.
constexpr uint32_t kHeavyWeno = 0x80000000u;      // WENO-AO is computed for the cell
constexpr uint32_t kHeavyJudge = 0x40000000u;     // a judged cell of the learned indicator
constexpr uint32_t kHeavyJudgeOnly = 0x20000000u; // judged but outside the WENO set: it keeps
                                                  // its linear states unless the judge's label
                                                  // says troubled (the cell-level fallback)
constexpr uint32_t kHeavyCell = kHeavyCellMax;

// Linear reconstruction of every cell on the FP64 tensor cores (mma.sync m8n8k4,
// the FP64 MMA of sm_100a; tcgen05 has no FP64 kind).  Per warp: one row of 32 cells
// of the block, in 4 groups of 8 cells.  For one group and variable v,
//   D[cell][row] = sum_k A[cell][k] B[k][row],  A = U(cell + offset k), B = weights,
// K runs over the stencil in steps of 4, N over the weight rows in tiles of 8;
// each DMMA does 256 FMAs where the scalar form issues 8 DFMAs.  The sum over
// stencil cells keeps its order in steps of four.  Lane l holds
// D[cell l/4][rows 2(l%4), 2(l%4)+1] of every N tile, i.e. the full state (all
// variables) of 2 NT face / interior points of its cell, and finishes them in FP64:
// positivity pre-check, indicator, stores.  The four lanes of a cell combine their
// in-bounds tests and GLM speed maxima by shuffles.
// The stencil has 4m + 1 cells (13 in 2D, 33 in 3D): the first 4m go through the
// MMAs in m K-steps and the last one is added in the epilogue by one FMA per row
// and variable, which spares a K-step that would be three quarters padding.
template <int DIM, int EQ, int NQ = 2>
struct DmmaShape {
  static constexpr int NR = LinRows<DIM, EQ, NQ>::NROWS;
  static constexpr int NT = (NR + 7) / 8;
  static constexpr int NK = (Cfg<DIM, EQ, NQ>::C - 1) / 4;
  static constexpr int BSIZE = NK * NT * 32;
  static_assert((Cfg<DIM, EQ, NQ>::C - 1) % 4 == 0, "stencil of 4m + 1 cells");
  // more than 7 row tiles (81 rows) go to recon_rows_kernel, not to the DMMA kernels
  static_assert(BSIZE <= kDmmaMaxB || NT > 7, "B fragment table too small");
};

__device__ __forceinline__ void dmma_884(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// One group of 8 cells of a row, the DMMA contraction: lane l ends with rows
// 8t + 2(l%4) + e of cell l/4 of the group in acc[v][t][e].  loadA(v, kc) gives
// variable v of stencil cell kc (kc < 4 NK) of this lane's cell and loadLast(v)
// that of the last stencil cell.
template <int DIM, int EQ, int NQ, class LoadA, class LoadLast>
__device__ __forceinline__ void recon_group_mma(int lane, const double *__restrict__ sB,
                                                const double *__restrict__ sWl, LoadA loadA, LoadLast loadLast,
                                                double (&acc)[Cfg<DIM, EQ, NQ>::NV][DmmaShape<DIM, EQ, NQ>::NT][2]) {
  using T = Cfg<DIM, EQ, NQ>;
  using Sh = DmmaShape<DIM, EQ, NQ>;
  constexpr int NV = T::NV, NT = Sh::NT, NK = Sh::NK;
#pragma unroll
  for (int v = 0; v < NV; v++)
#pragma unroll
    for (int t = 0; t < NT; t++) acc[v][t][0] = acc[v][t][1] = 0.0;
  // the whole K loop unrolled where the accumulators are few (Euler / NS with two
  // Gauss points: 15 pairs), by four otherwise (register pressure)
  constexpr int UNR = NV * NT <= 15 ? NK : 4;
#pragma unroll UNR
  for (int ks = 0; ks < NK; ks++) {
    const int kc = ks * 4 + (lane & 3);
    double a[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) a[v] = loadA(v, kc);
#pragma unroll
    for (int t = 0; t < NT; t++) {
      const double b = sB[(ks * NT + t) * 32 + lane];
#pragma unroll
      for (int v = 0; v < NV; v++) dmma_884(acc[v][t], a[v], b);
    }
  }
  {
    // the last stencil cell
    double ul[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) ul[v] = loadLast(v);
#pragma unroll
    for (int t = 0; t < NT; t++)
#pragma unroll
      for (int e = 0; e < 2; e++) {
        const double wl = sWl[t * 8 + 2 * (lane & 3) + e];
#pragma unroll
        for (int v = 0; v < NV; v++) acc[v][t][e] = fma(wl, ul[v], acc[v][t][e]);
      }
  }
}

// The FP64 epilogue of one group: limiter pre-check, KXRCF indicator, face-state
// and source-point stores, the cell's status and GLM speed maxima.  bdCell = the
// limiter bounds [minDens | maxDens | minEint] of the lane's cell, `stride` apart.
template <int DIM, int EQ, int NQ>
__device__ __forceinline__ void recon_group_epilogue(
    const Grid &g, int lane, int64_t i, int64_t j, int64_t k, bool live, const double *__restrict__ bdCell,
    int stride, int wantInd, double *const (&F)[3], float *const (&W)[3], double *__restrict__ src,
    uint8_t *__restrict__ status, double2 *__restrict__ lamvel,
    const double (&acc)[Cfg<DIM, EQ, NQ>::NV][DmmaShape<DIM, EQ, NQ>::NT][2]) {
  using T = Cfg<DIM, EQ, NQ>;
  using Sh = DmmaShape<DIM, EQ, NQ>;
  constexpr int NV = T::NV, NT = Sh::NT;
  bool inside = true;
  double lam = 0.0, vel = 0.0;
  if (live) {
    const int64_t c = (k * g.ny + j) * g.nx + i;
    PosBounds bd;
    bd.minDens = bdCell[0];
    bd.maxDens = bdCell[stride];
    bd.minEint = bdCell[2 * stride];
#pragma unroll
    for (int t = 0; t < NT; t++) {
      const int rw0 = t * 8 + 2 * (lane & 3);
#pragma unroll
      for (int e = 0; e < 2; e++) {
        // row 8t + 2(lane%4) + e: face point q = row % NQF of face f = row / NQF
        // (rows past the face points are interior points); with an even NQF both
        // rows of a lane lie on one face, which the compiler then computes once
        const int rw = rw0 + e;
        const int fr = (T::NQF % 2 == 0 ? rw0 : rw) / T::NQF;
        const int f = fr < T::NF ? fr : 0;
        const int d = f >> 1;
        const int hi = f & 1;
        const int64_t nf = g.nface[d];
        const int64_t fidx = ((k + (d == 2 && hi)) * g.fdim[d][1] + (j + (d == 1 && hi))) * g.fdim[d][0] +
                             (i + (d == 0 && hi));
        const int slot = hi ? 0 : 1;
        if (rw < Sh::NR) {
          double st[NV];
#pragma unroll
          for (int v = 0; v < NV; v++) st[v] = acc[v][t][e];
          // pos_inside, with the internal energy kept for the indicator's pressure
          double ei = 0.0;
          if constexpr (EQ == EQ_SR) {
            inside = inside && pos_inside<EQ>(bd, st);
          } else {
            // Euler / Navier-Stokes: without the IEEE division (GLM-MHD, whose
            // kernel it slowed, keeps the plain expression)
            if constexpr (EQ == EQ_GLM) ei = Eos<EQ>::eint(st);
            else ei = Eos<EQ>::eint_vs(st, bd.minEint);
            inside = inside && st[DENS] > bd.minDens && st[DENS] < bd.maxDens && ei > bd.minEint;
          }
          if (rw < T::NF * T::NQF) {
            const int q = rw % T::NQF;
            double *Fd = F[d];
            const int64_t a = (int64_t)((slot * T::NQF + q) * NV) * nf + fidx;
#pragma unroll
            for (int v = 0; v < NV; v++) Fd[a + v * nf] = st[v];
            if (wantInd) {
              // SR: the indicator is the density itself, stored rounded
              const float wv = EQ == EQ_SR ? __double2float_rn(st[DENS])
                                           : Eos<EQ>::template weno_store<DIM>(g.gamma, st[DENS], (g.gamma - 1.0) * ei);
              W[d][(int64_t)(slot * T::NQF + q) * nf + fidx] = wv;
            }
            if constexpr (T::SRC) {
              // SpeedEstimate_K<MHD_GLM> (MHD_GLM_K.H:213-310): x components on every face
              const double vv = fabs(st[MOMX] / st[DENS]);
              const double l = Eos<EQ>::fastMagSonic(g.gamma, st, st[MAGX]) + vv;
              vel = vv > vel ? vv : vel;
              lam = l > lam ? l : lam;
            }
          } else if constexpr (T::SRC) {
            const int q = rw - T::NF * T::NQF;
#pragma unroll
            for (int v = 0; v < NV; v++) src[(q * NV + v) * g.n + c] = st[v];
          }
        }
      }
    }
  }
  // combine the four lanes of each cell
  inside = __shfl_xor_sync(0xffffffffu, (int)inside, 1) && inside;
  inside = __shfl_xor_sync(0xffffffffu, (int)inside, 2) && inside;
  if constexpr (T::SRC) {
    lam = fmax(lam, __shfl_xor_sync(0xffffffffu, lam, 1));
    lam = fmax(lam, __shfl_xor_sync(0xffffffffu, lam, 2));
    vel = fmax(vel, __shfl_xor_sync(0xffffffffu, vel, 1));
    vel = fmax(vel, __shfl_xor_sync(0xffffffffu, vel, 2));
  }
  if (live && (lane & 3) == 0) {
    const int64_t c = (k * g.ny + j) * g.nx + i;
    if constexpr (T::SRC) lamvel[c] = make_double2(lam, vel);
    status[c] = inside ? 1 : 0;
  }
}

// contraction and epilogue of one group in the same warp
template <int DIM, int EQ, int NQ, class LoadA, class LoadLast>
__device__ __forceinline__ void recon_group(const Grid &g, int lane, int64_t i, int64_t j, int64_t k, bool live,
                                            const double *__restrict__ sB, const double *__restrict__ sWl,
                                            const double *__restrict__ bdCell, int stride, int wantInd,
                                            double *const (&F)[3], float *const (&W)[3], double *__restrict__ src,
                                            uint8_t *__restrict__ status, double2 *__restrict__ lamvel,
                                            LoadA loadA, LoadLast loadLast) {
  double acc[Cfg<DIM, EQ, NQ>::NV][DmmaShape<DIM, EQ, NQ>::NT][2];
  recon_group_mma<DIM, EQ, NQ>(lane, sB, sWl, loadA, loadLast, acc);
  recon_group_epilogue<DIM, EQ, NQ>(g, lane, i, j, k, live, bdCell, stride, wantInd, F, W, src, status, lamvel, acc);
}

template <int DIM, int EQ, int NQ>
__global__ void __launch_bounds__(128)
    recon_kernel(const double *__restrict__ U, Grid g, const DevStencil *__restrict__ S, int wantInd,
                 double *__restrict__ F0,
                 double *__restrict__ F1, double *__restrict__ F2, float *__restrict__ W0,
                 float *__restrict__ W1, float *__restrict__ W2, double *__restrict__ src,
                 uint8_t *__restrict__ status, double2 *__restrict__ lamvel, double *__restrict__ bnd) {
  using T = Cfg<DIM, EQ, NQ>;
  using Sh = DmmaShape<DIM, EQ, NQ>;
  constexpr int NT = Sh::NT, NK = Sh::NK;
  __shared__ double tile[6][PosTile<DIM>::N];
  __shared__ double sB[Sh::BSIZE];
  __shared__ int64_t sOff[NK * 4];
  __shared__ double sWl[NT * 8]; // weights of the last stencil cell per row
  const int tid = threadIdx.y * kBlockX + threadIdx.x;
  for (int t = tid; t < Sh::BSIZE; t += kBlockX * kBlockY) sB[t] = S->dmma_b[t];
  if (tid < NK * 4) sOff[tid] = g.loff[tid];
  if (tid < NT * 8) sWl[tid] = tid < Sh::NR ? S->lin[(T::C - 1) * Sh::NR + tid] : 0.0;
  const int64_t oLast = g.loff[T::C - 1];
  const int64_t k = blockIdx.z;
  pos_tile_fill<DIM, EQ>(U, g, blockIdx.x * (int64_t)kBlockX, blockIdx.y * (int64_t)kBlockY, k, tile);
  __syncthreads();
  // limiter bounds of each block cell, once (the four lanes of a cell share them);
  // computed here, where the other resident blocks' contraction hides their loads
  __shared__ double sBd[3][kBlockX * kBlockY];
  {
    const PosBounds bd = pos_bounds_tile<DIM, EQ>(tile, threadIdx.x, threadIdx.y);
    sBd[0][tid] = bd.minDens;
    sBd[1][tid] = bd.maxDens;
    sBd[2][tid] = bd.minEint;
    // and for the heavy pass
    const int64_t bi = blockIdx.x * (int64_t)kBlockX + threadIdx.x, bj = blockIdx.y * (int64_t)kBlockY + threadIdx.y;
    if (bi < g.nx && bj < g.ny) {
      const int64_t c = (k * g.ny + bj) * g.nx + bi;
      bnd[c] = bd.minDens;
      bnd[g.n + c] = bd.maxDens;
      bnd[2 * g.n + c] = bd.minEint;
    }
  }
  __syncthreads();
  const int lane = threadIdx.x;
  const int64_t j = blockIdx.y * (int64_t)kBlockY + threadIdx.y;
  const bool rowLive = j < g.ny;
  double *const F[3] = {F0, F1, F2};
  float *const W[3] = {W0, W1, W2};
#pragma unroll 1
  for (int grp = 0; grp < kBlockX / 8; grp++) {
    const int cx = grp * 8 + (lane >> 2);
    const int64_t i = blockIdx.x * (int64_t)kBlockX + cx;
    const bool live = rowLive && i < g.nx;
    const double *Uc = U + pidx(g, live ? i : 0, rowLive ? j : 0, k);
    recon_group<DIM, EQ, NQ>(
        g, lane, i, j, k, live, sB, sWl, &sBd[0][threadIdx.y * kBlockX + cx], kBlockX * kBlockY, wantInd, F, W, src,
        status, lamvel, [&](int v, int kc) { return __ldg(Uc + v * g.pvol + sOff[kc]); },
        [&](int v) { return __ldg(Uc + v * g.pvol + oLast); });
  }
}

// The same reconstruction with the state staged in shared memory by TMA (Euler,
// Navier-Stokes and SR; GLM-MHD in 2D): one 4D tensor load per variable brings the
// block's halo tile (the cell tile plus 2 cells on every side) into shared memory
// on one mbarrier; the limiter footprint and every stencil operand then come from
// there.  3D tile 32 x 4 x 2 cells, 2D 32 x 8; one warp per row of 32 cells.
template <int DIM>
struct DmmaTile {
  static constexpr int BX = kBlockX, BY = DIM == 3 ? 4 : 8, BZ = DIM == 3 ? 2 : 1;
  static constexpr int WARPS = BY * BZ, THREADS = 32 * WARPS, CELLS = BX * BY * BZ;
  static constexpr int R = kRad;
  static constexpr int TX = BX + 2 * R, TY = BY + 2 * R, TZ = DIM == 3 ? BZ + 2 * R : 1;
  static constexpr int N = TX * TY * TZ;  // halo tile of one variable
  static constexpr int PX = BX + 2, PY = BY + 2, PZ = DIM == 3 ? BZ + 2 : 1;
  static constexpr int PN = PX * PY * PZ; // limiter footprint: the block and a one-cell ring
  static_assert((TX * 8) % 16 == 0 && (N * 8) % 128 == 0, "TMA box inner extent, tile alignment");
};

template <int DIM, int EQ, int NQ>
struct DmmaTmaSmem {
  using T = Cfg<DIM, EQ, NQ>;
  using Sh = DmmaShape<DIM, EQ, NQ>;
  using D = DmmaTile<DIM>;
  static constexpr int NV = T::NV;
  static constexpr int NP = EQ == EQ_SR ? 1 : 2;  // footprint arrays besides rho: eint, sound speed (SR: E - |S|)
  static constexpr int OFF_P = NV * D::N * 8;      // the halo tiles [v][z][y][x] come first
  static constexpr int OFF_B = OFF_P + NP * D::PN * 8;
  static constexpr int OFF_BD = OFF_B + Sh::BSIZE * 8;
  static constexpr int OFF_WL = OFF_BD + 3 * D::CELLS * 8;
  static constexpr int OFF_TO = OFF_WL + Sh::NT * 8 * 8;
  static constexpr int OFF_BAR = (OFF_TO + (4 * Sh::NK + 1) * 4 + 7) / 8 * 8;
  static constexpr int BYTES = OFF_BAR + 8;
  static_assert(BYTES <= 113 * 1024, "two blocks per SM");
};

template <int DIM, int EQ, int NQ>
__global__ void __launch_bounds__(DmmaTile<DIM>::THREADS, (DIM == 2 && NQ == 2 && Eos<EQ>::NV == 5) ? 4 : 2)
    recon_tma_kernel(const __grid_constant__ CUtensorMap umap, Grid g, const DevStencil *__restrict__ S, int wantInd,
                     double *__restrict__ F0, double *__restrict__ F1, double *__restrict__ F2,
                     float *__restrict__ W0, float *__restrict__ W1, float *__restrict__ W2,
                     double *__restrict__ src, uint8_t *__restrict__ status, double2 *__restrict__ lamvel,
                     double *__restrict__ bnd, DevScalars *__restrict__ sc) {
  using T = Cfg<DIM, EQ, NQ>;
  using Sh = DmmaShape<DIM, EQ, NQ>;
  using D = DmmaTile<DIM>;
  using L = DmmaTmaSmem<DIM, EQ, NQ>;
  using E = Eos<EQ>;
  constexpr int NV = T::NV, NT = Sh::NT, NK = Sh::NK;
  static_assert(NV == 5 || DIM == 2, "nine-variable halo tiles in 2D only");
  extern __shared__ __align__(128) uint8_t smem[];
  const double *sU = reinterpret_cast<const double *>(smem);
  double *sP = reinterpret_cast<double *>(smem + L::OFF_P);
  double *sB = reinterpret_cast<double *>(smem + L::OFF_B);
  double *sBd = reinterpret_cast<double *>(smem + L::OFF_BD);
  double *sWl = reinterpret_cast<double *>(smem + L::OFF_WL);
  int *sTo = reinterpret_cast<int *>(smem + L::OFF_TO);
  const uint32_t bar = smem_u32(smem + L::OFF_BAR);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int ty = warp % D::BY, tz = warp / D::BY;
  // the tile's first padded coordinates: cell (i0 - 2, j0 - 2, k0 - 2)
  const int i0 = (int)(blockIdx.x * D::BX), j0 = (int)(blockIdx.y * D::BY), k0 = (int)(blockIdx.z * D::BZ);
  if (tid == 0) {
    mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    mbar_arrive_expect_tx(bar, (uint32_t)(NV * D::N * 8));
#pragma unroll
    for (int v = 0; v < NV; v++) tma_load_4d(smem_u32(smem + v * D::N * 8), &umap, i0, j0, k0, v, bar);
  }
  for (int t = tid; t < Sh::BSIZE; t += D::THREADS) sB[t] = S->dmma_b[t];
  if (tid < NT * 8) sWl[tid] = tid < Sh::NR ? S->lin[(T::C - 1) * Sh::NR + tid] : 0.0;
  if (tid < 4 * NK + 1) {
    // stencil cell c (the last one at 4 NK) as an offset in the halo tile
    const int c = tid < 4 * NK ? tid : T::C - 1;
    const int dz = DIM == 3 ? (int)S->w.off[2][c] : 0;
    sTo[tid] = (dz * D::TY + (int)S->w.off[1][c]) * D::TX + (int)S->w.off[0][c];
  }
  __syncthreads();  // the barrier's initialisation is visible to every waiting thread
  if (!mbar_wait(bar, 0)) {
    // the tile never arrived: record it, give the copies in flight a bounded time
    // to land, and leave
    if (tid == 0) atomicExch(&sc->fault, 1u);
    mbar_wait(bar, 0);
    return;
  }
  // limiter footprint: eint and sound speed (SR: E - |S|) of the block and its ring
  for (int t = tid; t < D::PN; t += D::THREADS) {
    const int a = t % D::PX, b = (t / D::PX) % D::PY, cz = t / (D::PX * D::PY);
    const int h = ((cz + (DIM == 3 ? 1 : 0)) * D::TY + (b + 1)) * D::TX + (a + 1);
    double st[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) st[v] = sU[v * D::N + h];
    if constexpr (EQ == EQ_SR) {
      sP[t] = sr::ediff(st);
    } else {
      const double ir = 1.0 / st[DENS];
      const double ei = E::eint_r(st, ir);
      sP[t] = ei;
      sP[D::PN + t] = sqrt(g.gamma * ((g.gamma - 1.0) * ei) * ir);
    }
  }
  __syncthreads();
  {
    // PositivityPreserve_K bounds (Common_K.H:331-380; SR: SRHydro_K.H:224-246) of
    // this thread's cell, from the footprint (the same values pos_bounds_tile gives)
    constexpr int zr = DIM == 3 ? 1 : 0;
    auto pt = [&](int xo, int yo, int zo) { return ((tz + zr + zo) * D::PY + (ty + 1 + yo)) * D::PX + (lane + 1 + xo); };
    auto ht = [&](int xo, int yo, int zo) {
      return ((tz + (DIM == 3 ? 2 : 0) + zo) * D::TY + (ty + 2 + yo)) * D::TX + (lane + 2 + xo);
    };
    double maxDens = -1.7976931348623157e308, minDens = 1.7976931348623157e308;
    double minEint = 1.7976931348623157e308, minSdSp = 1.7976931348623157e308;
#pragma unroll
    for (int xo = -1; xo <= 1; xo++)
#pragma unroll
      for (int yo = -1; yo <= 1; yo++)
#pragma unroll
        for (int zo = -zr; zo <= zr; zo++) {
          const double r = sU[DENS * D::N + ht(xo, yo, zo)];
          maxDens = fmax(maxDens, r);
          minDens = fmin(minDens, r);
          minEint = fmin(minEint, sP[pt(xo, yo, zo)]);
          if constexpr (EQ != EQ_SR) minSdSp = fmin(minSdSp, sP[D::PN + pt(xo, yo, zo)]);
        }
    PosBounds bd;
    if constexpr (EQ == EQ_SR) {
      bd = PosBounds{sU[DENS * D::N + ht(0, 0, 0)], minDens, maxDens, minEint};
    } else {
      // velocities as m / rho, as the reference's divergence estimate (Common_K.H:363-378)
      auto vel = [&](int m, int xo, int yo, int zo) {
        const int h = ht(xo, yo, zo);
        return sU[m * D::N + h] / sU[DENS * D::N + h];
      };
      const double dxU = vel(MOMX, 1, 0, 0) - vel(MOMX, -1, 0, 0);
      const double dyV = vel(MOMY, 0, 1, 0) - vel(MOMY, 0, -1, 0);
      const double dzW = vel(MOMZ, 0, 0, zr) - vel(MOMZ, 0, 0, -zr);
      const double divV = (dxU + dyV + dzW) / 2.0;
      double kappa = 0.2;
      const double eta = fmin(1.0, fmax(0.0, -(kappa * minSdSp + divV) / (kappa * minSdSp)));
      kappa *= (1.0 - eta);
      bd.rDens = sU[DENS * D::N + ht(0, 0, 0)];
      bd.maxDens = maxDens * (1.0 + kappa);
      bd.minDens = minDens * (1.0 - kappa);
      bd.minEint = minEint * (1.0 - kappa);
    }
    sBd[tid] = bd.minDens;
    sBd[D::CELLS + tid] = bd.maxDens;
    sBd[2 * D::CELLS + tid] = bd.minEint;
    // and for the heavy pass
    const int64_t bi = i0 + lane, bj = j0 + ty, bk = k0 + tz;
    if (bi < g.nx && bj < g.ny && bk < g.nz) {
      const int64_t c = (bk * g.ny + bj) * g.nx + bi;
      bnd[c] = bd.minDens;
      bnd[g.n + c] = bd.maxDens;
      bnd[2 * g.n + c] = bd.minEint;
    }
  }
  __syncthreads();
  const int64_t j = j0 + ty, k = k0 + tz;
  const bool rowLive = j < g.ny && k < g.nz;
  double *const F[3] = {F0, F1, F2};
  float *const W[3] = {W0, W1, W2};
  const int toLast = sTo[4 * NK];
#pragma unroll 1
  for (int grp = 0; grp < D::BX / 8; grp++) {
    const int cx = grp * 8 + (lane >> 2);
    const int64_t i = i0 + cx;
    const bool live = rowLive && i < g.nx;
    // the lane's cell in the halo tile
    const double *Uc = sU + ((tz + (DIM == 3 ? 2 : 0)) * D::TY + (ty + 2)) * D::TX + (cx + 2);
    recon_group<DIM, EQ, NQ>(
        g, lane, i, j, k, live, sB, sWl, sBd + (ty + D::BY * tz) * D::BX + cx, D::CELLS, wantInd, F, W, src,
        status, lamvel, [&](int v, int kc) { return Uc[v * D::N + sTo[kc]]; },
        [&](int v) { return Uc[v * D::N + toLast]; });
  }
}

// host: the 4D tensor map of a padded state buffer for the TMA-staged tiles (x, y,
// z, variable; box = the halo tile of one variable).  Returns nonzero where TMA
// cannot be used (an odd pitch breaks the 16-byte stride rule).
int recon_dmma_state_map(CUtensorMap *map, const double *U, const Grid &g, int dim, int nv) {
  if (g.px % 2 != 0) return 1;
  const uint64_t planes = (uint64_t)(g.pvol / (g.px * g.py));
  const uint64_t dims[4] = {(uint64_t)g.px, (uint64_t)g.py, planes, (uint64_t)nv};
  const uint64_t strides[3] = {(uint64_t)g.px * 8, (uint64_t)(g.px * g.py) * 8, (uint64_t)g.pvol * 8};
  const uint32_t box[4] = {(uint32_t)(dim == 3 ? DmmaTile<3>::TX : DmmaTile<2>::TX),
                           (uint32_t)(dim == 3 ? DmmaTile<3>::TY : DmmaTile<2>::TY),
                           (uint32_t)(dim == 3 ? DmmaTile<3>::TZ : DmmaTile<2>::TZ), 1u};
  return encode_tensor_map_8b(map, U, 4, dims, strides, box);
}

// Linear reconstruction for more rows than the DMMA kernels hold in registers
// (3D GLM-MHD with three Gauss points: 54 face points and 27 interior points per
// cell).  One thread per (cell, variable) sums its rows in passes, in stencil-cell
// order as KernelLinearRecon_K does (Stencil_K.H:56-119); the face points are
// staged in shared memory and finished per cell by the cell's NV threads (limiter
// pre-check, indicator, GLM speed maxima), the interior points go to the source
// array.  The limiter bounds come from pos_bounds and are stored for the heavy pass.
template <int DIM, int EQ, int NQ>
struct RowsShape {
  using T = Cfg<DIM, EQ, NQ>;
  static constexpr int NR = LinRows<DIM, EQ, NQ>::NROWS;
  static constexpr int NFQ = T::NF * T::NQF;
  static constexpr int CELLS = 16;
  static constexpr int RCH = 27;  // rows per pass
  // cell stride of the face-state table, odd so that a warp's cells fall on
  // different shared-memory banks
  static constexpr int CS = (NFQ * T::NV) | 1;
  static constexpr size_t BYTES =
      (size_t)(T::C * NR + CELLS * CS + 3 * CELLS + 3 * T::NV * CELLS) * sizeof(double);
};

template <int DIM, int EQ, int NQ>
__global__ void __launch_bounds__(RowsShape<DIM, EQ, NQ>::CELLS * Eos<EQ>::NV)
    recon_rows_kernel(const double *__restrict__ U, Grid g, const DevStencil *__restrict__ S, int wantInd,
                      double *__restrict__ F0, double *__restrict__ F1, double *__restrict__ F2,
                      float *__restrict__ W0, float *__restrict__ W1, float *__restrict__ W2,
                      double *__restrict__ src, uint8_t *__restrict__ status, double2 *__restrict__ lamvel,
                      double *__restrict__ bnd) {
  using T = Cfg<DIM, EQ, NQ>;
  using R = RowsShape<DIM, EQ, NQ>;
  using E = Eos<EQ>;
  constexpr int NV = T::NV, NR = R::NR, NFQ = R::NFQ, C = T::C, NQF = T::NQF;
  extern __shared__ __align__(16) double rsm[];
  double *sW = rsm;                        // [stencil cell][row]
  double *sS = sW + C * NR;                // face states [cell][face row][v], cell stride CS
  double *sBd = sS + R::CELLS * R::CS;     // [minDens | maxDens | minEint][cell]
  double *sRed = sBd + 3 * R::CELLS;       // [inside | lam | vel][v][cell]
  const int x = threadIdx.x, v = threadIdx.y, tid = v * R::CELLS + x, nt = R::CELLS * NV;
  for (int t = tid; t < C * NR; t += nt) sW[t] = S->lin[t];
  const int64_t c = blockIdx.x * (int64_t)R::CELLS + x;
  const bool live = c < g.n;
  const int64_t i = live ? c % g.nx : 0, j = live ? (c / g.nx) % g.ny : 0, k = live ? c / (g.nx * g.ny) : 0;
  const double *Uc = U + pidx(g, i, j, k);
  if (v == 0 && live) {
    const PosBounds bd = pos_bounds<DIM, EQ>(Uc, g);
    sBd[x] = bd.minDens;
    sBd[R::CELLS + x] = bd.maxDens;
    sBd[2 * R::CELLS + x] = bd.minEint;
    bnd[c] = bd.minDens;
    bnd[g.n + c] = bd.maxDens;
    bnd[2 * g.n + c] = bd.minEint;
  }
  __syncthreads();
  if (live) {
    double u[C];
#pragma unroll
    for (int q = 0; q < C; q++) u[q] = Uc[v * g.pvol + g.loff[q]];
#pragma unroll 1
    for (int r0 = 0; r0 < NR; r0 += R::RCH) {
      double acc[R::RCH];
#pragma unroll
      for (int r = 0; r < R::RCH; r++) acc[r] = 0.0;
#pragma unroll
      for (int q = 0; q < C; q++) {
        const double uq = u[q];
#pragma unroll
        for (int r = 0; r < R::RCH; r++)
          if (r0 + r < NR) acc[r] = fma(sW[q * NR + r0 + r], uq, acc[r]);
      }
#pragma unroll
      for (int r = 0; r < R::RCH; r++) {
        const int row = r0 + r;
        if (row < NFQ) sS[x * R::CS + row * NV + v] = acc[r];
        else if (row < NR) src[((int64_t)(row - NFQ) * NV + v) * g.n + c] = acc[r];
      }
    }
  }
  __syncthreads();
  // the cell's face rows shared among its NV threads (rows v, v + NV, ...)
  bool inside = true;
  double lam = 0.0, vel = 0.0;
  if (live) {
    PosBounds bd;
    bd.rDens = Uc[DENS * g.pvol];
    bd.minDens = sBd[x];
    bd.maxDens = sBd[R::CELLS + x];
    bd.minEint = sBd[2 * R::CELLS + x];
    double *const F[3] = {F0, F1, F2};
    float *const W[3] = {W0, W1, W2};
    for (int row = v; row < NFQ; row += NV) {
      double st[NV];
#pragma unroll
      for (int w = 0; w < NV; w++) st[w] = sS[x * R::CS + row * NV + w];
      double ei = 0.0;
      if constexpr (EQ == EQ_SR) {
        inside = inside && pos_inside<EQ>(bd, st);
      } else {
        ei = E::eint(st);
        inside = inside && st[DENS] > bd.minDens && st[DENS] < bd.maxDens && ei > bd.minEint;
      }
      const int f = row / NQF, q = row % NQF, d = f >> 1, hi = f & 1;
      const int64_t nf = g.nface[d];
      const int64_t fidx = ((k + (d == 2 && hi)) * g.fdim[d][1] + (j + (d == 1 && hi))) * g.fdim[d][0] +
                           (i + (d == 0 && hi));
      const int slot = hi ? 0 : 1;
#pragma unroll
      for (int w = 0; w < NV; w++) F[d][((int64_t)(slot * NQF + q) * NV + w) * nf + fidx] = st[w];
      if (wantInd)
        W[d][(int64_t)(slot * NQF + q) * nf + fidx] =
            EQ == EQ_SR ? __double2float_rn(st[DENS])
                        : E::template weno_store<DIM>(g.gamma, st[DENS], (g.gamma - 1.0) * ei);
      if constexpr (T::SRC) {
        // SpeedEstimate_K<MHD_GLM> (MHD_GLM_K.H:213-310): x components on every face
        const double vv = fabs(st[MOMX] / st[DENS]);
        const double l = E::fastMagSonic(g.gamma, st, st[MAGX]) + vv;
        vel = vv > vel ? vv : vel;
        lam = l > lam ? l : lam;
      }
    }
  }
  sRed[v * R::CELLS + x] = inside ? 1.0 : 0.0;
  sRed[(NV + v) * R::CELLS + x] = lam;
  sRed[(2 * NV + v) * R::CELLS + x] = vel;
  __syncthreads();
  if (v == 0 && live) {
    bool all = true;
    double l = 0.0, vv = 0.0;
#pragma unroll
    for (int w = 0; w < NV; w++) {
      all = all && sRed[w * R::CELLS + x] != 0.0;
      l = fmax(l, sRed[(NV + w) * R::CELLS + x]);
      vv = fmax(vv, sRed[(2 * NV + w) * R::CELLS + x]);
    }
    status[c] = all ? 1 : 0;
    if constexpr (T::SRC) lamvel[c] = make_double2(l, vv);
  }
}

// PositivityPreserve_K bounds of every cell (Common_K.H:331-380; SR: SRHydro_K.H:224-246)
// from a per-block footprint tile: [minDens | maxDens | minEint][cell], the same
// values recon_kernel computes in its own prologue.  The pre-pass of the tensor-core
// reconstruction, whose shared memory holds the halo tiles instead (2D; 3D uses
// bounds_march_kernel below).
template <int DIM, int EQ>
__global__ void __launch_bounds__(128) bounds_kernel(const double *__restrict__ U, Grid g, double *__restrict__ bnd) {
  __shared__ double tile[6][PosTile<DIM>::N];
  const int64_t k = blockIdx.z;
  pos_tile_fill<DIM, EQ>(U, g, blockIdx.x * (int64_t)kBlockX, blockIdx.y * (int64_t)kBlockY, k, tile);
  __syncthreads();
  const int64_t i = blockIdx.x * (int64_t)kBlockX + threadIdx.x, j = blockIdx.y * (int64_t)kBlockY + threadIdx.y;
  if (i < g.nx && j < g.ny) {
    const PosBounds bd = pos_bounds_tile<DIM, EQ>(tile, threadIdx.x, threadIdx.y);
    const int64_t c = (k * g.ny + j) * g.nx + i;
    bnd[c] = bd.minDens;
    bnd[g.n + c] = bd.maxDens;
    bnd[2 * g.n + c] = bd.minEint;
  }
}

// The same bounds in 3D from blocks that march along z over zc planes with a ring of
// three footprint planes: each plane's quantities are computed once per block
// instead of once for each of the three cell planes that read them.  The state of
// plane k + 2 is loaded into registers while the bounds of plane k are computed,
// so the global loads do not sit between the barriers of consecutive planes.
template <int EQ>
__global__ void __launch_bounds__(128)
    bounds_march_kernel(const double *__restrict__ U, Grid g, int zc, double *__restrict__ bnd) {
  using P = PosTile<3>;
  using E = Eos<EQ>;
  constexpr int NV = E::NV;
  constexpr int PL = P::TX * P::TY;
  constexpr int NPT = (PL + 127) / 128;   // plane positions per thread (block of 128 threads)
  __shared__ double ring[6][3 * PL];      // plane kp in slot (kp + 3) % 3
  const int64_t i0 = blockIdx.x * (int64_t)kBlockX, j0 = blockIdx.y * (int64_t)kBlockY;
  const int64_t k0 = blockIdx.z * (int64_t)zc, k1 = k0 + zc < g.nz ? k0 + zc : g.nz;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  // this thread's plane positions t = tid + 128 n; false beyond the ring of any live cell
  bool use[NPT];
  int64_t off[NPT];
#pragma unroll
  for (int n = 0; n < NPT; n++) {
    const int t = tid + 128 * n;
    const int a = t % P::TX, b = t / P::TX;
    const int64_t gi = i0 - 1 + a, gj = j0 - 1 + b;
    use[n] = t < PL && gi <= g.nx && gj <= g.ny;
    off[n] = use[n] ? pidx(g, gi, gj, 0) : 0;
  }
  const int64_t pz = pidx(g, 0, 0, 1) - pidx(g, 0, 0, 0);   // one plane along z
  double st[NPT][NV];
  auto load = [&](int64_t kp) {   // the state of footprint plane kp (-1 .. nz) into st
#pragma unroll
    for (int n = 0; n < NPT; n++)
      if (use[n]) {
        const double *Uc = U + off[n] + kp * pz;
#pragma unroll
        for (int v = 0; v < NV; v++) st[n][v] = Uc[v * g.pvol];
      }
  };
  auto put = [&](int64_t kp) {    // its quantities into the plane's ring slot
    const int slot = (int)((kp + 3) % 3);
#pragma unroll
    for (int n = 0; n < NPT; n++)
      if (use[n]) pos_quantities<EQ>(st[n], g, ring, slot * PL + tid + 128 * n);
  };
  load(k0 - 1);
  put(k0 - 1);
  load(k0);
  put(k0);
  load(k0 + 1);
  const int64_t i = i0 + threadIdx.x, j = j0 + threadIdx.y;
  const int base = (threadIdx.y + 1) * P::TX + threadIdx.x + 1;
  for (int64_t k = k0; k < k1; k++) {
    put(k + 1);
    __syncthreads();
    if (k + 2 <= k1) load(k + 2);   // consumed by the next plane
    if (i < g.nx && j < g.ny) {
      const int sLo = (int)((k + 2) % 3) * PL, sMid = (int)(k % 3) * PL, sHi = (int)((k + 1) % 3) * PL;
      const PosBounds bd = pos_bounds_at<3, EQ>(ring, [&](int xo, int yo, int zo) {
        return (zo < 0 ? sLo : (zo > 0 ? sHi : sMid)) + base + yo * P::TX + xo;
      });
      const int64_t c = (k * g.ny + j) * g.nx + i;
      bnd[c] = bd.minDens;
      bnd[g.n + c] = bd.maxDens;
      bnd[2 * g.n + c] = bd.minEint;
    }
    __syncthreads();   // the next plane goes into the slot of plane k - 1
  }
}

// Throughput probe of the FP64 tensor pipe (the roofline denominator of the FP64
// reconstruction): every warp runs `iters` rounds of 8 independent m8n8k4 FP64
// MMAs on register operands; out[0] += a checksum so nothing is optimised away.
__global__ void __launch_bounds__(128) dmma_peak_kernel(int iters, double *out) {
  double acc[8][2];
  const double a = 1.0 + 1e-9 * threadIdx.x, b = 1.0 - 1e-9 * blockIdx.x;
#pragma unroll
  for (int q = 0; q < 8; q++) acc[q][0] = acc[q][1] = 0.0;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int q = 0; q < 8; q++) dmma_884(acc[q], a, b);
  }
  double sum = 0.0;
#pragma unroll
  for (int q = 0; q < 8; q++) sum += acc[q][0] + acc[q][1];
  if (sum == 1.2345) out[0] += sum;  // never true for these operands; keeps the work
}

cudaError_t launch_dmma_peak(int blocks, int iters, double *out, cudaStream_t s) {
  dmma_peak_kernel<<<blocks, 128, 0, s>>>(iters, out);
  return cudaGetLastError();
}

// KXRCF flags (WenoSelect_K, Numeric_K.H:292-398): largest indicator jump across the
// cell's faces over the cell value; the outer slot of a boundary face follows
// setFaceBCs (periodic partner face, or the inner slot at an outflow boundary).
//
// The face indicators arrive in FP32 (Eos::weno_store: in 3D the hardware
// approximation, relative error < kWenoApproxEps; in 2D the FP64 value rounded,
// < kWenoRoundEps).  The decision is taken from them only when it is certain:
// the exact jump lies within 2 eps max|w| (+ the FP32 rounding of the difference)
// of the approximate one, and the cell value is exact FP64.  Otherwise (a cell near
// the threshold, or a NaN marker) every face-point indicator is recomputed exactly
// in FP64 from the face states, as the reference computes it, so the flags are
// the reference's.
template <int DIM, int EQ>
__device__ __forceinline__ void kxrcf_face(const Grid &g, int fc, int64_t i, int64_t j, int64_t k,
                                           int64_t &fidx, int64_t &oidx, int &own, int &oth) {
  const int d = fc >> 1, hi = fc & 1;
  const int64_t fx = g.fdim[d][0], fy = g.fdim[d][1];
  const int64_t fi = i + (d == 0 && hi), fj = j + (d == 1 && hi), fk = k + (d == 2 && hi);
  fidx = (fk * fy + fj) * fx + fi;
  oidx = fidx;
  own = hi ? 0 : 1;
  oth = 1 - own;
  const int64_t m = d == 0 ? fi : (d == 1 ? fj : fk);
  const int64_t nd = d == 0 ? g.nx : (d == 1 ? g.ny : g.nz);
  const int64_t stride = d == 0 ? 1 : (d == 1 ? fx : fx * fy);
  if (m == 0 || m == nd) {
    if (g.bc[fc] == KFVM_BC_PERIODIC) oidx = m == 0 ? fidx + nd * stride : fidx - nd * stride;
    else if (!outer_in_face(g.bc[fc])) oth = own;  // an exchange / user face holds its outer slot
  }
}

template <int DIM, int EQ, int NQ>
__global__ void __launch_bounds__(128, 8)
    flag_kernel(const double *__restrict__ U, Grid g, const float *__restrict__ W0,
                const float *__restrict__ W1, const float *__restrict__ W2,
                const double *__restrict__ F0, const double *__restrict__ F1,
                const double *__restrict__ F2, const double *__restrict__ theta,
                uint8_t *__restrict__ flag, DevScalars *__restrict__ sc, double wThresh) {
  using T = Cfg<DIM, EQ, NQ>;
  constexpr int NV = T::NV;
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t j = blockIdx.y * (int64_t)blockDim.y + threadIdx.y;
  const int64_t k = blockIdx.z;
  bool f = false;
  if (i < g.nx && j < g.ny) {
    const int64_t c = (k * g.ny + j) * g.nx + i;
    f = theta[c] < 1.0;
    if (!f) {
      const float *W[3] = {W0, W1, W2};
      float jf = 0.0f, wmax = 0.0f;
      bool bad = false;
#pragma unroll
      for (int fc = 0; fc < T::NF; fc++) {
        int64_t fidx, oidx;
        int own, oth;
        kxrcf_face<DIM, EQ>(g, fc, i, j, k, fidx, oidx, own, oth);
        const int d = fc >> 1;
        const int64_t nf = g.nface[d];
#pragma unroll
        for (int q = 0; q < T::NQF; q++) {
          const float wIn = W[d][(int64_t)(own * T::NQF + q) * nf + fidx];
          const float wOut = W[d][(int64_t)(oth * T::NQF + q) * nf + oidx];
          bad = bad || !(isfinite(wIn) && isfinite(wOut));
          jf = fmaxf(jf, fabsf(wOut - wIn));
          wmax = fmaxf(wmax, fmaxf(fabsf(wIn), fabsf(wOut)));
        }
      }
      double uAv[NV];
      const double *Uc = U + pidx(g, i, j, k);
#pragma unroll
      for (int v = 0; v < NV; v++) uAv[v] = Uc[v * g.pvol];
      const double wc = Eos<EQ>::weno(g.gamma, uAv);
      bool certain = false;
      if (!bad && wc > 0.0 && isfinite(wc)) {
        const double eps = (DIM == 2 || EQ == EQ_SR) ? kWenoRoundEps : kWenoApproxEps;
        const double margin = 2.01 * eps * (double)wmax + 2e-7 * (double)jf + 1e-300;
        const double lo = ((double)jf - margin) / wc, hi = ((double)jf + margin) / wc;
        if (lo >= wThresh) {
          f = true;
          certain = true;
        } else if (hi < wThresh) {
          f = false;
          certain = true;
        }
      }
      if (!certain) {
        const double *F[3] = {F0, F1, F2};
        double maxJump = 0.0;
        for (int fc = 0; fc < T::NF; fc++) {
          int64_t fidx, oidx;
          int own, oth;
          kxrcf_face<DIM, EQ>(g, fc, i, j, k, fidx, oidx, own, oth);
          const int d = fc >> 1;
          const int64_t nf = g.nface[d];
          for (int q = 0; q < T::NQF; q++) {
            double sIn[NV], sOut[NV];
#pragma unroll
            for (int v = 0; v < NV; v++) {
              sIn[v] = F[d][((int64_t)(own * T::NQF + q) * NV + v) * nf + fidx];
              sOut[v] = F[d][((int64_t)(oth * T::NQF + q) * NV + v) * nf + oidx];
            }
            maxJump = fmax(maxJump, fabs(Eos<EQ>::weno(g.gamma, sOut) - Eos<EQ>::weno(g.gamma, sIn)));
          }
        }
        const double w = maxJump / wc;
        f = w >= wThresh;
      }
    }
    flag[c] = f ? 1 : 0;
  }
  const unsigned ball = __ballot_sync(0xffffffffu, f);
  if ((threadIdx.x & 31) == 0 && ball) atomicAdd(&sc->nflag, (unsigned)__popc(ball));
}

// WENO decision with the flag-map semantics of WenoSelector::update
// (Solver.cpp:687-742: the key set is replaced only when some cell was flagged),
// theta = 1 for in-bounds linear cells, and the heavy list.
template <int DIM, int EQ>
__global__ void __launch_bounds__(256)
    compact_kernel(Grid g, int mode, const uint8_t *__restrict__ flag, uint8_t *__restrict__ wset,
                   const uint8_t *__restrict__ status, uint8_t *__restrict__ applied,
                   double *__restrict__ theta, uint32_t *__restrict__ heavy,
                   const double2 *__restrict__ lamvel, DevScalars *__restrict__ sc, JudgeArgs jd) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  bool useWeno = false, push = false, judged = false, judgeOnly = false;
  double lam = 0.0, vel = 0.0;
  if (c < g.n) {
    if (mode == RECON_FULL) {
      useWeno = true;
    } else if (mode == RECON_SPARSE) {
      if (sc->nflag > 0) {
        useWeno = flag[c] != 0;
        wset[c] = useWeno ? 1 : 0;
      } else {
        useWeno = wset[c] != 0;
      }
    }
    // the judge's cells compute full WENO whatever the flags say (they do not enter
    // the set); one outside the set keeps its linear states unless judged troubled.
    // The judge samples runs of 32 consecutive cells (along x), so that the heavy
    // pass loads their stencils coalesced
    judged = mode == RECON_SPARSE && jd.frac > 0.0 && unit_hash(jd.seed, (uint64_t)(c >> 5)) < jd.frac;
    judgeOnly = judged && !useWeno;
    useWeno = useWeno || judged;
    applied[c] = useWeno ? 1 : 0;
    if (useWeno || !status[c]) {
      push = true;
    } else {
      theta[c] = 1.0;
      if constexpr (EQ == EQ_GLM) {
        const double2 lv = lamvel[c];
        lam = lv.x;
        vel = lv.y;
      }
    }
  }
  const unsigned lane = threadIdx.x & 31;
  const unsigned ball = __ballot_sync(0xffffffffu, push);
  const unsigned wball = __ballot_sync(0xffffffffu, useWeno);
  unsigned base = 0;
  if (lane == 0 && ball) base = atomicAdd(&sc->nheavy, (unsigned)__popc(ball));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (push)
    heavy[base + __popc(ball & ((1u << lane) - 1u))] =
        (uint32_t)c | (useWeno ? kHeavyWeno : 0u) | (judged ? kHeavyJudge : 0u) |
        (judgeOnly ? kHeavyJudgeOnly : 0u);
  if (lane == 0 && wball) atomicAdd(&sc->napplied, (unsigned)__popc(wball));
  if constexpr (EQ == EQ_GLM) {
    lam = warp_max(lam);
    vel = warp_max(vel);
    if (lane == 0) {
      atomic_max_pos(&sc->glm_lam_bits, lam);
      atomic_max_pos(&sc->glm_vel_bits, vel);
    }
  }
}

// ---------------------------------------------------------------------------
// Heavy pass, split by variable.  WENO-AO (KernelWenoRecon_K, Stencil_K.H:164-283,
// 416-590) works variable by variable on the linearised primitives: smoothness
// indicators, nonlinear weights and the blend of the substencil reconstructions
// of variable v need only that variable.  So a block takes 32 listed cells and one
// thread per (cell, variable) (threadIdx.x = cell, threadIdx.y = variable, one warp
// per variable) computes that variable at every face / interior point into
// shared memory, with all WENO weights staged in shared memory once per block;
// then one thread per cell converts back to conserved variables and runs the
// positivity procedure (PositivityPreserve_K) and the stores.  Each sum keeps the
// reference's order.
template <int DIM, int EQ, int NQ = 2>
struct HeavyShape {
  using T = Cfg<DIM, EQ, NQ>;
  static constexpr int NR = LinRows<DIM, EQ, NQ>::NROWS;      // face points, then interior points
  static constexpr int NSUM = T::C + T::CC + T::NB * T::CB;   // stencil cells over all substencils
  static constexpr int NIP = (T::NI + 1) & ~1;                // derivative rows padded to pairs
  static constexpr int DER = NIP * NSUM;                      // derivative weights [s][p][i]
  static constexpr int NRP = (NR + 1) & ~1;                  // rows padded to pairs
  static constexpr int FW = NRP * NSUM;                       // reconstruction weights [s][p][row]
  // cells per block (one thread per cell and variable); 16 where 32 cells' rows
  // would not fit in shared memory (3D GLM-MHD with three points: 81 rows x 9)
  static constexpr int CELLS = NR * T::NV > 400 ? 16 : 32;
  // 3D Euler / Navier-Stokes with two Gauss points (24 rows): both contractions
  // (derivative rows for the smoothness indicators, substencil rows for the blend)
  // on the FP64 MMA.  In 2D the per-thread form is faster: its contractions are
  // short, and the WENO cells are sparse among the listed ones, which the MMA form
  // computes for every cell of a block that has one
  static constexpr bool MMA = DIM == 3 && (EQ == EQ_HYDRO || EQ == EQ_NS) && NR <= 24 && CELLS == 32;
  static constexpr int MI = (T::NI + 7) / 8;                 // m-tiles of derivative rows
  static constexpr int MR = (NR + 7) / 8;                    // m-tiles of reconstruction rows
  static constexpr int VS = 36;                              // row stride of the stencil values [q][cell]
  // cell stride of the row results [cell][row][v], made odd so that the lanes of a
  // warp (its cells) fall on different banks (an even stride of 120 doubles put
  // all 32 lanes on two banks)
  static constexpr int CS = (NR * T::NV) | 1;
  // the MMA form's stencil values [v][q][VS] overlay the row results
  static constexpr int UNION = MMA && T::NV * T::C * VS > CELLS * CS ? T::NV * T::C * VS : CELLS * CS;
  static constexpr int COEF = MMA ? T::NV * T::NSUB * 32 : 0; // [v][s][cell]
  static constexpr size_t BYTES = (size_t)(DER + FW + UNION + CELLS * 2 + CELLS * T::NV + COEF) * sizeof(double) +
                                  (size_t)T::NB * T::CB * sizeof(int);
  __host__ __device__ static constexpr int n(int s) { return s == 0 ? T::C : (s == 1 ? T::CC : T::CB); }
  __host__ __device__ static constexpr int off(int s) {
    return s == 0 ? 0 : (s == 1 ? T::C : T::C + T::CC + (s - 2) * T::CB);
  }
};

template <int DIM, int EQ, int NQ>
__global__ void __launch_bounds__(HeavyShape<DIM, EQ, NQ>::CELLS * Eos<EQ>::NV, Eos<EQ>::NV > 5 ? 1 : 2)
    heavy_var_kernel(const double *__restrict__ U, Grid g, const DevStencil *__restrict__ S,
                     double *__restrict__ theta, double *__restrict__ F0, double *__restrict__ F1,
                     double *__restrict__ F2, double *__restrict__ src, const uint32_t *__restrict__ heavy,
                     const double *__restrict__ bnd, DevScalars *__restrict__ sc, JudgeArgs jd) {
  using T = Cfg<DIM, EQ, NQ>;
  using H = HeavyShape<DIM, EQ, NQ>;
  using E = Eos<EQ>;
  constexpr int NV = T::NV, NR = H::NR;
  extern __shared__ __align__(16) double hsm[];
  double *sDer = hsm;                       // [s][p][i], i padded to NIP
  double *sFw = sDer + H::DER;              // [s][p][row]
  double *sFs = sFw + H::FW;                // [cell][row][v], cell stride CS
  double *sV = sFs;                         // MMA form: stencil values [v][q][VS], before the rows
  double *sDep = sFs + H::UNION;            // [cell][2]
  double *sTh = sDep + H::CELLS * 2;        // limiter theta of each thread's rows [v][cell]
  double *sCo = sTh + H::CELLS * NV;        // MMA form: [v][s][cell] indicators, then blend coefficients
  int *sSub = reinterpret_cast<int *>(sCo + H::COEF);
  const kfvm_stencil &st = S->w;
  const int tid = threadIdx.y * H::CELLS + threadIdx.x, nt = H::CELLS * NV;
  // weights transposed so that the rows of one stencil value are adjacent and
  // load as 16-byte pairs
  for (int t = tid; t < H::DER; t += nt) {
    int s = 0;
    while (s + 1 < T::NSUB && t >= H::NIP * H::off(s + 1)) s++;
    const int r = t - H::NIP * H::off(s), p = r / H::NIP, i = r % H::NIP;
    sDer[t] = i < T::NI ? st.deriv_w[s][i][p] : 0.0;
  }
  for (int t = tid; t < H::FW; t += nt) {
    int s = 0;
    while (s + 1 < T::NSUB && t >= H::NRP * H::off(s + 1)) s++;
    const int r = t - H::NRP * H::off(s), p = r / H::NRP, row = r % H::NRP;
    const int nfq = T::NF * T::NQF;
    sFw[t] = row >= NR ? 0.0 : (row < nfq ? st.face_w[s][row / T::NQF][row % T::NQF][p] : st.cell_w[s][row - nfq][p]);
  }
  for (int t = tid; t < T::NB * T::CB; t += nt) sSub[t] = (int)st.sub_idx[t / T::CB][t % T::CB];
  __syncthreads();

  const unsigned count = sc->nheavy;
  const int x = threadIdx.x, v = threadIdx.y;
  double *F[3] = {F0, F1, F2};
  double lam = 0.0, vel = 0.0;
  for (unsigned base = blockIdx.x * H::CELLS; base < count; base += gridDim.x * H::CELLS) {
    const unsigned t = base + x;
    const bool have = t < count;
    const uint32_t e = have ? heavy[t] : 0u;
    const int64_t c = e & kHeavyCell;
    const int64_t i = c % g.nx, j = (c / g.nx) % g.ny, k = c / (g.nx * g.ny);
    const double *Uc = U + pidx(g, i, j, k);
    double *rs = sFs + x * H::CS;
    if constexpr (H::MMA) {
      // ---- WENO-AO with both contractions on the FP64 MMA (mma.sync m8n8k4): warp v
      // takes variable v of the block's 32 cells as the N dimension, the derivative
      // rows (smoothness indicators) and the substencil rows (reconstructions) as M,
      // the substencil's stencil entries as K.  Lanes of cells outside the WENO set
      // contribute zeros and discard their results.
      const bool mine = have && (e & kHeavyWeno);
      if (__syncthreads_or(mine)) {   // uniform over the block: every warp sees the same cells
        const int lq = x & 3, ln = x >> 2;
        double *sVw = sV + v * (T::C * H::VS);
        double *sCw = sCo + v * (T::NSUB * 32);
        double ref[NV];
#pragma unroll
        for (int w = 0; w < NV; w++) ref[w] = Uc[w * g.pvol];
        VarConv<EQ> vc(ref, g.gamma);
        {
          // component v of the linearised primitives on this lane's cell's stencil,
          // into the warp's [q][cell] table
          auto lin = [&](auto cTag) {
            constexpr int CV = decltype(cTag)::value;
#pragma unroll 4
            for (int q = 0; q < T::C; q++) {
              const int64_t o = S->loff[q];
              double u[NV];
#pragma unroll
              for (int w = 0; w < NV; w++)
                u[w] = (CV == ETOT || w == CV || w == DENS) ? Uc[w * g.pvol + o] : 0.0;
              sVw[q * H::VS + x] = vc.lin1(u, CV);
            }
          };
          if (mine) {
            switch (v) {
              case DENS: lin(std::integral_constant<int, DENS>{}); break;
              case MOMX: lin(std::integral_constant<int, MOMX>{}); break;
              case MOMY: lin(std::integral_constant<int, MOMY>{}); break;
              case MOMZ: lin(std::integral_constant<int, MOMZ>{}); break;
              default: lin(std::integral_constant<int, ETOT>{}); break;
            }
          } else {
            for (int q = 0; q < T::C; q++) sVw[q * H::VS + x] = 0.0;
          }
        }
        __syncwarp();
        auto cellOf = [&](int s, int p) { return s < 2 ? p : sSub[(s - 2) * T::CB + p]; };
        // smoothness indicators: b = D_s V_s per substencil, beta = sum of b^2 over
        // the rows (lane l holds rows 8 m + l / 4 of cells 8 t + 2 (l % 4) + e)
#pragma unroll 1
        for (int s = 0; s < T::NSUB; s++) {
          const int n = H::n(s);
          const double *D = sDer + H::NIP * H::off(s);
          double bd[H::MI][4][2];
#pragma unroll
          for (int mm = 0; mm < H::MI; mm++)
#pragma unroll
            for (int t = 0; t < 4; t++) bd[mm][t][0] = bd[mm][t][1] = 0.0;
          for (int p0 = 0; p0 < n; p0 += 4) {
            const int p = p0 + lq;
            const bool pk = p < n;
            const int q = pk ? cellOf(s, p) : 0;
            double bv[4];
#pragma unroll
            for (int t = 0; t < 4; t++) bv[t] = pk ? sVw[q * H::VS + 8 * t + ln] : 0.0;
#pragma unroll
            for (int mm = 0; mm < H::MI; mm++) {
              const int row = 8 * mm + ln;
              const double av = pk && row < T::NI ? D[p * H::NIP + row] : 0.0;
#pragma unroll
              for (int t = 0; t < 4; t++) dmma_884(bd[mm][t], av, bv[t]);
            }
          }
#pragma unroll
          for (int t = 0; t < 4; t++)
#pragma unroll
            for (int ee = 0; ee < 2; ee++) {
              double sq = 0.0;
#pragma unroll
              for (int mm = 0; mm < H::MI; mm++) sq += bd[mm][t][ee] * bd[mm][t][ee];
#pragma unroll
              for (int o = 4; o < 32; o <<= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
              if (ln == 0) sCw[s * 32 + 8 * t + 2 * lq + ee] = sq;
            }
        }
        __syncwarp();
        double om[T::NSUB];
#pragma unroll
        for (int s = 0; s < T::NSUB; s++) om[s] = sCw[s * 32 + x];
        if (mine) {
          // nonlinear weights, the judge's departure and the adaptive-order transform,
          // as the per-thread kernel computes them
          bool sig = false;
          if (jd.frac > 0.0 && (e & kHeavyJudge) && (v == DENS || v == ETOT)) {
            double lin[NV];
#pragma unroll
            for (int w = 0; w < NV; w++) lin[w] = ref[w];
            vc.cons2LinPrim(lin);
            sig = sqrt(om[0]) > kMlpFloor * fabs(v == DENS ? lin[DENS] : lin[ETOT]);
          }
          constexpr double gHi = 0.7, gLo = 0.7;
          double gam[T::NSUB];
          gam[0] = gHi;
          gam[1] = (1.0 - gHi) * gLo;
#pragma unroll
          for (int s = 2; s < T::NSUB; s++) gam[s] = (1.0 - gHi) * (1.0 - gLo) / (DIM == 2 ? 4.0 : 6.0);
          double tot = 0.0;
#pragma unroll
          for (int s = 0; s < T::NSUB; s++) {
            om[s] = gam[s] / (om[s] * om[s] + 1.e-40);
            tot += om[s];
          }
#pragma unroll
          for (int s = 0; s < T::NSUB; s++) om[s] /= tot;
          double dep = 0.0;
          if (sig)
#pragma unroll
            for (int s = 0; s < T::NSUB; s++) dep = fmax(dep, fabs(om[s] - gam[s]));
          if (v == DENS) sDep[x * 2] = dep;
          if (v == ETOT) sDep[x * 2 + 1] = dep;
          om[0] /= gam[0];
#pragma unroll
          for (int s = 1; s < T::NSUB; s++) om[s] -= om[0] * gam[s];
        }
        // each lane overwrites only its own cell's column
#pragma unroll
        for (int s = 0; s < T::NSUB; s++) sCw[s * 32 + x] = mine ? om[s] : 0.0;
        __syncwarp();
        // blend: acc = sum over s of om_s (W_s V_s), each W_s V_s summed first as the
        // reference does (per row and cell)
        double acc[H::MR][4][2];
#pragma unroll
        for (int mm = 0; mm < H::MR; mm++)
#pragma unroll
          for (int t = 0; t < 4; t++) acc[mm][t][0] = acc[mm][t][1] = 0.0;
#pragma unroll 1
        for (int s = 0; s < T::NSUB; s++) {
          const int n = H::n(s);
          const double *Wr = sFw + H::NRP * H::off(s);
          double tt[H::MR][4][2];
#pragma unroll
          for (int mm = 0; mm < H::MR; mm++)
#pragma unroll
            for (int t = 0; t < 4; t++) tt[mm][t][0] = tt[mm][t][1] = 0.0;
          for (int p0 = 0; p0 < n; p0 += 4) {
            const int p = p0 + lq;
            const bool pk = p < n;
            const int q = pk ? cellOf(s, p) : 0;
            double bv[4];
#pragma unroll
            for (int t = 0; t < 4; t++) bv[t] = pk ? sVw[q * H::VS + 8 * t + ln] : 0.0;
#pragma unroll
            for (int mm = 0; mm < H::MR; mm++) {
              const int row = 8 * mm + ln;
              const double av = pk && row < NR ? Wr[p * H::NRP + row] : 0.0;
#pragma unroll
              for (int t = 0; t < 4; t++) dmma_884(tt[mm][t], av, bv[t]);
            }
          }
#pragma unroll
          for (int t = 0; t < 4; t++)
#pragma unroll
            for (int ee = 0; ee < 2; ee++) {
              const double c = sCw[s * 32 + 8 * t + 2 * lq + ee];
              if (c != 0.0)
#pragma unroll
                for (int mm = 0; mm < H::MR; mm++) acc[mm][t][ee] += c * tt[mm][t][ee];
            }
        }
        __syncthreads();   // every warp is done with the stencil values the rows overlay
        const unsigned wm = __ballot_sync(0xffffffffu, mine);
#pragma unroll
        for (int t = 0; t < 4; t++)
#pragma unroll
          for (int ee = 0; ee < 2; ee++) {
            const int cell = 8 * t + 2 * lq + ee;
            if ((wm >> cell) & 1u)
#pragma unroll
              for (int mm = 0; mm < H::MR; mm++) {
                const int row = 8 * mm + ln;
                if (row < NR) sFs[cell * H::CS + row * NV + v] = acc[mm][t][ee];
              }
          }
      }
    } else
    if (have && (e & kHeavyWeno)) {
      // ---- variable v of WENO-AO on the linearised primitives
      double ref[NV];
#pragma unroll
      for (int w = 0; w < NV; w++) ref[w] = Uc[w * g.pvol];
      VarConv<EQ> vc(ref, g.gamma);
      // component v of the linearised primitives on the stencil (the variable is
      // uniform in the warp, so each case loads only what its component needs)
      double Vf[T::C];
      auto lin = [&](auto cTag) {
        constexpr int CV = decltype(cTag)::value;
#pragma unroll 4
        for (int q = 0; q < T::C; q++) {
          const int64_t o = S->loff[q];
          double u[NV];
#pragma unroll
          for (int w = 0; w < NV; w++)
            u[w] = (CV == ETOT || w == CV || w == DENS) ? Uc[w * g.pvol + o] : 0.0;
          Vf[q] = vc.lin1(u, CV);
        }
      };
      switch (v) {
        case DENS: lin(std::integral_constant<int, DENS>{}); break;
        case MOMX: lin(std::integral_constant<int, MOMX>{}); break;
        case MOMY: lin(std::integral_constant<int, MOMY>{}); break;
        case MOMZ: lin(std::integral_constant<int, MOMZ>{}); break;
        case ETOT: lin(std::integral_constant<int, ETOT>{}); break;
        default:
          for (int q = 0; q < T::C; q++) Vf[q] = Uc[v * g.pvol + S->loff[q]]; // magnetic field, psi
      }
      auto cellOf = [&](int s, int p) { return s < 2 ? p : sSub[(s - 2) * T::CB + p]; };
      // smoothness indicators: each stencil value is read once and feeds all
      // NI derivative rows (per row the sum over p keeps its order)
      double om[T::NSUB];
#pragma unroll 1
      for (int s = 0; s < T::NSUB; s++) {
        const int n = H::n(s);
        const double *D = sDer + H::NIP * H::off(s);
        double b[T::NI];
#pragma unroll
        for (int ii = 0; ii < T::NI; ii++) b[ii] = 0.0;
        for (int p = 0; p < n; p++) {
          const double val = Vf[cellOf(s, p)];
          const double2 *D2 = reinterpret_cast<const double2 *>(D + p * H::NIP);
#pragma unroll
          for (int i2 = 0; i2 < H::NIP / 2; i2++) {
            const double2 d = D2[i2];
            b[2 * i2] += d.x * val;
            if (2 * i2 + 1 < T::NI) b[2 * i2 + 1] += d.y * val;
          }
        }
        double beta = 0.0;
#pragma unroll
        for (int ii = 0; ii < T::NI; ii++) beta += b[ii] * b[ii];
        om[s] = beta;
      }
      bool sig = false;
      if (jd.frac > 0.0 && (e & kHeavyJudge) && (v == DENS || v == ETOT)) {
        double lin[NV];
#pragma unroll
        for (int w = 0; w < NV; w++) lin[w] = ref[w];
        vc.cons2LinPrim(lin);
        sig = sqrt(om[0]) > kMlpFloor * fabs(v == DENS ? lin[DENS] : lin[ETOT]);
      }
      constexpr double gHi = 0.7, gLo = 0.7;
      double gam[T::NSUB];
      gam[0] = gHi;
      gam[1] = (1.0 - gHi) * gLo;
#pragma unroll
      for (int s = 2; s < T::NSUB; s++) gam[s] = (1.0 - gHi) * (1.0 - gLo) / (DIM == 2 ? 4.0 : 6.0);
      double tot = 0.0;
#pragma unroll
      for (int s = 0; s < T::NSUB; s++) {
        om[s] = gam[s] / (om[s] * om[s] + 1.e-40);
        tot += om[s];
      }
#pragma unroll
      for (int s = 0; s < T::NSUB; s++) om[s] /= tot;
      double dep = 0.0;
      if (sig)
#pragma unroll
        for (int s = 0; s < T::NSUB; s++) dep = fmax(dep, fabs(om[s] - gam[s]));
      if (v == DENS) sDep[x * 2] = dep;
      if (v == ETOT) sDep[x * 2 + 1] = dep;
      om[0] /= gam[0];
#pragma unroll
      for (int s = 1; s < T::NSUB; s++) om[s] -= om[0] * gam[s];
      // blend of the substencil reconstructions at every row; each stencil value
      // feeds all rows of its substencil (per row the sum over p keeps its order).
      // Many rows (3D with three Gauss points, GLM-MHD's interior points) go in
      // passes of RCH rows, so the partial sums stay in registers.
      constexpr int RCH = H::NRP <= 24 ? H::NRP : (H::NRP % 18 == 0 ? 18 : 16);
#pragma unroll 1
      for (int r0 = 0; r0 < H::NRP; r0 += RCH) {
        double acc[RCH];
#pragma unroll
        for (int r = 0; r < RCH; r++) acc[r] = 0.0;
#pragma unroll 1
        for (int s = 0; s < T::NSUB; s++) {
          const int n = H::n(s);
          const double *Wr = sFw + H::NRP * H::off(s) + r0;
          double tt[RCH];
#pragma unroll
          for (int r = 0; r < RCH; r++) tt[r] = 0.0;
          for (int p = 0; p < n; p++) {
            const double val = Vf[cellOf(s, p)];
            const double2 *W2 = reinterpret_cast<const double2 *>(Wr + p * H::NRP);
#pragma unroll
            for (int r2 = 0; r2 < RCH / 2; r2++) {
              if (H::NRP % RCH == 0 || r0 + 2 * r2 < H::NRP) {
                const double2 w = W2[r2];
                tt[2 * r2] += w.x * val;
                tt[2 * r2 + 1] += w.y * val;
              }
            }
          }
          if (om[s] != 0.0)
#pragma unroll
            for (int r = 0; r < RCH; r++) acc[r] += om[s] * tt[r];
        }
#pragma unroll
        for (int r = 0; r < RCH; r++)
          if (r0 + r < NR) rs[(r0 + r) * NV + v] = acc[r];
      }
    }
    auto load_linear = [&]() {
      // the linear states the reconstruction pass wrote
      for (int r = 0; r < NR; r++) {
        double val;
        if (r < T::NF * T::NQF) {
          const int f = r / T::NQF, q = r % T::NQF;
          val = F[f >> 1][face_slot_addr(g, f, i, j, k, q, v, T::NQF, NV)];
        } else {
          val = src[((r - T::NF * T::NQF) * NV + v) * g.n + c];
        }
        rs[r * NV + v] = val;
      }
    };
    if (have && !(e & kHeavyWeno)) load_linear();  // limiter only
    __syncthreads();
    // a judged cell outside the WENO set that the judge finds smooth keeps its
    // linear states: the judge measures the network without perturbing the flow
    const bool keepLinear = have && (e & kHeavyJudgeOnly) && !(fmax(sDep[x * 2], sDep[x * 2 + 1]) > jd.tau);
    if (keepLinear) load_linear();
    __syncthreads();
    // ---- back to conserved variables and PositivityPreserve_K (Common_K.H:299-643;
    // SR: SRHydro_K.H:248-437).  The cell's rows are shared among its NV threads
    // (rows v, v + NV, ...); each theta is a minimum over rows, gathered through
    // shared memory, so every row ends exactly as a one-thread procedure over the
    // cell's rows in order would leave it.
    double ref[NV];
    PosBounds bd{};
    if (have) {
#pragma unroll
      for (int w = 0; w < NV; w++) ref[w] = Uc[w * g.pvol];
      if ((e & kHeavyWeno) && !keepLinear) {
        VarConv<EQ> vc(ref, g.gamma);
        for (int r = v; r < NR; r += NV) vc.linPrim2Cons(rs + r * NV);
      }
      if (v == 0 && (e & kHeavyWeno) && (e & kHeavyJudge)) {
        const double dep = fmax(sDep[x * 2], sDep[x * 2 + 1]);
        const bool lab = dep > jd.tau, p = jd.pred[c] != 0;
        atomicAdd(&sc->mlp_judged, 1ull);
        if (lab) atomicAdd(&sc->mlp_pos, 1ull);
        if (lab && !p) atomicAdd(&sc->mlp_missed, 1ull);
        if (!lab && p) atomicAdd(&sc->mlp_false, 1ull);
      }
      if (bnd) {
        // the reconstruction pass computed them (pos_bounds_tile)
        bd.rDens = ref[DENS];
        bd.minDens = bnd[c];
        bd.maxDens = bnd[g.n + c];
        bd.minEint = bnd[2 * g.n + c];
      } else {
        bd = pos_bounds<DIM, EQ>(Uc, g);
      }
    }
    const double rDens = bd.rDens, minDens = bd.minDens, maxDens = bd.maxDens, minEint = bd.minEint;
    const double rDP = maxDens - rDens, rDM = rDens - minDens;
    // the minimum of every thread's partial theta of this cell
    auto gather = [&](double th) {
      __syncthreads();  // the previous gather's reads are done
      sTh[v * H::CELLS + x] = th;
      __syncthreads();
      double m = 1.0;
#pragma unroll
      for (int w = 0; w < NV; w++) m = fmin(m, sTh[w * H::CELLS + x]);
      return m;
    };
    auto mix = [&](double th) {
      for (int r = v; r < NR; r += NV)
#pragma unroll
        for (int w = 0; w < NV; w++) rs[r * NV + w] = ref[w] + th * (rs[r * NV + w] - ref[w]);
    };
    auto replace = [&]() {
      for (int r = v; r < NR; r += NV)
#pragma unroll
        for (int w = 0; w < NV; w++) rs[r * NV + w] = ref[w];
    };
    __syncthreads();  // every row is converted
    double thD = 1.0, th2 = 1.0;
    if (have)
      for (int r = v; r < NR; r += NV) {
        const double rho = rs[r * NV + DENS];
        if constexpr (EQ == EQ_SR) {
          thD = rho < minDens ? fmin(thD, rDM / (rDens - rho)) : thD;
          thD = rho > maxDens ? fmin(thD, rDP / (rho - rDens)) : thD;
        } else {
          thD = rho > minDens ? thD : fmin(thD, rDM / (rDens - rho));
          thD = rho < maxDens ? thD : fmin(thD, rDP / (rho - rDens));
        }
      }
    thD = gather(thD);
    if (have) {
      if constexpr (EQ == EQ_SR) {
        // both thetas applied also when they are 1
        mix(thD);
        const double edRef = sr::ediff(ref), edd = edRef - minEint;
        for (int r = v; r < NR; r += NV) {
          const double ed = sr::ediff(rs + r * NV);
          th2 = ed < minEint ? fmin(th2, edd / (edRef - ed)) : th2;
        }
      } else {
        if (thD > 0.0 && thD < 1.0) mix(thD);
        else if (thD < 1.0) replace();
        for (int r = v; r < NR; r += NV) {
          double st[NV];
#pragma unroll
          for (int w = 0; w < NV; w++) st[w] = rs[r * NV + w];
          if (!(E::eint(st) > minEint)) {
            double a = 0.0, b = 1.0;
            for (int itb = 0; itb < 10; itb++) {
              const double cm = 0.5 * (a + b);
              double sm[NV];
#pragma unroll
              for (int w = 0; w < NV; w++) sm[w] = ref[w] + cm * (st[w] - ref[w]);
              if (E::eint(sm) - minEint > 0.0) a = cm;
              else b = cm;
            }
            th2 = fmin(th2, a);
          }
        }
      }
    }
    th2 = gather(th2);
    if (have) {
      if constexpr (EQ == EQ_SR) {
        mix(th2);
      } else {
        if (th2 > 0.0 && th2 < 1.0) mix(th2);
        else if (th2 < 1.0) replace();
      }
      if (v == 0) theta[c] = fmin(thD, th2);
      if constexpr (T::SRC) {
        for (int r = v; r < T::NF * T::NQF; r += NV) {
          const double *u = rs + r * NV;
          const double vv = fabs(u[MOMX] / u[DENS]);
          const double l = E::fastMagSonic(g.gamma, u, u[MAGX]) + vv;
          vel = vv > vel ? vv : vel;
          lam = l > lam ? l : lam;
        }
      }
    }
    __syncthreads();
    // stores: thread (cell, v) writes variable v of every row
    if (have) {
      for (int r = 0; r < NR; r++) {
        const double val = rs[r * NV + v];
        if (r < T::NF * T::NQF) {
          const int f = r / T::NQF, q = r % T::NQF;
          F[f >> 1][face_slot_addr(g, f, i, j, k, q, v, T::NQF, NV)] = val;
        } else {
          src[((r - T::NF * T::NQF) * NV + v) * g.n + c] = val;
        }
      }
    }
    __syncthreads();
  }
  if constexpr (T::SRC) {
    // every variable thread holds the maxima of its share of the face rows; each
    // offers them itself (a block of 16 cells x 9 variables ends in a half warp,
    // so no warp shuffle here; the read-before-atomic skips all but the raising ones)
    atomic_max_pos(&sc->glm_lam_bits, lam);
    atomic_max_pos(&sc->glm_vel_bits, vel);
  }
}

// ---------------------------------------------------------------------------
// Riemann fluxes of direction D: one thread per face point (block = 32 faces x NQF
// points, points along threadIdx.y), so each thread keeps only one solve live and
// more warps hide the FP64 latency.  The quadrature-weighted sum over a face's
// points goes through shared memory in point order, and the max wave speed
// through a warp maximum and an atomic only from warps that raise it.
// SAME: faces whose two states agree to kSameTol take the consistent flux F(u)
// without the wave fan (Eos::solve_same); one block in
// kSameSample counts such faces so that the host can fall back to the plain
// variant where few faces qualify (its slow path spills more registers).
constexpr int kSameSample = 1024;

template <int DIM, int EQ, int D, int NQ, bool SAME>
__global__ void __launch_bounds__(32 * Cfg<DIM, EQ, NQ>::NQF,
                                  EQ == EQ_GLM ? 1
                                               : (EQ == EQ_SR ? (DIM == 2 ? 8 : 4)
                                                              : (DIM == 2 ? 16 : (NQ == 3 ? 7 : 8))))
    riemann_kernel(const double *__restrict__ F, double *__restrict__ G, Grid g,
                   DevScalars *__restrict__ sc) {
  using T = Cfg<DIM, EQ, NQ>;
  using E = Eos<EQ>;
  constexpr int NV = T::NV, NQF = T::NQF;
  __shared__ double part[NQF][NV][32];
  const int64_t fx = g.fdim[D][0], fy = g.fdim[D][1], nf = g.nface[D];
  // the face within its (x, y) plane, split with 32-bit arithmetic (a plane holds
  // far fewer than 2^32 faces)
  const unsigned flat = blockIdx.x * 32u + threadIdx.x, ux = (unsigned)fx;
  const unsigned jj = flat / ux;
  const int64_t i = (int64_t)(flat - jj * ux), j = jj;
  const int64_t k = blockIdx.z;
  const int q = threadIdx.y;
  double vmax = 0.0;
  const bool live = j < fy;
  bool same = false;
  if (live) {
    const int64_t fidx = (k * fy + j) * fx + i;
    const int64_t m = D == 0 ? i : (D == 1 ? j : k);
    const int64_t nd = D == 0 ? g.nx : (D == 1 ? g.ny : g.nz);
    // face BCs (setFaceBCs): boundary faces take the missing slot from the
    // periodic partner face, or copy the interior slot at an outflow boundary
    int64_t f0 = fidx, f1 = fidx;
    int s0 = 0, s1 = 1;
    const int64_t stride = D == 0 ? 1 : (D == 1 ? fx : fx * fy);
    // (an exchange or user face holds the outer state in its own outer slot)
    if (m == 0) {
      if (g.bc[2 * D] == KFVM_BC_PERIODIC) f0 = fidx + nd * stride;
      else if (!outer_in_face(g.bc[2 * D])) s0 = 1;
    } else if (m == nd) {
      if (g.bc[2 * D + 1] == KFVM_BC_PERIODIC) f1 = fidx - nd * stride;
      else if (!outer_in_face(g.bc[2 * D + 1])) s1 = 0;
    }
    const double ch = EQ == EQ_GLM ? __longlong_as_double((long long)sc->glm_lam_bits) -
                                         __longlong_as_double((long long)sc->glm_vel_bits)
                                   : 0.0;
    double uL[NV], uR[NV], Fq[NV];
    const double *pL = F + (int64_t)(s0 * NQF + q) * NV * nf + f0;
    const double *pR = F + (int64_t)(s1 * NQF + q) * NV * nf + f1;
#pragma unroll
    for (int v = 0; v < NV; v++) {
      uL[v] = __ldg(pL + v * nf);
      uR[v] = __ldg(pR + v * nf);
    }
    if (s0 == 1 || s1 == 0) {
      // a wall face (reflecting / no-slip) mirrors the inner state with sign flips
      const unsigned flipL = s0 == 1 ? g.bflip[2 * D] : 0u, flipR = s1 == 0 ? g.bflip[2 * D + 1] : 0u;
#pragma unroll
      for (int v = 0; v < NV; v++) {
        if ((flipL >> v) & 1u) uL[v] = -uL[v];
        if ((flipR >> v) & 1u) uR[v] = -uR[v];
      }
    }
    if constexpr (SAME) {
      // a face inside a uniform region needs no wave fan (kSameTol)
      same = E::same_state(uL, uR);
      if (same) vmax = E::solve_same(g.gamma, ch, D, uL, Fq);
      else vmax = E::solve(g.rs, g.gamma, ch, D, uL, uR, Fq);
    } else {
      vmax = E::solve(g.rs, g.gamma, ch, D, uL, uR, Fq);
    }
    // Gauss weight of point q (3D: the product of the two transverse weights)
    const double wq = DIM == 2 ? gl_wt<NQ>(q) : gl_wt<NQ>(q / NQ) * gl_wt<NQ>(q % NQ);
#pragma unroll
    for (int v = 0; v < NV; v++) part[q][v][threadIdx.x] = wq * Fq[v];
  }
  __shared__ unsigned cnt[2];
  const bool sampled = SAME && (blockIdx.x + 11u * blockIdx.z) % kSameSample == 0;
  if (sampled && threadIdx.x == 0 && q == 0) cnt[0] = cnt[1] = 0u;
  __syncthreads();
  if (sampled) {
    const unsigned bs = __ballot_sync(0xffffffffu, same), bl = __ballot_sync(0xffffffffu, live);
    if (threadIdx.x == 0) {
      atomicAdd(&cnt[0], (unsigned)__popc(bs));
      atomicAdd(&cnt[1], (unsigned)__popc(bl));
    }
  }
  if (live && q == 0) {
    const int64_t fidx = (k * fy + j) * fx + i;
#pragma unroll
    for (int v = 0; v < NV; v++) {
      double acc = 0.0;
#pragma unroll
      for (int p = 0; p < NQF; p++) acc += part[p][v][threadIdx.x];
      G[(int64_t)v * nf + fidx] = acc;
    }
  }
  vmax = warp_max(vmax);
  if (threadIdx.x == 0) atomic_max_pos(&sc->maxvel_bits, vmax);
  if (sampled) {
    __syncthreads();
    if (threadIdx.x == 0 && q == 0) {
      atomicAdd(&sc->nsame, (unsigned long long)cnt[0]);
      atomicAdd(&sc->nsamp, (unsigned long long)cnt[1]);
    }
  }
}

// ---------------------------------------------------------------------------
// GLM source terms at the interior points of a cell (SourceTerms_K<MHD_GLM>,
// MHD_GLM_K.H:316-547, zero user forcing), added to rhs with the cell quadrature
template <int DIM, int NQ>
__device__ void glm_sources(const double *__restrict__ Uc, const Grid &g, int64_t i, int64_t j,
                            int64_t k, int64_t c, const double *__restrict__ F0,
                            const double *__restrict__ F1, const double *__restrict__ F2,
                            const double *__restrict__ src, double th, double *rhs) {
  using T = Cfg<DIM, EQ_GLM, NQ>;
  constexpr int NV = 9, NQF = T::NQF;
  constexpr int nzq = DIM == 3 ? NQ : 1;
  static_assert(NQ == 2 || NQ == 3, "differentiation matrices for 2 and 3 points");
  // LGL -> GL differentiation matrix, row-major NQ x (NQ + 2): output point, inputs
  // [left face, interior points in abscissa order, right face] (Numeric.cpp:50-70)
  constexpr double D2[2][4] = {
      {-2.7320508075688767, 1.732050807568877, 1.7320508075688767, -0.7320508075688767},
      {0.7320508075688767, -1.7320508075688767, -1.732050807568877, 2.7320508075688767}};
  constexpr double D3[3][5] = {
      {1.5, 0.0, -3.2274861218395139, 3.2274861218395148, -1.5},
      {-5.323790007724451, 2.06559111797729, 3.872983346207419, -1.2909944487358063, 0.6762099922755506},
      {-0.6762099922755498, -2.0655911179772883, 1.2909944487358065, -3.8729833462074184, 5.323790007724451}};
  auto Dm = [&](int r, int col) {
    if constexpr (NQ == 3) return D3[r][col];
    else return D2[r][col];
  };
  const double *Fd[3] = {F0, F1, F2};
  // face value of variable v at point q of face (d, index fi,fj,fk), slot s with face BCs
  auto fv = [&](int d, int64_t fi, int64_t fj, int64_t fk, int s, int q, int v) {
    const int64_t fx = g.fdim[d][0], fy = g.fdim[d][1];
    const int64_t m = d == 0 ? fi : (d == 1 ? fj : fk);
    const int64_t nd = d == 0 ? g.nx : (d == 1 ? g.ny : g.nz);
    const int64_t stride = d == 0 ? 1 : (d == 1 ? fx : fx * fy);
    int64_t fidx = (fk * fy + fj) * fx + fi;
    unsigned flip = 0u;
    if (m == 0 && s == 0) {
      if (g.bc[2 * d] == KFVM_BC_PERIODIC) fidx += nd * stride;
      else if (!outer_in_face(g.bc[2 * d])) {
        s = 1;
        flip = g.bflip[2 * d];
      }
    } else if (m == nd && s == 1) {
      if (g.bc[2 * d + 1] == KFVM_BC_PERIODIC) fidx -= nd * stride;
      else if (!outer_in_face(g.bc[2 * d + 1])) {
        s = 0;
        flip = g.bflip[2 * d + 1];
      }
    }
    const double x = Fd[d][((int64_t)(s * NQF + q) * NV + v) * g.nface[d] + fidx];
    return (flip >> v) & 1u ? -x : x;
  };
  double wt[NQ];
#pragma unroll
  for (int q = 0; q < NQ; q++) wt[q] = gl_wt<NQ>(q);
  double divB = 0.0;
  for (int nQ = 0; nQ < NQ; nQ++)
    for (int nS = 0; nS < nzq; nS++) {
      const int qIdx = nS * NQ + nQ;
      const double twt = DIM == 2 ? wt[nQ] : wt[nQ] * wt[nS];
      const double bAvW = 0.5 * (fv(0, i, j, k, 1, qIdx, MAGX) + fv(0, i, j, k, 0, qIdx, MAGX));
      const double bAvE = 0.5 * (fv(0, i + 1, j, k, 0, qIdx, MAGX) + fv(0, i + 1, j, k, 1, qIdx, MAGX));
      divB += twt * (bAvE - bAvW) / g.dx;
      const double bAvS = 0.5 * (fv(1, i, j, k, 1, qIdx, MAGY) + fv(1, i, j, k, 0, qIdx, MAGY));
      const double bAvN = 0.5 * (fv(1, i, j + 1, k, 0, qIdx, MAGY) + fv(1, i, j + 1, k, 1, qIdx, MAGY));
      divB += twt * (bAvN - bAvS) / g.dy;
      if (DIM == 3) {
        const double bAvB = 0.5 * (fv(2, i, j, k, 1, qIdx, MAGZ) + fv(2, i, j, k, 0, qIdx, MAGZ));
        const double bAvT = 0.5 * (fv(2, i, j, k + 1, 0, qIdx, MAGZ) + fv(2, i, j, k + 1, 1, qIdx, MAGZ));
        divB += twt * (bAvT - bAvB) / g.dz;
      }
    }
  auto cv = [&](int a, int b, int e, int v) {
    return src[((int64_t)((a * NQ + b) * nzq + e) * NV + v) * g.n + c];
  };
  const int64_t sy = g.px, sz = g.px * g.py;
  for (int nQ = 0; nQ < NQ; nQ++)
    for (int nR = 0; nR < NQ; nR++)
      for (int nS = 0; nS < nzq; nS++) {
        double st[NV];
#pragma unroll
        for (int v = 0; v < NV; v++) st[v] = cv(nQ, nR, nS, v);
        const double rho = st[DENS];
        const double vx = st[MOMX] / rho, vy = st[MOMY] / rho, vz = st[MOMZ] / rho;
        double dpx, dpy, dpz = 0.0;
        if (th < 0.75) {
          const double tdx = 1.0 / (2.0 * g.dx), tdy = 1.0 / (2.0 * g.dy);
          dpx = tdx * (Uc[PSI * g.pvol + 1] - Uc[PSI * g.pvol - 1]);
          dpy = tdy * (Uc[PSI * g.pvol + sy] - Uc[PSI * g.pvol - sy]);
          if (DIM == 3) {
            const double tdz = 1.0 / (2.0 * g.dz);
            dpz = tdz * (Uc[PSI * g.pvol + sz] - Uc[PSI * g.pvol - sz]);
          }
        } else {
          {
            const int fIdx = DIM == 2 ? nR : nR * NQ + nS;
            double d = Dm(nQ, 0) * fv(0, i, j, k, 1, fIdx, PSI) + Dm(nQ, NQ + 1) * fv(0, i + 1, j, k, 0, fIdx, PSI);
            for (int m = 1; m <= NQ; m++) d += Dm(nQ, m) * cv(m - 1, nR, nS, PSI);
            dpx = d / g.dx;
          }
          {
            const int fIdx = DIM == 2 ? nQ : nQ * NQ + nS;
            double d = Dm(nR, 0) * fv(1, i, j, k, 1, fIdx, PSI) + Dm(nR, NQ + 1) * fv(1, i, j + 1, k, 0, fIdx, PSI);
            for (int m = 1; m <= NQ; m++) d += Dm(nR, m) * cv(nQ, m - 1, nS, PSI);
            dpy = d / g.dy;
          }
          if (DIM == 3) {
            const int fIdx = nQ * NQ + nR;
            double d = Dm(nS, 0) * fv(2, i, j, k, 1, fIdx, PSI) + Dm(nS, NQ + 1) * fv(2, i, j, k + 1, 0, fIdx, PSI);
            for (int m = 1; m <= NQ; m++) d += Dm(nS, m) * cv(nQ, nR, m - 1, PSI);
            dpz = d / g.dz;
          }
        }
        const double gpsiDu = vx * dpx + vy * dpy + vz * dpz;
        const double uDb = vx * st[MAGX] + vy * st[MAGY] + vz * st[MAGZ];
        double sv[NV];
        sv[DENS] = 0.0;
        sv[MOMX] = -divB * st[MAGX];
        sv[MOMY] = -divB * st[MAGY];
        sv[MOMZ] = -divB * st[MAGZ];
        sv[ETOT] = -(divB * uDb + gpsiDu * st[PSI]);
        sv[MAGX] = -divB * vx;
        sv[MAGY] = -divB * vy;
        sv[MAGZ] = -divB * vz;
        sv[PSI] = -gpsiDu;
        const double w = DIM == 2 ? wt[nQ] * wt[nR] : wt[nQ] * wt[nR] * wt[nS];
#pragma unroll
        for (int v = 0; v < NV; v++) rhs[v] += w * sv[v];
      }
}

// compact viscous stress and heat flux (Viscosity_K<NavierStokes>, NavierStokes_K.H:190-407)
template <int DIM>
__device__ void viscous(const double (*vt)[PosTile<DIM>::N], const Grid &g, int tx, int ty, double Re,
                        double Pr, double *rhs) {
  // velocities and temperature of the 3^d neighbourhood from the block's tile
  using P = PosTile<DIM>;
  constexpr int zr = DIM == 3 ? 1 : 0;
  // the reference's divisions by 3 and 6 as products with the rounded reciprocals
  constexpr double kThird = 1.0 / 3.0, kSixth = 1.0 / 6.0;
  auto prim = [&](int xo, int yo, int zo, double &u, double &v, double &w, double &T) {
    const int t = ((zr + zo) * P::TY + (ty + 1 + yo)) * P::TX + (tx + 1 + xo);
    u = vt[0][t];
    v = vt[1][t];
    w = vt[2][t];
    T = vt[3][t];
  };
  if constexpr (DIM == 2) {
    const double rdx = g.rdx, rdy = g.rdy;
    double u[3][3], v[3][3], w[3][3], T[3][3];
#pragma unroll
    for (int xo = -1; xo <= 1; xo++)
#pragma unroll
      for (int yo = -1; yo <= 1; yo++)
        prim(xo, yo, 0, u[xo + 1][yo + 1], v[xo + 1][yo + 1], w[xo + 1][yo + 1], T[xo + 1][yo + 1]);
    double px[4], mx[4], py[4], my[4];
    px[0] = 4.0 * rdx * (u[2][1] - u[1][1]) * kThird;
    px[0] -= rdy * (v[1][2] + v[2][2] - v[1][0] - v[2][0]) * kSixth;
    px[1] = rdy * (u[1][2] + u[2][2] - u[1][0] - u[2][0]) * 0.25;
    px[1] += rdx * (v[2][1] - v[1][1]);
    px[2] = rdx * (w[2][1] - w[1][1]);
    mx[0] = 4.0 * rdx * (u[1][1] - u[0][1]) * kThird;
    mx[0] -= rdy * (v[0][2] + v[1][2] - v[0][0] - v[1][0]) * kSixth;
    mx[1] = rdy * (u[0][2] + u[1][2] - u[0][0] - u[1][0]) * 0.25;
    mx[1] += rdx * (v[1][1] - v[0][1]);
    mx[2] = rdx * (w[1][1] - w[0][1]);
    py[0] = rdx * (v[2][2] + v[2][1] - v[0][2] - v[0][1]) * 0.25;
    py[0] += rdy * (u[1][2] - u[1][1]);
    py[1] = 4.0 * rdy * (v[1][2] - v[1][1]) * kThird;
    py[1] -= rdx * (u[2][2] + u[2][1] - u[0][2] - u[0][1]) * kSixth;
    py[2] = rdy * (w[1][2] - w[1][1]);
    my[0] = rdx * (v[2][1] + v[2][0] - v[0][1] - v[0][0]) * 0.25;
    my[0] += rdy * (u[1][1] - u[1][0]);
    my[1] = 4.0 * rdy * (v[1][1] - v[1][0]) * kThird;
    my[1] -= rdx * (u[2][1] + u[2][0] - u[0][1] - u[0][0]) * kSixth;
    my[2] = rdy * (w[1][1] - w[1][0]);
    px[3] = rdx * (T[2][1] - T[1][1]);
    mx[3] = rdx * (T[1][1] - T[0][1]);
    py[3] = rdy * (T[1][2] - T[1][1]);
    my[3] = rdy * (T[1][1] - T[1][0]);
    const double rRe = 1.0 / Re;
    const double sru = rRe * (rdx * (px[0] - mx[0]) + rdy * (py[0] - my[0]));
    const double srv = rRe * (rdx * (px[1] - mx[1]) + rdy * (py[1] - my[1]));
    const double srw = rRe * (rdx * (px[2] - mx[2]) + rdy * (py[2] - my[2]));
    const double rAl = 1.0 / (Pr * Re);
    const double ste = rAl * (rdx * (px[3] - mx[3]) + rdy * (py[3] - my[3]));
    rhs[MOMX] += sru;
    rhs[MOMY] += srv;
    rhs[MOMZ] += srw;
    rhs[ETOT] += ste + u[1][1] * sru + v[1][1] * srv + w[1][1] * srw;
  } else {
    const double rdx = g.rdx, rdy = g.rdy, rdz = g.rdz;
    double u[3][3][3], v[3][3][3], w[3][3][3], T[3][3][3];
#pragma unroll
    for (int xo = -1; xo <= 1; xo++)
#pragma unroll
      for (int yo = -1; yo <= 1; yo++)
#pragma unroll
        for (int zo = -1; zo <= 1; zo++)
          prim(xo, yo, zo, u[xo + 1][yo + 1][zo + 1], v[xo + 1][yo + 1][zo + 1],
               w[xo + 1][yo + 1][zo + 1], T[xo + 1][yo + 1][zo + 1]);
    double px[4], mx[4], py[4], my[4], pz[4], mz[4];
    px[0] = 4.0 * rdx * (u[2][1][1] - u[1][1][1]) * kThird;
    px[0] -= rdy * (v[1][2][1] + v[2][2][1] - v[1][0][1] - v[2][0][1]) * kSixth;
    px[0] -= rdz * (w[1][1][2] + w[2][1][2] - w[1][1][0] - w[2][1][0]) * kSixth;
    px[1] = rdy * (u[1][2][1] + u[2][2][1] - u[1][0][1] - u[2][0][1]) * 0.25;
    px[1] += rdx * (v[2][1][1] - v[1][1][1]);
    px[2] = rdz * (u[2][1][2] + u[1][1][2] - u[2][1][0] - u[1][1][0]) * 0.25;
    px[2] += rdx * (w[2][1][1] - w[1][1][1]);
    mx[0] = 4.0 * rdx * (u[1][1][1] - u[0][1][1]) * kThird;
    mx[0] -= rdy * (v[0][2][1] + v[1][2][1] - v[0][0][1] - v[1][0][1]) * kSixth;
    mx[0] -= rdz * (w[0][1][2] + w[1][1][2] - w[0][1][0] - w[1][1][0]) * kSixth;
    mx[1] = rdy * (u[0][2][1] + u[1][2][1] - u[0][0][1] - u[1][0][1]) * 0.25;
    mx[1] += rdx * (v[1][1][1] - v[0][1][1]);
    mx[2] = rdz * (u[1][1][2] + u[0][1][2] - u[1][1][0] - u[0][1][0]) * 0.25;
    mx[2] += rdx * (w[1][1][1] - w[0][1][1]);
    py[0] = rdx * (v[2][2][1] + v[2][1][1] - v[0][2][1] - v[0][1][1]) * 0.25;
    py[0] += rdy * (u[1][2][1] - u[1][1][1]);
    py[1] = 4.0 * rdy * (v[1][2][1] - v[1][1][1]) * kThird;
    py[1] -= rdx * (u[2][2][1] + u[2][1][1] - u[0][2][1] - u[0][1][1]) * kSixth;
    py[1] -= rdz * (w[1][2][2] + w[1][1][2] - w[1][2][0] - w[1][1][0]) * kSixth;
    py[2] = rdz * (v[1][2][2] + v[1][1][2] - v[1][2][0] - v[1][1][0]) * 0.25;
    py[2] += rdy * (w[1][2][1] - w[1][1][1]);
    my[0] = rdx * (v[2][1][1] + v[2][0][1] - v[0][1][1] - v[0][0][1]) * 0.25;
    my[0] += rdy * (u[1][1][1] - u[1][0][1]);
    my[1] = 4.0 * rdy * (v[1][1][1] - v[1][0][1]) * kThird;
    my[1] -= rdx * (u[2][1][1] + u[2][0][1] - u[0][1][1] - u[0][0][1]) * kSixth;
    my[1] -= rdz * (w[1][1][2] + w[1][0][2] - w[1][1][0] - w[1][0][0]) * kSixth;
    my[2] = rdz * (v[1][1][2] + v[1][0][2] - v[1][1][0] - v[1][0][0]) * 0.25;
    my[2] += rdy * (w[1][1][1] - w[1][0][1]);
    pz[0] = rdx * (w[2][2][1] + w[2][1][1] - w[0][2][1] - w[0][1][1]) * 0.25;
    pz[0] += rdz * (u[1][1][2] - u[1][1][1]);
    pz[1] = rdy * (w[1][2][2] + w[1][2][1] - w[1][0][2] - w[1][0][1]) * 0.25;
    pz[1] += rdz * (v[1][1][2] - v[1][1][1]);
    pz[2] = 4.0 * rdz * (w[1][1][2] - w[1][1][1]) * kThird;
    pz[2] -= rdx * (u[2][2][1] + u[2][1][1] - u[0][2][1] - u[0][1][1]) * kSixth;
    pz[2] -= rdy * (v[1][2][2] + v[1][2][1] - v[1][0][2] - v[1][0][1]) * kSixth;
    mz[0] = rdx * (w[2][2][0] + w[2][1][0] - w[0][2][0] - w[0][1][0]) * 0.25;
    mz[0] += rdz * (u[1][1][1] - u[1][1][0]);
    mz[1] = rdy * (w[1][2][1] + w[1][2][0] - w[1][0][1] - w[1][0][0]) * 0.25;
    mz[1] += rdz * (v[1][1][1] - v[1][1][0]);
    mz[2] = 4.0 * rdz * (w[1][1][1] - w[1][1][0]) * kThird;
    mz[2] -= rdx * (u[2][2][0] + u[2][1][0] - u[0][2][0] - u[0][1][0]) * kSixth;
    mz[2] -= rdy * (v[1][2][1] + v[1][2][0] - v[1][0][1] - v[1][0][0]) * kSixth;
    px[3] = rdx * (T[2][1][1] - T[1][1][1]);
    mx[3] = rdx * (T[1][1][1] - T[0][1][1]);
    py[3] = rdy * (T[1][2][1] - T[1][1][1]);
    my[3] = rdy * (T[1][1][1] - T[1][0][1]);
    pz[3] = rdz * (T[1][1][2] - T[1][1][1]);
    mz[3] = rdz * (T[1][1][1] - T[1][1][0]);
    const double rRe = 1.0 / Re;
    const double sru = rRe * (rdx * (px[0] - mx[0]) + rdy * (py[0] - my[0]) + rdz * (pz[0] - mz[0]));
    const double srv = rRe * (rdx * (px[1] - mx[1]) + rdy * (py[1] - my[1]) + rdz * (pz[1] - mz[1]));
    const double srw = rRe * (rdx * (px[2] - mx[2]) + rdy * (py[2] - my[2]) + rdz * (pz[2] - mz[2]));
    const double rAl = 1.0 / (Re * Pr);
    const double ste = rAl * (rdx * (px[3] - mx[3]) + rdy * (py[3] - my[3]) + rdz * (pz[3] - mz[3]));
    rhs[MOMX] += sru;
    rhs[MOMY] += srv;
    rhs[MOMZ] += srw;
    rhs[ETOT] += ste + u[1][1][1] * sru + v[1][1][1] * srv + w[1][1][1] * srw;
  }
}

// ---------------------------------------------------------------------------
// flux divergence (+ viscous, + GLM sources) fused with the RK register update
template <int DIM, int EQ, int NQ>
__global__ void __launch_bounds__(128)
    stage_kernel(const double *__restrict__ U, double *__restrict__ Unext,
                 const double *__restrict__ Uprev, double *__restrict__ Uhat,
                 double *__restrict__ Utmp, double *__restrict__ K, Grid g,
                 const double *__restrict__ G0, const double *__restrict__ G1,
                 const double *__restrict__ G2, const double *__restrict__ F0,
                 const double *__restrict__ F1, const double *__restrict__ F2,
                 const double *__restrict__ src, const double *__restrict__ theta, int mode,
                 StageCoef co, double Re, double Pr, double atol, double rtol,
                 double *__restrict__ part) {
  using T = Cfg<DIM, EQ, NQ>;
  using E = Eos<EQ>;
  constexpr int NV = T::NV;
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t j = blockIdx.y * (int64_t)blockDim.y + threadIdx.y;
  const int64_t k = blockIdx.z;
  double err = 0.0, pos = 1.0;
  // Navier-Stokes: velocities and temperature of the block's cells and a
  // one-cell ring, once per cell (one reciprocal of the density each)
  constexpr int NVT = EQ == EQ_NS ? 4 : 1, NTT = EQ == EQ_NS ? PosTile<DIM>::N : 1;
  __shared__ double vt[NVT][NTT];
  if constexpr (EQ == EQ_NS) {
    using P = PosTile<DIM>;
    const int64_t i0 = blockIdx.x * (int64_t)blockDim.x, j0 = blockIdx.y * (int64_t)blockDim.y;
    for (int t = threadIdx.y * blockDim.x + threadIdx.x; t < P::N; t += blockDim.x * blockDim.y) {
      const int a = t % P::TX, b = (t / P::TX) % P::TY, cz = t / (P::TX * P::TY);
      const int64_t gi = i0 - 1 + a, gj = j0 - 1 + b, gk = k - (DIM == 3 ? 1 : 0) + cz;
      if (gi > g.nx || gj > g.ny) continue; // beyond the ring of any live cell
      const double *Uq = U + pidx(g, gi, gj, gk);
      double uq[NV];
#pragma unroll
      for (int v = 0; v < NV; v++) uq[v] = Uq[v * g.pvol];
      const double ir = 1.0 / uq[DENS];
      const double pr = (g.gamma - 1.0) * (uq[ETOT] - 0.5 * (uq[MOMX] * uq[MOMX] + uq[MOMY] * uq[MOMY] +
                                                               uq[MOMZ] * uq[MOMZ]) * ir);
      vt[0][t] = uq[MOMX] * ir;
      vt[1][t] = uq[MOMY] * ir;
      vt[2][t] = uq[MOMZ] * ir;
      vt[3][t] = pr * ir;
    }
    __syncthreads();
  }
  if (i < g.nx && j < g.ny) {
    const int64_t c = (k * g.ny + j) * g.nx + i;
    const int64_t p = pidx(g, i, j, k);
    const double *Uc = U + p;
    double r[NV];
    {
      const int64_t f0 = (k * g.fdim[0][1] + j) * g.fdim[0][0] + i;
      const int64_t f1 = (k * g.fdim[1][1] + j) * g.fdim[1][0] + i;
#pragma unroll
      for (int v = 0; v < NV; v++) {
        r[v] = (G0[v * g.nface[0] + f0] - G0[v * g.nface[0] + f0 + 1]) * g.rdx;
        r[v] += (G1[v * g.nface[1] + f1] - G1[v * g.nface[1] + f1 + g.fdim[1][0]]) * g.rdy;
      }
      if constexpr (DIM == 3) {
        const int64_t f2 = (k * g.fdim[2][1] + j) * g.fdim[2][0] + i;
        const int64_t sz = g.fdim[2][0] * g.fdim[2][1];
#pragma unroll
        for (int v = 0; v < NV; v++) r[v] += (G2[v * g.nface[2] + f2] - G2[v * g.nface[2] + f2 + sz]) * g.rdz;
      }
    }
    if constexpr (EQ == EQ_GLM) glm_sources<DIM, NQ>(Uc, g, i, j, k, c, F0, F1, F2, src, theta[c], r);
    if constexpr (EQ == EQ_NS) viscous<DIM>(vt, g, threadIdx.x, threadIdx.y, Re, Pr, r);

    if (mode == STAGE_EVAL) {
#pragma unroll
      for (int v = 0; v < NV; v++) K[v * g.n + c] = r[v];
    } else if (mode == STAGE_UPDATE) {
#pragma unroll
      for (int v = 0; v < NV; v++) {
        const double u = Uc[v * g.pvol];
        double un = co.g1 * u;
        if (co.use_tmp) {
          const double ut = Utmp[v * g.n + c] + co.delta * u;
          Utmp[v * g.n + c] = ut;
          un += co.g2 * ut;
        }
        if (co.g3 != 0.0) un += co.g3 * Uprev[v * g.pvol + p];
        un += co.betaDt * r[v];
        Unext[v * g.pvol + p] = un;
        Uhat[v * g.n + c] += co.bhatDt * r[v];
      }
    } else { // STAGE_FSAL: K = rhs, Uhat += bhat_fsal dt K, error estimate
      bool hasNan = false;
      double st[NV];
#pragma unroll
      for (int v = 0; v < NV; v++) {
        K[v * g.n + c] = r[v];
        const double uh = Uhat[v * g.n + c] + co.bhatDt * r[v];
        Uhat[v * g.n + c] = uh;
        const double u = Uc[v * g.pvol];
        st[v] = u;
        hasNan = hasNan || isnan(u);
        const double e = (u - uh) / (atol + rtol * fmax(fabs(u), fabs(uh)));
        err += e * e;
      }
      pos = hasNan ? -1.0 : E::positivity(st);
    }
  }
  if (mode == STAGE_FSAL) {
    // deterministic two-level reduction: block partials here, fixed-order sum later
    __shared__ double se[kBlockX * kBlockY / 32], sp[kBlockX * kBlockY / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      err += __shfl_xor_sync(0xffffffffu, err, o);
      pos = fmin(pos, __shfl_xor_sync(0xffffffffu, pos, o));
    }
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    if ((tid & 31) == 0) {
      se[tid >> 5] = err;
      sp[tid >> 5] = pos;
    }
    __syncthreads();
    if (tid == 0) {
      double a = 0.0, b = 1.0;
      for (int w = 0; w < (int)(blockDim.x * blockDim.y / 32); w++) {
        a += se[w];
        b = b > sp[w] ? sp[w] : b;
      }
      const int64_t blk = ((int64_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
      part[2 * blk] = a;
      part[2 * blk + 1] = b;
    }
  }
}

// fixed-order sum of the block partials (one block)
__global__ void __launch_bounds__(1024) finalize_kernel(const double *__restrict__ part,
                                                         int64_t nblk, DevScalars *sc) {
  __shared__ double se[1024], sp[1024];
  double a = 0.0, b = 1.0;
  for (int64_t t = threadIdx.x; t < nblk; t += blockDim.x) {
    a += part[2 * t];
    b = b > part[2 * t + 1] ? part[2 * t + 1] : b;
  }
  se[threadIdx.x] = a;
  sp[threadIdx.x] = b;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      se[threadIdx.x] += se[threadIdx.x + s];
      sp[threadIdx.x] = sp[threadIdx.x] > sp[threadIdx.x + s] ? sp[threadIdx.x + s] : sp[threadIdx.x];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    sc->err = se[0];
    sc->posmin = sp[0];
  }
}

// first stage of a step (RKFSAL_StagePre_K, Numeric_K.H:198-220)
template <int NV>
__global__ void __launch_bounds__(128)
    stage_pre_kernel(double *__restrict__ U1, const double *__restrict__ Uprev,
                     double *__restrict__ Uhat, double *__restrict__ Utmp,
                     const double *__restrict__ K, Grid g, double betaDt, double bhatDt,
                     int use_tmp) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t j = blockIdx.y * (int64_t)blockDim.y + threadIdx.y;
  const int64_t k = blockIdx.z;
  if (i >= g.nx || j >= g.ny) return;
  const int64_t c = (k * g.ny + j) * g.nx + i, p = pidx(g, i, j, k);
#pragma unroll
  for (int v = 0; v < NV; v++) {
    const double up = Uprev[v * g.pvol + p], kk = K[v * g.n + c];
    U1[v * g.pvol + p] = up + betaDt * kk;
    Uhat[v * g.n + c] = up + bhatDt * kk;
    if (use_tmp) Utmp[v * g.n + c] = up;
  }
}

// copy of the interior of one padded buffer into another
template <int NV>
__global__ void __launch_bounds__(128) copy_interior_kernel(double *__restrict__ dst,
                                                            const double *__restrict__ src, Grid g) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t j = blockIdx.y * (int64_t)blockDim.y + threadIdx.y;
  const int64_t k = blockIdx.z;
  if (i >= g.nx || j >= g.ny) return;
  const int64_t p = pidx(g, i, j, k);
#pragma unroll
  for (int v = 0; v < NV; v++) dst[v * g.pvol + p] = src[v * g.pvol + p];
}

// ---------------------------------------------------------------------------
// host launchers
static dim3 cell_grid(const Grid &g) {
  return dim3((unsigned)((g.nx + kBlockX - 1) / kBlockX), (unsigned)((g.ny + kBlockY - 1) / kBlockY),
              (unsigned)g.nz);
}

template <int DIM, int EQ, int NQ>
struct Launch {
  static constexpr int NV = Eos<EQ>::NV;
  static cudaError_t bc(double *U, const Grid &g, cudaStream_t s) {
    const int64_t r = kRad, hx = g.nx + 2 * r, hy = g.ny + 2 * r;
    const int64_t total = 2 * r * g.ny * g.nz + hx * 2 * r * g.nz + (DIM == 3 ? hx * hy * 2 * r : 0);
    const int64_t blocks = (total + 255) / 256;
    bc_fill_kernel<DIM, NV><<<(unsigned)(blocks < 65535 * 16 ? blocks : 65535 * 16), 256, 0, s>>>(U, g);
    return cudaGetLastError();
  }
  static cudaError_t bounds(const double *U, const Grid &g, double *bnd, cudaStream_t s) {
    if constexpr (DIM == 3) {
      constexpr int kZc = 16;   // planes per block
      const dim3 cg = cell_grid(g);
      bounds_march_kernel<EQ><<<dim3(cg.x, cg.y, (unsigned)((g.nz + kZc - 1) / kZc)), dim3(kBlockX, kBlockY), 0, s>>>(
          U, g, kZc, bnd);
    } else {
      bounds_kernel<DIM, EQ><<<cell_grid(g), dim3(kBlockX, kBlockY), 0, s>>>(U, g, bnd);
    }
    return cudaGetLastError();
  }
  static cudaError_t recon(const double *U, const CUtensorMap *umap, const Grid &g, const DevStencil *S,
                           int wantInd, double *const *F, float *const *W, double *src, uint8_t *status,
                           double2 *lamvel, double *bnd, DevScalars *sc, cudaStream_t s) {
    if constexpr (DmmaShape<DIM, EQ, NQ>::NT > 7) {
      // more rows than the DMMA kernels hold (3D GLM-MHD, three points)
      using R = RowsShape<DIM, EQ, NQ>;
      static const cudaError_t attrR = cudaFuncSetAttribute(
          recon_rows_kernel<DIM, EQ, NQ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)R::BYTES);
      if (attrR != cudaSuccess) return attrR;
      recon_rows_kernel<DIM, EQ, NQ><<<(unsigned)((g.n + R::CELLS - 1) / R::CELLS), dim3(R::CELLS, NV), R::BYTES, s>>>(
          U, g, S, wantInd, F[0], F[1], F[2], W[0], W[1], W[2], src, status, lamvel, bnd);
      return cudaGetLastError();
    } else {
    // (3D with three Gauss points keeps the global-load kernel: its 54 rows need
    // more accumulator registers than two 256-thread blocks per SM leave; so does
    // GLM-MHD in 3D, whose nine halo tiles would not leave room for two blocks, and
    // with three points in 2D)
    if constexpr ((NV == 5 && (DIM == 2 || NQ == 2)) || (NV == 9 && DIM == 2 && NQ == 2)) {
      if (umap) {
        // the halo tiles staged by TMA (five variables: Euler, Navier-Stokes, SR)
        using D = DmmaTile<DIM>;
        using L = DmmaTmaSmem<DIM, EQ, NQ>;
        static const cudaError_t attr = cudaFuncSetAttribute(
            recon_tma_kernel<DIM, EQ, NQ>, cudaFuncAttributeMaxDynamicSharedMemorySize, L::BYTES);
        if (attr != cudaSuccess) return attr;
        const dim3 grid((unsigned)((g.nx + D::BX - 1) / D::BX), (unsigned)((g.ny + D::BY - 1) / D::BY),
                        (unsigned)((g.nz + D::BZ - 1) / D::BZ));
        recon_tma_kernel<DIM, EQ, NQ><<<grid, D::THREADS, L::BYTES, s>>>(
            *umap, g, S, wantInd, F[0], F[1], F[2], W[0], W[1], W[2], src, status, lamvel, bnd, sc);
        return cudaGetLastError();
      }
    }
    recon_kernel<DIM, EQ, NQ><<<cell_grid(g), dim3(kBlockX, kBlockY), 0, s>>>(
        U, g, S, wantInd, F[0], F[1], F[2], W[0], W[1], W[2], src, status, lamvel, bnd);
    return cudaGetLastError();
    }
  }
  static cudaError_t flag(const double *U, const Grid &g, float *const *W, double *const *F,
                          const double *theta, uint8_t *flag, DevScalars *sc, double thr, cudaStream_t s) {
    flag_kernel<DIM, EQ, NQ><<<cell_grid(g), dim3(kBlockX, kBlockY), 0, s>>>(U, g, W[0], W[1], W[2], F[0], F[1],
                                                                          F[2], theta, flag, sc, thr);
    return cudaGetLastError();
  }
  static cudaError_t compact(const Grid &g, int mode, const uint8_t *flag, uint8_t *wset,
                             const uint8_t *status, uint8_t *applied, double *theta, uint32_t *heavy,
                             const double2 *lamvel, DevScalars *sc, const JudgeArgs &jd, cudaStream_t s) {
    compact_kernel<DIM, EQ><<<(unsigned)((g.n + 255) / 256), 256, 0, s>>>(g, mode, flag, wset, status, applied,
                                                                           theta, heavy, lamvel, sc, jd);
    return cudaGetLastError();
  }
  static cudaError_t heavy(const double *U, const Grid &g, const DevStencil *S, double *theta,
                           double *const *F, double *src, const uint32_t *heavy, const double *bnd,
                           DevScalars *sc, const JudgeArgs &jd, int heavy_blocks, cudaStream_t s) {
    // set once per process (a function-local static is initialised once, also when
    // several host threads drive solvers)
    static const cudaError_t attr = cudaFuncSetAttribute(
        heavy_var_kernel<DIM, EQ, NQ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)HeavyShape<DIM, EQ, NQ>::BYTES);
    if (attr != cudaSuccess) return attr;
    heavy_var_kernel<DIM, EQ, NQ><<<heavy_blocks, dim3(HeavyShape<DIM, EQ, NQ>::CELLS, NV), HeavyShape<DIM, EQ, NQ>::BYTES, s>>>(
        U, g, S, theta, F[0], F[1], F[2], src, heavy, bnd, sc, jd);
    return cudaGetLastError();
  }
  template <bool SAME>
  static void riemann_dirs(double *const *F, double *const *G, const Grid &g, DevScalars *sc, cudaStream_t s) {
#pragma unroll 1
    for (int d = 0; d < DIM; d++) {
      // 32 consecutive faces of an (x, y) face plane per block (rows of the x faces
      // hold nx + 1 faces, which would leave a nearly empty block per row), NQF
      // points along threadIdx.y
      const dim3 grid((unsigned)((g.fdim[d][0] * g.fdim[d][1] + 31) / 32), 1u, (unsigned)g.fdim[d][2]);
      const dim3 blk(32, Cfg<DIM, EQ, NQ>::NQF);
      if (d == 0) riemann_kernel<DIM, EQ, 0, NQ, SAME><<<grid, blk, 0, s>>>(F[0], G[0], g, sc);
      if (d == 1) riemann_kernel<DIM, EQ, 1, NQ, SAME><<<grid, blk, 0, s>>>(F[1], G[1], g, sc);
      if (DIM == 3 && d == 2)
        riemann_kernel<DIM, EQ, (DIM == 3 ? 2 : 1), NQ, SAME><<<grid, blk, 0, s>>>(F[2], G[2], g, sc);
    }
  }
  static cudaError_t riemann(double *const *F, double *const *G, const Grid &g, DevScalars *sc, bool same,
                             cudaStream_t s) {
    if (same) riemann_dirs<true>(F, G, g, sc, s);
    else riemann_dirs<false>(F, G, g, sc, s);
    return cudaGetLastError();
  }
  static cudaError_t stage(const StageArgs &a, const Grid &g, cudaStream_t s) {
    const dim3 grid = cell_grid(g);
    stage_kernel<DIM, EQ, NQ><<<grid, dim3(kBlockX, kBlockY), 0, s>>>(
        a.U, a.Unext, a.Uprev, a.Uhat, a.Utmp, a.K, g, a.G[0], a.G[1], a.G[2], a.F[0], a.F[1],
        a.F[2], a.src, a.theta, a.mode, a.co, a.Re, a.Pr, a.atol, a.rtol, a.part);
    if (a.mode == STAGE_FSAL) {
      const int64_t nblk = (int64_t)grid.x * grid.y * grid.z;
      finalize_kernel<<<1, 1024, 0, s>>>(a.part, nblk, a.sc);
    }
    return cudaGetLastError();
  }
  static cudaError_t stage_pre(double *U1, const double *Uprev, double *Uhat, double *Utmp,
                               const double *K, const Grid &g, double betaDt, double bhatDt,
                               int use_tmp, cudaStream_t s) {
    stage_pre_kernel<NV><<<cell_grid(g), dim3(kBlockX, kBlockY), 0, s>>>(U1, Uprev, Uhat, Utmp, K, g,
                                                                          betaDt, bhatDt, use_tmp);
    return cudaGetLastError();
  }
  static cudaError_t copy(double *dst, const double *src, const Grid &g, cudaStream_t s) {
    copy_interior_kernel<NV><<<cell_grid(g), dim3(kBlockX, kBlockY), 0, s>>>(dst, src, g);
    return cudaGetLastError();
  }
};

// host: B fragments of the FP64 MMA from the [cell][row] linear weights
void fill_dmma_weights(DevStencil &S, int nrows) {
  // all stencil cells but the last (added in the kernel's epilogue)
  const int C = S.w.n_cells - 1, nt = (nrows + 7) / 8, nk = (C + 3) / 4;
  std::memset(S.dmma_b, 0, sizeof(S.dmma_b));
  if (nk * nt * 32 > kDmmaMaxB) return;  // more rows than the DMMA kernels take (they are not used)
  for (int ks = 0; ks < nk; ks++)
    for (int t = 0; t < nt; t++)
      for (int l = 0; l < 32; l++) {
        const int c = ks * 4 + (l & 3), n = t * 8 + (l >> 2);
        if (c < C && n < nrows) S.dmma_b[(ks * nt + t) * 32 + l] = S.lin[c * nrows + n];
      }
}

int64_t stage_blocks(const Grid &g) {
  const dim3 gr = cell_grid(g);
  return (int64_t)gr.x * gr.y * gr.z;
}

// one instantiation per (dimension, equations, Gauss points): 2 points for both
// dimensions, 3 points for 2D and for 3D Euler / Navier-Stokes / GLM-MHD (not SR);
// the grid's nq selects
#define KFVM_DISPATCH(DIM_, EQ_, CALL)                                                  \
  do {                                                                                \
    if (g.nq == 2) {                                                                  \
      if ((DIM_) == 2 && (EQ_) == EQ_HYDRO) return Launch<2, EQ_HYDRO, 2>::CALL;      \
      if ((DIM_) == 3 && (EQ_) == EQ_HYDRO) return Launch<3, EQ_HYDRO, 2>::CALL;      \
      if ((DIM_) == 2 && (EQ_) == EQ_NS) return Launch<2, EQ_NS, 2>::CALL;            \
      if ((DIM_) == 3 && (EQ_) == EQ_NS) return Launch<3, EQ_NS, 2>::CALL;            \
      if ((DIM_) == 2 && (EQ_) == EQ_GLM) return Launch<2, EQ_GLM, 2>::CALL;          \
      if ((DIM_) == 3 && (EQ_) == EQ_GLM) return Launch<3, EQ_GLM, 2>::CALL;          \
      if ((DIM_) == 2 && (EQ_) == EQ_SR) return Launch<2, EQ_SR, 2>::CALL;            \
      if ((DIM_) == 3 && (EQ_) == EQ_SR) return Launch<3, EQ_SR, 2>::CALL;            \
    } else if (g.nq == 3 && (DIM_) == 2) {                                            \
      if ((EQ_) == EQ_HYDRO) return Launch<2, EQ_HYDRO, 3>::CALL;                     \
      if ((EQ_) == EQ_NS) return Launch<2, EQ_NS, 3>::CALL;                           \
      if ((EQ_) == EQ_GLM) return Launch<2, EQ_GLM, 3>::CALL;                         \
      if ((EQ_) == EQ_SR) return Launch<2, EQ_SR, 3>::CALL;                           \
    } else if (g.nq == 3 && (DIM_) == 3) {                                            \
      if ((EQ_) == EQ_HYDRO) return Launch<3, EQ_HYDRO, 3>::CALL;                     \
      if ((EQ_) == EQ_NS) return Launch<3, EQ_NS, 3>::CALL;                           \
      if ((EQ_) == EQ_GLM) return Launch<3, EQ_GLM, 3>::CALL;                         \
    }                                                                                 \
    return cudaErrorInvalidValue;                                                     \
  } while (0)

// host-order interior (variable, k, j, i; i fastest) <-> padded device layout:
// one thread per cell of a row, rows (j, k) and variables over the grid
template <bool TO_PADDED>
__global__ void __launch_bounds__(256) interior_kernel(double *__restrict__ Up, double *__restrict__ flat, Grid g) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= g.nx) return;
  const int64_t j = blockIdx.y, k = blockIdx.z % g.nz, v = blockIdx.z / g.nz;
  const int64_t f = v * g.n + (k * g.ny + j) * g.nx + i;
  const int64_t p = v * g.pvol + pidx(g, i, j, k);
  if (TO_PADDED) Up[p] = flat[f];
  else flat[f] = Up[p];
}

__global__ void __launch_bounds__(256) fill_kernel(double *__restrict__ p, int64_t n, double val) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
    p[t] = val;
}

// accuracy probe of rcp_nr against the IEEE reciprocal and quotient
__global__ void __launch_bounds__(256) rcp_probe_kernel(int64_t n, uint64_t seed, unsigned long long *out) {
  unsigned long long worst = 0, worstQ = 0;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t h = mix64(seed ^ (uint64_t)t), h2 = mix64(h);
    // mantissa from the hash, exponent uniform in [-300, 300], random sign
    const double m = 1.0 + (double)(h >> 12) * 0x1.0p-52;
    const int ex = (int)(h2 % 601) - 300;
    const double y = ((h2 >> 32) & 1 ? -1.0 : 1.0) * scalbn(m, ex);
    const double x = 1.0 + (double)(h2 >> 12) * 0x1.0p-52;
    const double r = rcp_nr(y), q = 1.0 / y;
    const long long d = __double_as_longlong(r) - __double_as_longlong(q);
    const unsigned long long du = (unsigned long long)(d < 0 ? -d : d);
    worst = du > worst ? du : worst;
    const double rel = fabs(x * r - x / y) / fabs(x / y);
    const unsigned long long rq = (unsigned long long)__double_as_longlong(rel);
    worstQ = rq > worstQ ? rq : worstQ;
  }
  atomicMax(&out[0], worst);
  atomicMax(&out[1], worstQ);
}

cudaError_t launch_rcp_probe(int64_t n, uint64_t seed, unsigned long long *out, cudaStream_t s) {
  rcp_probe_kernel<<<148 * 4, 256, 0, s>>>(n, seed, out);
  return cudaGetLastError();
}

cudaError_t launch_interior(double *Up, double *flat, const Grid &g, int nv, bool toPadded, cudaStream_t s) {
  const dim3 grid((unsigned)((g.nx + 255) / 256), (unsigned)g.ny, (unsigned)(g.nz * nv));
  if (toPadded) interior_kernel<true><<<grid, 256, 0, s>>>(Up, flat, g);
  else interior_kernel<false><<<grid, 256, 0, s>>>(Up, flat, g);
  return cudaGetLastError();
}

cudaError_t launch_fill(double *p, int64_t n, double val, cudaStream_t s) {
  const int64_t blocks = std::min<int64_t>((n + 255) / 256, 148 * 16);
  fill_kernel<<<(unsigned)std::max<int64_t>(blocks, 1), 256, 0, s>>>(p, n, val);
  return cudaGetLastError();
}

cudaError_t launch_bc(int dim, int eq, double *U, const Grid &g, cudaStream_t s) {
  KFVM_DISPATCH(dim, eq, bc(U, g, s));
}
cudaError_t launch_bounds(int dim, int eq, const double *U, const Grid &g, double *bnd, cudaStream_t s) {
  KFVM_DISPATCH(dim, eq, bounds(U, g, bnd, s));
}

cudaError_t launch_recon(int dim, int eq, const double *U, const CUtensorMap *umap, const Grid &g,
                         const DevStencil *S, int wantInd, double *const *F, float *const *W, double *src,
                         uint8_t *status, double2 *lamvel, double *bnd, DevScalars *sc, cudaStream_t s) {
  KFVM_DISPATCH(dim, eq, recon(U, umap, g, S, wantInd, F, W, src, status, lamvel, bnd, sc, s));
}
cudaError_t launch_flag(int dim, int eq, const double *U, const Grid &g, float *const *W, double *const *F,
                        const double *theta, uint8_t *flag, DevScalars *sc, double thr,
                        cudaStream_t s) {
  KFVM_DISPATCH(dim, eq, flag(U, g, W, F, theta, flag, sc, thr, s));
}
cudaError_t launch_compact(int dim, int eq, const Grid &g, int mode, const uint8_t *flag, uint8_t *wset,
                           const uint8_t *status, uint8_t *applied, double *theta, uint32_t *heavy,
                           const double2 *lamvel, DevScalars *sc, const JudgeArgs &jd, cudaStream_t s) {
  KFVM_DISPATCH(dim, eq, compact(g, mode, flag, wset, status, applied, theta, heavy, lamvel, sc, jd, s));
}
cudaError_t launch_heavy(int dim, int eq, const double *U, const Grid &g, const DevStencil *S,
                         double *theta, double *const *F, double *src, const uint32_t *heavy,
                         const double *bnd, DevScalars *sc, const JudgeArgs &jd, int heavy_blocks,
                         cudaStream_t s) {
  KFVM_DISPATCH(dim, eq, heavy(U, g, S, theta, F, src, heavy, bnd, sc, jd, heavy_blocks, s));
}
cudaError_t launch_riemann(int dim, int eq, double *const *F, double *const *G, const Grid &g,
                           DevScalars *sc, bool same, cudaStream_t s) {
  KFVM_DISPATCH(dim, eq, riemann(F, G, g, sc, same, s));
}
cudaError_t launch_stage(int dim, int eq, const StageArgs &a, const Grid &g, cudaStream_t s) {
  KFVM_DISPATCH(dim, eq, stage(a, g, s));
}
cudaError_t launch_stage_pre(int dim, int eq, double *U1, const double *Uprev, double *Uhat,
                             double *Utmp, const double *K, const Grid &g, double betaDt,
                             double bhatDt, int use_tmp, cudaStream_t s) {
  KFVM_DISPATCH(dim, eq, stage_pre(U1, Uprev, Uhat, Utmp, K, g, betaDt, bhatDt, use_tmp, s));
}
cudaError_t launch_copy(int dim, int eq, double *dst, const double *src, const Grid &g,
                        cudaStream_t s) {
  KFVM_DISPATCH(dim, eq, copy(dst, src, g, s));
}

} // namespace kfvm
