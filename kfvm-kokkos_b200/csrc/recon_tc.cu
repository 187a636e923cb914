// recon_tc.cu -- the linear reconstruction contraction on the tcgen05 tensor cores
// (the FP32 form: 3xTF32 products, FP32 accumulation in tensor memory).
//
// Same outputs as recon_kernel (KernelLinearRecon_K, src/stencil/Stencil_K.H:56-119
// of the reference, plus the KXRCF indicator and the positivity pre-check), with
// the sum over stencil cells done as one MMA tile per block of 128 cells:
//
//   D[m][n] = sum_k A[m][k] B[k][n]      m: cell of the block (TMEM lane)
//                                        k: stencil cell (33 in 3D, 13 in 2D, zero padded)
//                                        n: weight row (face points, interior points)
//   A[m][k] = u(cell m + offset k) - u(cell m)   (per variable; FP64 difference, FP32 value)
//
// Reconstructing the deviation from the cell average (the weights of every row sum
// to one) keeps the FP32 rounding relative to the local variation, not to the
// state.  Each FP32 operand x is split as x = hi + lo with hi = tf32(x),
// lo = tf32(x - hi), and D accumulates lo_A hi_B + hi_A lo_B + hi_A hi_B, which
// carries about 21 significant bits per product.  The face state is then
// u(cell) + D in FP64; positivity checks, the indicator and everything after the
// reconstruction stay FP64.
//
// Per block (256 threads, two per cell = per row of the tile, 128 cells):
//   warp 0 allocates the TMEM columns (variables x N, rounded to a power of two)
//   the split weights (B, hi and lo) and the limiter footprint tile are loaded,
//     and the limiter bounds of each cell are computed once
//   per variable: the two threads of a row write its A row (hi and lo, half of
//     the K chunks each) into shared memory in the canonical K-major no-swizzle
//     layout (8-row x 16-byte core matrices); thread 0 issues 3 MMAs per K step
//     of 8 into the variable's TMEM columns and commits them to an mbarrier; the
//     next variable waits for that mbarrier before it overwrites the A buffer
//   epilogue: each warp reads its 32 lanes (tcgen05.ld 32x32b), the two threads
//     of a row take half of its face / interior points each, add the cell
//     average in FP64 and write face states and indicators; the in-bounds test
//     and the GLM speeds of a cell are combined in shared memory
// Every mbarrier wait is bounded (iteration count and a 1 s global-timer limit);
// on timeout the block records DevScalars::fault, frees its TMEM and returns.
// Shared memory per block is sized so that at most 512 / columns blocks are
// resident on an SM, so a TMEM allocation never waits for another block.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <type_traits>

#include "kernels.cuh"
#include "launch.h"
#include "recon_common.cuh"
#include "tcgen05.cuh"

namespace kfvm {

// Two threads per tile row (cell): threads 0..127 are part 0, 128..255 part 1;
// warp w reads TMEM lanes 32 (w % 4) .. +31, so both parts reach every row.
constexpr int kTcParts = 2;
constexpr int kTcThreads = 128 * kTcParts;

template <int DIM, int EQ>
struct TcShape {
  using T = Cfg<DIM, EQ>;
  static constexpr int NR = LinRows<DIM, EQ>::NROWS;
  static constexpr int NP = DIM == 2 ? 16 : 32;       // MMA N (M = 128: N multiple of 16)
  static constexpr int KP = DIM == 2 ? 16 : 40;       // stencil cells padded to K steps of 8
  static constexpr int NKS = KP / 8;
  static constexpr int NCH = KP / 4;                  // 16-byte core-matrix columns along K
  // epilogue rows per part, even (TMEM loads of column pairs)
  static constexpr int RPP = (((NR + kTcParts - 1) / kTcParts) + 1) / 2 * 2;
  static constexpr int COLS_USED = T::NV * NP;
  static constexpr int COLS = COLS_USED <= 128 ? 128 : (COLS_USED <= 256 ? 256 : 512);
  static constexpr int MAX_RES = 512 / COLS;          // blocks per SM that fit in TMEM
  static constexpr int A_CH = 128 * 16;               // one K chunk of A: 128 rows x 16 B
  static constexpr int A_PART = NCH * A_CH;           // hi or lo part of A
  static constexpr int B_CH = NP * 16;
  static constexpr int B_PART = NCH * B_CH;
  static constexpr int OFF_B = 2 * A_PART;
  static constexpr int OFF_TILE = OFF_B + 2 * B_PART;
  static constexpr int OFF_BD = OFF_TILE + 6 * PosTile<DIM>::N * (int)sizeof(double); // bounds [3][128]
  static constexpr int OFF_RED = OFF_BD + 3 * 128 * (int)sizeof(double);              // lam, vel [2][128], in-bounds [128]
  static constexpr int OFF_BAR = OFF_RED + 2 * 128 * 8 + 128 * 4;
  static constexpr int USED = OFF_BAR + 16;
  // 228 KB of shared memory per SM: MAX_RES + 1 blocks of FLOOR bytes do not fit
  static constexpr int FLOOR = 233472 / (MAX_RES + 1) + 256;
  static constexpr int SMEM = USED > FLOOR ? USED : FLOOR;
  static_assert(NR <= NP, "weight rows exceed the MMA N");
  static_assert(kTcParts * RPP <= NP, "epilogue rows beyond the MMA N");
  static_assert(T::C <= KP, "stencil exceeds the MMA K");
  static_assert(KP <= kTcMaxK && NP <= kTcMaxN, "B table too small");
  static_assert(SMEM <= 227 * 1024, "shared memory per block");
  static_assert(kBlockX * kBlockY == 128, "one tile row per cell");
  static_assert(OFF_BAR % 8 == 0 && OFF_BD % 8 == 0, "alignment");
};

// ---------------------------------------------------------------------------
template <int DIM, int EQ>
__global__ void __launch_bounds__(kTcThreads, 2)
    recon_tc_kernel(const double *__restrict__ U, Grid g, const DevStencil *__restrict__ S, int wantInd,
                    double *__restrict__ F0, double *__restrict__ F1, double *__restrict__ F2,
                    float *__restrict__ W0, float *__restrict__ W1, float *__restrict__ W2,
                    double *__restrict__ src, uint8_t *__restrict__ status, double2 *__restrict__ lamvel,
                    double *__restrict__ bnd, DevScalars *__restrict__ sc) {
  using T = Cfg<DIM, EQ>;
  using Sh = TcShape<DIM, EQ>;
  constexpr int NV = T::NV;
  extern __shared__ __align__(128) uint8_t smem[];
  double(*tile)[PosTile<DIM>::N] = reinterpret_cast<double(*)[PosTile<DIM>::N]>(smem + Sh::OFF_TILE);
  double(*sBd)[128] = reinterpret_cast<double(*)[128]>(smem + Sh::OFF_BD);
  unsigned long long *sLam = reinterpret_cast<unsigned long long *>(smem + Sh::OFF_RED);
  unsigned long long *sVel = sLam + 128;
  int *sIn = reinterpret_cast<int *>(smem + Sh::OFF_RED + 2 * 128 * 8);
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + Sh::OFF_BAR);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(smem + Sh::OFF_BAR + 8);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int quarter = warp & 3, part = warp >> 2;
  const int row = quarter * 32 + lane;     // tile row = TMEM lane = cell (lane, quarter) of the block
  const int tid = threadIdx.x;
  const int64_t i = blockIdx.x * (int64_t)kBlockX + lane;
  const int64_t j = blockIdx.y * (int64_t)kBlockY + quarter;
  const int64_t k = blockIdx.z;
  const bool live = i < g.nx && j < g.ny;
  const uint32_t barA = smem_u32(bar);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"((uint32_t)Sh::COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(barA) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // B operand (split weights, already in core-matrix order) and the limiter tile
  {
    const float4 *bh = reinterpret_cast<const float4 *>(S->tcw[0]);
    const float4 *bl = reinterpret_cast<const float4 *>(S->tcw[1]);
    float4 *dh = reinterpret_cast<float4 *>(smem + Sh::OFF_B);
    float4 *dl = reinterpret_cast<float4 *>(smem + Sh::OFF_B + Sh::B_PART);
    for (int t = tid; t < Sh::B_PART / 16; t += kTcThreads) {
      dh[t] = bh[t];
      dl[t] = bl[t];
    }
  }
  {
    // the footprint tile, filled by all threads (pos_tile_fill strides by blockDim)
    using P = PosTile<DIM>;
    const int64_t i0 = blockIdx.x * (int64_t)kBlockX, j0 = blockIdx.y * (int64_t)kBlockY;
    for (int t = tid; t < P::N; t += kTcThreads) {
      const int a = t % P::TX, b = (t / P::TX) % P::TY, cz = t / (P::TX * P::TY);
      const int64_t gi = i0 - 1 + a, gj = j0 - 1 + b, gk = k - (DIM == 3 ? 1 : 0) + cz;
      if (gi > g.nx || gj > g.ny) continue;
      const double *Uq = U + pidx(g, gi, gj, gk);
      double st[NV];
#pragma unroll
      for (int v = 0; v < NV; v++) st[v] = Uq[v * g.pvol];
      const double ir = 1.0 / st[DENS];
      const double ei = Eos<EQ>::eint_r(st, ir);
      tile[0][t] = st[DENS];
      tile[1][t] = ei;
      tile[2][t] = sqrt(g.gamma * ((g.gamma - 1.0) * ei) * ir);
      tile[3][t] = st[MOMX] * ir;
      tile[4][t] = st[MOMY] * ir;
      tile[5][t] = st[MOMZ] * ir;
    }
  }
  if (part == 0) {
    sIn[row] = 1;
    sLam[row] = 0ull;
    sVel[row] = 0ull;
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  if (part == 0 && live) {
    const PosBounds bd = pos_bounds_tile<DIM, EQ>(tile, lane, quarter);
    sBd[0][row] = bd.minDens;
    sBd[1][row] = bd.maxDens;
    sBd[2][row] = bd.minEint;
    const int64_t c = (k * g.ny + j) * g.nx + i;
    bnd[c] = bd.minDens;
    bnd[g.n + c] = bd.maxDens;
    bnd[2 * g.n + c] = bd.minEint;
  }

  const double *Uc = U + pidx(g, live ? i : 0, live ? j : 0, k);
  const uint32_t aHi = smem_u32(smem), aLo = aHi + Sh::A_PART;
  const uint32_t bHi = smem_u32(smem + Sh::OFF_B), bLo = bHi + Sh::B_PART;
  constexpr uint32_t idesc = tf32_idesc<Sh::NP>();

  bool ok = true;
#pragma unroll 1
  for (int v = 0; v < NV; v++) {
    if (v > 0) ok = mbar_wait(barA, (uint32_t)(v - 1) & 1u);
    if (!__syncthreads_and(ok)) break;
    // this thread's share of the A row for variable v: chunks part, part + 2, ...
    const double *Uv = Uc + v * g.pvol;
    const double ucv = live ? Uv[0] : 0.0;
#pragma unroll
    for (int ch = part; ch < Sh::NCH; ch += kTcParts) {
      uint32_t hi[4], lo[4];
#pragma unroll
      for (int t = 0; t < 4; t++) {
        const int c = ch * 4 + t;
        float d = 0.0f;
        if (c < T::C && live) d = (float)(__ldg(Uv + g.loff[c]) - ucv);
        hi[t] = to_tf32(d);
        lo[t] = to_tf32(d - __uint_as_float(hi[t]));
      }
      st_shared_v4(aHi + ch * Sh::A_CH + row * 16, hi);
      st_shared_v4(aLo + ch * Sh::A_CH + row * 16, lo);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t d = tmem + (uint32_t)(v * Sh::NP);
#pragma unroll
      for (int s = 0; s < Sh::NKS; s++) {
        const uint64_t ah = umma_desc(aHi + 2 * s * Sh::A_CH, Sh::A_CH, 128);
        const uint64_t al = umma_desc(aLo + 2 * s * Sh::A_CH, Sh::A_CH, 128);
        const uint64_t bh = umma_desc(bHi + 2 * s * Sh::B_CH, Sh::B_CH, 128);
        const uint64_t bl = umma_desc(bLo + 2 * s * Sh::B_CH, Sh::B_CH, 128);
        mma_tf32(d, al, bh, idesc, s > 0);
        mma_tf32(d, ah, bl, idesc, 1);
        mma_tf32(d, ah, bh, idesc, 1);
      }
      mma_commit(barA);
    }
  }
  if (ok) ok = mbar_wait(barA, (uint32_t)(NV - 1) & 1u);
  if (__syncthreads_and(ok)) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    PosBounds bd;
    bd.minDens = sBd[0][row];
    bd.maxDens = sBd[1][row];
    bd.minEint = sBd[2][row];
    double uc[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) uc[v] = live ? Uc[v * g.pvol] : 0.0;
    const uint32_t lanes = (uint32_t)(quarter * 32) << 16;
    const int64_t c = (k * g.ny + j) * g.nx + i;
    bool inside = true;
    double lam = 0.0, vel = 0.0;
    // the rows of each part are known at compile time (face, direction, point)
    auto epilogue = [&](auto partTag) {
      constexpr int PART = decltype(partTag)::value;
      constexpr int R0 = PART * Sh::RPP;
#pragma unroll
      for (int rp = 0; rp < Sh::RPP; rp += 2) {
        float a0[NV], a1[NV];
#pragma unroll
        for (int v = 0; v < NV; v++) tmem_ld2(tmem + lanes + (uint32_t)(v * Sh::NP + R0 + rp), a0[v], a1[v]);
        if (live) {
#pragma unroll
          for (int e = 0; e < 2; e++) {
            const int rw = R0 + rp + e;
            if (rw < Sh::NR) {
              double st[NV];
#pragma unroll
              for (int v = 0; v < NV; v++) st[v] = uc[v] + (double)(e ? a1[v] : a0[v]);
              // pos_inside, with the internal energy kept for the indicator's pressure
              const double ei = Eos<EQ>::eint(st);
              inside = inside && st[DENS] > bd.minDens && st[DENS] < bd.maxDens && ei > bd.minEint;
              if (rw < T::NF * T::NQF) {
                const int f = rw / T::NQF, q = rw % T::NQF, d = f >> 1;
                double *Fd = d == 0 ? F0 : (d == 1 ? F1 : F2);
                const int64_t a = face_slot_addr(g, f, i, j, k, q, 0, T::NQF, NV);
                const int64_t nf = g.nface[d];
#pragma unroll
                for (int v = 0; v < NV; v++) Fd[a + v * nf] = st[v];
                if (wantInd)
                  (d == 0 ? W0 : (d == 1 ? W1 : W2))[face_slot_addr(g, f, i, j, k, q, 0, T::NQF, 1)] =
                      Eos<EQ>::template weno_store<DIM>(g.gamma, st[DENS], (g.gamma - 1.0) * ei);
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
    };
    static_assert(kTcParts == 2, "epilogue specialised for two parts");
    if (part == 0) epilogue(std::integral_constant<int, 0>{});
    else epilogue(std::integral_constant<int, 1>{});
    // combine the two parts of each cell
    if (live && !inside) atomicAnd(&sIn[row], 0);
    if constexpr (T::SRC) {
      if (live) {
        if (lam >= 0.0) atomicMax(&sLam[row], (unsigned long long)__double_as_longlong(lam));
        if (vel >= 0.0) atomicMax(&sVel[row], (unsigned long long)__double_as_longlong(vel));
      }
    }
    __syncthreads();
    if (live && part == 0) {
      if constexpr (T::SRC)
        lamvel[c] = make_double2(__longlong_as_double((long long)sLam[row]), __longlong_as_double((long long)sVel[row]));
      status[c] = sIn[row] ? 1 : 0;
    }
  } else if (tid == 0) {
    atomicExch(&sc->fault, 1u);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)Sh::COLS)
                 : "memory");
}

// Self-test of the bounded wait: one block waits on an mbarrier that nothing
// arrives on, with the given limit, and records whether it gave up and how long
// it waited.  The kernel always returns.
__global__ void wait_probe_kernel(uint64_t limit_ns, unsigned long long *out) {
  __shared__ uint64_t bar;
  const uint32_t b = smem_u32(&bar);
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  const uint64_t t0 = global_ns();
  const bool done = mbar_wait(b, 0u, limit_ns);
  out[0] = done ? 0ull : 1ull;
  out[1] = global_ns() - t0;
}

cudaError_t launch_wait_probe(uint64_t limit_ns, unsigned long long *out, cudaStream_t s) {
  wait_probe_kernel<<<1, 1, 0, s>>>(limit_ns, out);
  return cudaGetLastError();
}

template <int DIM, int EQ>
static cudaError_t recon_tc_launch(const double *U, const Grid &g, const DevStencil *S, int wantInd,
                                   double *const *F, float *const *W, double *src, uint8_t *status,
                                   double2 *lamvel, double *bnd, DevScalars *sc, cudaStream_t s) {
  using Sh = TcShape<DIM, EQ>;
  static bool attr = false; // the attribute is per function and process-wide
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(recon_tc_kernel<DIM, EQ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         Sh::SMEM);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const dim3 grid((unsigned)((g.nx + kBlockX - 1) / kBlockX), (unsigned)((g.ny + kBlockY - 1) / kBlockY),
                  (unsigned)g.nz);
  recon_tc_kernel<DIM, EQ><<<grid, kTcThreads, Sh::SMEM, s>>>(
      U, g, S, wantInd, F[0], F[1], F[2], W[0], W[1], W[2], src, status, lamvel, bnd, sc);
  return cudaGetLastError();
}

cudaError_t launch_recon_tc(int dim, int eq, const double *U, const Grid &g, const DevStencil *S, int wantInd,
                            double *const *F, float *const *W, double *src, uint8_t *status, double2 *lamvel,
                            double *bnd, DevScalars *sc, cudaStream_t s) {
  if (dim == 2) {
    if (eq == EQ_GLM) return recon_tc_launch<2, EQ_GLM>(U, g, S, wantInd, F, W, src, status, lamvel, bnd, sc, s);
    if (eq == EQ_NS) return recon_tc_launch<2, EQ_NS>(U, g, S, wantInd, F, W, src, status, lamvel, bnd, sc, s);
    return recon_tc_launch<2, EQ_HYDRO>(U, g, S, wantInd, F, W, src, status, lamvel, bnd, sc, s);
  }
  if (eq == EQ_GLM) return recon_tc_launch<3, EQ_GLM>(U, g, S, wantInd, F, W, src, status, lamvel, bnd, sc, s);
  if (eq == EQ_NS) return recon_tc_launch<3, EQ_NS>(U, g, S, wantInd, F, W, src, status, lamvel, bnd, sc, s);
  return recon_tc_launch<3, EQ_HYDRO>(U, g, S, wantInd, F, W, src, status, lamvel, bnd, sc, s);
}

// host: W = hi + lo split of the [cell][row] linear weights into the B layout
void fill_tc_weights(DevStencil &S, int dim, int nrows) {
  const int np = dim == 2 ? 16 : 32, C = S.w.n_cells;
  auto tf32 = [](double x) {
    float f = (float)x;
    uint32_t b;
    std::memcpy(&b, &f, 4);
    b = (b + 0x1000u) & 0xFFFFE000u; // round to nearest, ties away, on the magnitude
    std::memcpy(&f, &b, 4);
    return f;
  };
  std::memset(S.tcw, 0, sizeof(S.tcw));
  for (int c = 0; c < C; c++)
    for (int n = 0; n < nrows; n++) {
      const double w = S.lin[c * nrows + n];
      const float hi = tf32(w);
      const float lo = tf32(w - (double)hi);
      const int idx = ((c / 4) * np + n) * 4 + (c % 4);
      S.tcw[0][idx] = hi;
      S.tcw[1][idx] = lo;
    }
}

} // namespace kfvm
