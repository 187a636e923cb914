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
//   the split weights (B, hi and lo) are loaded and each cell's limiter bounds
//     read (bounds_kernel computed them)
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
#include "tma.cuh"

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
  static constexpr int OFF_BD = OFF_B + 2 * B_PART;   // limiter bounds of the block's cells [3][128]
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
  if (part == 0) {
    sIn[row] = 1;
    sLam[row] = 0ull;
    sVel[row] = 0ull;
    if (live) {
      // limiter bounds of the cell (bounds_kernel)
      const int64_t c = (k * g.ny + j) * g.nx + i;
      sBd[0][row] = bnd[c];
      sBd[1][row] = bnd[g.n + c];
      sBd[2][row] = bnd[2 * g.n + c];
    }
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;

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
        tmem_ld2_n<NV>(tmem + lanes + (uint32_t)(R0 + rp), (uint32_t)Sh::NP, a0, a1);
        if (live) {
#pragma unroll
          for (int e = 0; e < 2; e++) {
            const int rw = R0 + rp + e;
            if (rw < Sh::NR) {
              double st[NV];
#pragma unroll
              for (int v = 0; v < NV; v++) st[v] = uc[v] + (double)(e ? a1[v] : a0[v]);
              // pos_inside, with the internal energy kept for the indicator's pressure
              // Euler / Navier-Stokes: the certified internal energy (no IEEE division)
              double ei;
              if constexpr (EQ == EQ_GLM) ei = Eos<EQ>::eint(st);
              else ei = Eos<EQ>::eint_vs(st, bd.minEint);
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

// ---------------------------------------------------------------------------
// The same contraction with the halo tile staged by TMA.  Per variable v one 4D
// tensor load (x, y, z, v of the padded state; box 36 x 8 x 5 in 3D, 36 x 8 x 1 in
// 2D) brings the block's stencil footprint into shared memory; the A rows are
// built from it (the same FP64 differences as above, so the products are the
// same bits), and the load of variable v + 2 is issued as soon as the build
// of v - 1 has read its buffer (three buffers: loads run two variables ahead of
// the build).  The cell averages of the block are kept in shared memory for the
// FP64 epilogue; the limiter bounds come from bounds_kernel.  Used when the padded
// row pitch is even (TMA strides are multiples of 16 bytes).
template <int DIM>
struct HaloTile {
  static constexpr int R = 2;
  static constexpr int TX = kBlockX + 2 * R, TY = kBlockY + 2 * R, TZ = DIM == 3 ? 2 * R + 1 : 1;
  static constexpr int N = TX * TY * TZ;
  static constexpr int BYTES = N * 8;
  static_assert((TX * 8) % 16 == 0, "TMA box inner extent");
};

template <int DIM, int EQ>
struct TcTmaShape {
  using Sh = TcShape<DIM, EQ>;
  using H = HaloTile<DIM>;
  static constexpr int NV = Cfg<DIM, EQ>::NV;
  static constexpr int NBUF = 3;                                           // tiles in flight: v .. v + 2
  static constexpr int HT_BYTES = (H::BYTES + 127) / 128 * 128;
  static constexpr int OFF_HT = (Sh::USED + 127) / 128 * 128;            // halo tiles of NBUF variables
  static constexpr int OFF_UC = OFF_HT + NBUF * HT_BYTES;                 // cell averages [v][128]
  static constexpr int OFF_TO = OFF_UC + NV * 128 * 8;                    // stencil offsets in the tile [KP]
  static constexpr int OFF_BT = (OFF_TO + Sh::KP * 4 + 7) / 8 * 8;        // tile barriers [NBUF], B barrier
  static constexpr int USED = OFF_BT + 8 * (NBUF + 1);
  static constexpr int SMEM = USED > Sh::FLOOR ? USED : Sh::FLOOR;
  static_assert(SMEM <= 227 * 1024, "shared memory per block");
  static_assert(Sh::OFF_B % 16 == 0 && Sh::B_PART % 16 == 0, "bulk copy of the B operand");
  static_assert(Sh::MAX_RES < 2 || SMEM <= 113 * 1024, "two blocks per SM where TMEM allows them");
};

template <int DIM, int EQ>
__global__ void __launch_bounds__(kTcThreads, 2)
    recon_tc_tma_kernel(const __grid_constant__ CUtensorMap umap, const double *__restrict__ U, Grid g,
                        const DevStencil *__restrict__ S, int wantInd, double *__restrict__ F0,
                        double *__restrict__ F1, double *__restrict__ F2, float *__restrict__ W0,
                        float *__restrict__ W1, float *__restrict__ W2, double *__restrict__ src,
                        uint8_t *__restrict__ status, double2 *__restrict__ lamvel, double *__restrict__ bnd,
                        DevScalars *__restrict__ sc) {
  using T = Cfg<DIM, EQ>;
  using Sh = TcShape<DIM, EQ>;
  using L = TcTmaShape<DIM, EQ>;
  using H = HaloTile<DIM>;
  constexpr int NV = T::NV;
  extern __shared__ __align__(128) uint8_t smem[];
  double(*sBd)[128] = reinterpret_cast<double(*)[128]>(smem + Sh::OFF_BD);
  unsigned long long *sLam = reinterpret_cast<unsigned long long *>(smem + Sh::OFF_RED);
  unsigned long long *sVel = sLam + 128;
  int *sIn = reinterpret_cast<int *>(smem + Sh::OFF_RED + 2 * 128 * 8);
  double(*sUc)[128] = reinterpret_cast<double(*)[128]>(smem + L::OFF_UC);
  int *sTo = reinterpret_cast<int *>(smem + L::OFF_TO);
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
  const uint32_t barA = smem_u32(bar), barT = smem_u32(smem + L::OFF_BT);  // tile barriers barT + 8 b
  // padded coordinates of the tile's first cell: (i0 - 2, j0 - 2, k - 2) in cells
  const int tx0 = (int)(blockIdx.x * kBlockX), ty0 = (int)(blockIdx.y * kBlockY), tz0 = (int)k;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"((uint32_t)Sh::COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  // variable v's halo tile lands in buffer v % NBUF, completing on barrier v % NBUF
  auto issue_tile = [&](int v) {
    const int b = v % L::NBUF;
    mbar_arrive_expect_tx(barT + 8 * b, (uint32_t)H::BYTES);
    tma_load_4d(smem_u32(smem + L::OFF_HT + b * L::HT_BYTES), &umap, tx0, ty0, tz0, v, barT + 8 * b);
  };
  if (tid == 0) {
    mbar_init(barA, 1);
    for (int b = 0; b < L::NBUF; b++) mbar_init(barT + 8 * b, 1);
    mbar_init(barT + 8 * L::NBUF, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    // the split weights (B operand) on their own barrier, then the first tiles
    mbar_arrive_expect_tx(barT + 8 * L::NBUF, (uint32_t)(2 * Sh::B_PART));
    bulk_load(smem_u32(smem + Sh::OFF_B), S->tcw[0], Sh::B_PART, barT + 8 * L::NBUF);
    bulk_load(smem_u32(smem + Sh::OFF_B + Sh::B_PART), S->tcw[1], Sh::B_PART, barT + 8 * L::NBUF);
    for (int v = 0; v < L::NBUF - 1 && v < NV; v++) issue_tile(v);
  }
  for (int c = tid; c < Sh::KP; c += kTcThreads) {
    // stencil cell c relative to the cell in the halo tile
    const int dx = c < T::C ? (int)S->w.off[0][c] : 0, dy = c < T::C ? (int)S->w.off[1][c] : 0;
    const int dz = (DIM == 3 && c < T::C) ? (int)S->w.off[2][c] : 0;
    sTo[c] = (dz * H::TY + dy) * H::TX + dx;
  }
  if (part == 0) {
    sIn[row] = 1;
    sLam[row] = 0ull;
    sVel[row] = 0ull;
    if (live) {
      // limiter bounds of the cell (bounds_kernel)
      const int64_t c = (k * g.ny + j) * g.nx + i;
      sBd[0][row] = bnd[c];
      sBd[1][row] = bnd[g.n + c];
      sBd[2][row] = bnd[2 * g.n + c];
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;

  const int cm = ((DIM == 3 ? 2 : 0) * H::TY + quarter + 2) * H::TX + lane + 2; // the cell in the halo tile
  const uint32_t aHi = smem_u32(smem), aLo = aHi + Sh::A_PART;
  const uint32_t bHi = smem_u32(smem + Sh::OFF_B), bLo = bHi + Sh::B_PART;
  constexpr uint32_t idesc = tf32_idesc<Sh::NP>();
  // this thread's stencil cells (chunks part, part + 2, ...) as tile offsets (of
  // either sign), kNoCell past the stencil
  constexpr int MYCH = (Sh::NCH + kTcParts - 1) / kTcParts;
  constexpr int kNoCell = -0x40000000;
  int toff[MYCH * 4];
#pragma unroll
  for (int m = 0; m < MYCH; m++)
#pragma unroll
    for (int t = 0; t < 4; t++) {
      const int c = (part + kTcParts * m) * 4 + t;
      toff[m * 4 + t] = (c < T::C && part + kTcParts * m < Sh::NCH) ? sTo[c] : kNoCell;
    }
  // matrix descriptors of K step 0; step s adds 2 s chunks to the start address
  const uint64_t dAh = umma_desc(aHi, Sh::A_CH, 128), dAl = umma_desc(aLo, Sh::A_CH, 128);
  const uint64_t dBh = umma_desc(bHi, Sh::B_CH, 128), dBl = umma_desc(bLo, Sh::B_CH, 128);

  bool ok = mbar_wait(barT + 8 * L::NBUF, 0u);                 // the B operand
  int issued = NV < L::NBUF - 1 ? NV : L::NBUF - 1;            // tile loads issued (thread 0)
  int consumed = 0;                                            // tile loads waited for
#pragma unroll 1
  for (int v = 0; v < NV; v++) {
    if (v > 0) ok = ok && mbar_wait(barA, (uint32_t)(v - 1) & 1u);   // the MMAs of v - 1 have read A
    ok = ok && mbar_wait(barT + 8 * (v % L::NBUF), (uint32_t)(v / L::NBUF) & 1u);  // v's tile has landed
    if (!__syncthreads_and(ok)) break;
    consumed = v + 1;
    const double *ht = reinterpret_cast<const double *>(smem + L::OFF_HT + (v % L::NBUF) * L::HT_BYTES);
    const double ucv = live ? ht[cm] : 0.0;
    if (part == 0) sUc[v][row] = ucv;
#pragma unroll
    for (int m = 0; m < MYCH; m++) {
      const int ch = part + kTcParts * m;
      if (ch < Sh::NCH) {
        uint32_t hi[4], lo[4];
#pragma unroll
        for (int t = 0; t < 4; t++) {
          const int o = toff[m * 4 + t];
          const float d = (o != kNoCell && live) ? (float)(ht[cm + o] - ucv) : 0.0f;
          hi[t] = tf32_rna_bits(d);
          lo[t] = tf32_rna_bits(d - __uint_as_float(hi[t]));
        }
        st_shared_v4(aHi + ch * Sh::A_CH + row * 16, hi);
        st_shared_v4(aLo + ch * Sh::A_CH + row * 16, lo);
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      if (v + L::NBUF - 1 < NV) {
        // variable v + NBUF - 1 into the buffer of v - 1, whose build finished last iteration
        issue_tile(v + L::NBUF - 1);
        issued++;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t d = tmem + (uint32_t)(v * Sh::NP);
#pragma unroll
      for (int s = 0; s < Sh::NKS; s++) {
        // the descriptor's start-address field counts 16-byte units
        const uint64_t sa = (uint64_t)(2 * s * Sh::A_CH) >> 4, sb = (uint64_t)(2 * s * Sh::B_CH) >> 4;
        mma_tf32(d, dAl + sa, dBh + sb, idesc, s > 0);
        mma_tf32(d, dAh + sa, dBl + sb, idesc, 1);
        mma_tf32(d, dAh + sa, dBh + sb, idesc, 1);
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
    for (int v = 0; v < NV; v++) uc[v] = sUc[v][row];
    const uint32_t lanes = (uint32_t)(quarter * 32) << 16;
    const int64_t c = (k * g.ny + j) * g.nx + i;
    bool inside = true;
    double lam = 0.0, vel = 0.0;
    auto epilogue = [&](auto partTag) {
      constexpr int PART = decltype(partTag)::value;
      constexpr int R0 = PART * Sh::RPP;
#pragma unroll
      for (int rp = 0; rp < Sh::RPP; rp += 2) {
        float a0[NV], a1[NV];
        tmem_ld2_n<NV>(tmem + lanes + (uint32_t)(R0 + rp), (uint32_t)Sh::NP, a0, a1);
        if (live) {
#pragma unroll
          for (int e = 0; e < 2; e++) {
            const int rw = R0 + rp + e;
            if (rw < Sh::NR) {
              double st[NV];
#pragma unroll
              for (int v = 0; v < NV; v++) st[v] = uc[v] + (double)(e ? a1[v] : a0[v]);
              // Euler / Navier-Stokes: the certified internal energy (no IEEE division)
              double ei;
              if constexpr (EQ == EQ_GLM) ei = Eos<EQ>::eint(st);
              else ei = Eos<EQ>::eint_vs(st, bd.minEint);
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
    if (part == 0) epilogue(std::integral_constant<int, 0>{});
    else epilogue(std::integral_constant<int, 1>{});
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
    // tile loads still in flight land before the block leaves
    for (int v = consumed; v < issued; v++) mbar_wait(barT + 8 * (v % L::NBUF), (uint32_t)(v / L::NBUF) & 1u);
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
static cudaError_t recon_tc_launch(const double *U, const CUtensorMap *umap, const Grid &g, const DevStencil *S,
                                   int wantInd, double *const *F, float *const *W, double *src, uint8_t *status,
                                   double2 *lamvel, double *bnd, DevScalars *sc, cudaStream_t s) {
  using Sh = TcShape<DIM, EQ>;
  using L = TcTmaShape<DIM, EQ>;
  const dim3 grid((unsigned)((g.nx + kBlockX - 1) / kBlockX), (unsigned)((g.ny + kBlockY - 1) / kBlockY),
                  (unsigned)g.nz);
  if (umap) {
    // the attribute is per function and process-wide: set once (a function-local
    // static is initialised once, also when several host threads drive solvers)
    static const cudaError_t attrT =
        cudaFuncSetAttribute(recon_tc_tma_kernel<DIM, EQ>, cudaFuncAttributeMaxDynamicSharedMemorySize, L::SMEM);
    if (attrT != cudaSuccess) return attrT;
    recon_tc_tma_kernel<DIM, EQ><<<grid, kTcThreads, L::SMEM, s>>>(
        *umap, U, g, S, wantInd, F[0], F[1], F[2], W[0], W[1], W[2], src, status, lamvel, bnd, sc);
    return cudaGetLastError();
  }
  static const cudaError_t attr =
      cudaFuncSetAttribute(recon_tc_kernel<DIM, EQ>, cudaFuncAttributeMaxDynamicSharedMemorySize, Sh::SMEM);
  if (attr != cudaSuccess) return attr;
  recon_tc_kernel<DIM, EQ><<<grid, kTcThreads, Sh::SMEM, s>>>(
      U, g, S, wantInd, F[0], F[1], F[2], W[0], W[1], W[2], src, status, lamvel, bnd, sc);
  return cudaGetLastError();
}

cudaError_t launch_recon_tc(int dim, int eq, const double *U, const CUtensorMap *umap, const Grid &g,
                            const DevStencil *S, int wantInd, double *const *F, float *const *W, double *src,
                            uint8_t *status, double2 *lamvel, double *bnd, DevScalars *sc, cudaStream_t s) {
  if (dim == 2) {
    if (eq == EQ_GLM) return recon_tc_launch<2, EQ_GLM>(U, umap, g, S, wantInd, F, W, src, status, lamvel, bnd, sc, s);
    if (eq == EQ_NS) return recon_tc_launch<2, EQ_NS>(U, umap, g, S, wantInd, F, W, src, status, lamvel, bnd, sc, s);
    return recon_tc_launch<2, EQ_HYDRO>(U, umap, g, S, wantInd, F, W, src, status, lamvel, bnd, sc, s);
  }
  if (eq == EQ_GLM) return recon_tc_launch<3, EQ_GLM>(U, umap, g, S, wantInd, F, W, src, status, lamvel, bnd, sc, s);
  if (eq == EQ_NS) return recon_tc_launch<3, EQ_NS>(U, umap, g, S, wantInd, F, W, src, status, lamvel, bnd, sc, s);
  return recon_tc_launch<3, EQ_HYDRO>(U, umap, g, S, wantInd, F, W, src, status, lamvel, bnd, sc, s);
}

// 4D map (x, y, z, variable) of a padded state for the halo-tile loads, or a
// nonzero return where TMA cannot address it (odd row pitch)
int recon_tc_state_map(CUtensorMap *map, const double *U, const Grid &g, int dim, int nv) {
  if (g.px % 2 != 0) return 1;
  const uint64_t planes = (uint64_t)(g.pvol / (g.px * g.py));
  const uint64_t dims[4] = {(uint64_t)g.px, (uint64_t)g.py, planes, (uint64_t)nv};
  const uint64_t strides[3] = {(uint64_t)g.px * 8, (uint64_t)(g.px * g.py) * 8, (uint64_t)g.pvol * 8};
  const uint32_t box[4] = {(uint32_t)(dim == 3 ? HaloTile<3>::TX : HaloTile<2>::TX),
                           (uint32_t)(dim == 3 ? HaloTile<3>::TY : HaloTile<2>::TY),
                           (uint32_t)(dim == 3 ? HaloTile<3>::TZ : HaloTile<2>::TZ), 1u};
  return encode_tensor_map_8b(map, U, 4, dims, strides, box);
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
