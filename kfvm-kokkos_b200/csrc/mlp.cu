// mlp.cu -- the learned troubled-cell indicator: training-sample collection,
// training (forward + backward + Adam), and inference inside the stage.
//
// Labels come from the method itself: a cell is troubled when its WENO-AO
// nonlinear weights depart from the linear ones by more than tau
// (weno_departure).  Inference replaces the KXRCF selector (WenoSelect_K,
// Numeric_K.H:292-398 of the reference): it writes the same per-cell flags that
// compact_kernel turns into the WENO set, with the positivity-history rule
// (theta < 1 flags a cell) kept.  A sampled fraction of cells (the judge) always
// runs full WENO; heavy_var_kernel computes their labels on the way and counts the
// cells the network missed, which the host uses to fall back to KXRCF.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.cuh"
#include "launch.h"
#include "mlp.cuh"
#include "tcgen05.cuh"

namespace kfvm {

// ---------------------------------------------------------------------------
// sample collection: every cell's label; positives always kept, negatives with
// probability keep_frac; features stored as BF16
template <int DIM, int EQ>
__global__ void __launch_bounds__(128)
    mlp_collect_kernel(const double *__restrict__ U, Grid g, const DevStencil *__restrict__ S, double tau,
                       double keep_frac, uint64_t seed, uint16_t *__restrict__ feats, uint8_t *__restrict__ labels,
                       int64_t *__restrict__ cells, unsigned long long *__restrict__ count, int64_t cap) {
  using M = MlpShape<DIM>;
  using Tl = MlpTile<DIM>;
  __shared__ float tile[2][Tl::N];
  const int64_t i0 = blockIdx.x * (int64_t)kBlockX, j0 = blockIdx.y * (int64_t)kBlockY, k = blockIdx.z;
  mlp_tile_fill<DIM, EQ>(U, g, i0, j0, k, tile);
  __syncthreads();
  const int64_t i = i0 + threadIdx.x, j = j0 + threadIdx.y;
  if (i >= g.nx || j >= g.ny) return;
  const int64_t c = (k * g.ny + j) * g.nx + i;
  const double dep = weno_departure<DIM, EQ>(U + pidx(g, i, j, k), g, S);
  const bool pos = dep > tau;
  if (!pos && !(unit_hash(seed, (uint64_t)c) < keep_frac)) return;
  const unsigned long long idx = atomicAdd(count, 1ull);
  if ((int64_t)idx >= cap) return;
  float rc, pc, sr, sp;
  mlp_scales<DIM>(tile, threadIdx.x, threadIdx.y, rc, pc, sr, sp);
  constexpr int R = Tl::R, ZR = DIM == 3 ? R : 0;
  const int c0 = (ZR * Tl::TY + threadIdx.y + R) * Tl::TX + threadIdx.x + R;
  uint16_t *x = feats + (int64_t)idx * M::NI;
  int q = 0;
  for (int dz = -ZR; dz <= ZR; dz++)
    for (int dy = -R; dy <= R; dy++)
      for (int dx = -R; dx <= R; dx++, q++) {
        const int n = c0 + (dz * Tl::TY + dy) * Tl::TX + dx;
        x[q] = __bfloat16_as_ushort(__float2bfloat16_rn(mlp_feature(tile[0][n], rc, sr)));
        x[M::P + q] = __bfloat16_as_ushort(__float2bfloat16_rn(mlp_feature(tile[1][n], pc, sp)));
      }
  labels[idx] = pos ? 1 : 0;
  cells[idx] = c;
}

// ---------------------------------------------------------------------------
// training: one block = kTrainB samples drawn uniformly (with replacement) from
// the collected set; forward and backward in FP32 with the BF16-rounded weights,
// gradients of the weighted binary cross entropy summed into grad
constexpr int kTrainB = 64;

template <int DIM>
struct TrainSmem {
  using M = MlpShape<DIM>;
  static constexpr int W = 0;
  static constexpr int X = W + M::NW;
  static constexpr int Z1 = X + kTrainB * M::NI;
  static constexpr int Z2 = Z1 + kTrainB * M::NH;
  static constexpr int H1 = Z2 + kTrainB * M::NH;
  static constexpr int H2 = H1 + kTrainB * M::NH;
  static constexpr int D1 = H2 + kTrainB * M::NH;
  static constexpr int D2 = D1 + kTrainB * M::NH;
  static constexpr int DY = D2 + kTrainB * M::NH;
  static constexpr int LB = DY + kTrainB;
  static constexpr int FLOATS = LB + kTrainB;
  static constexpr size_t BYTES = (size_t)FLOATS * sizeof(float);
};

template <int DIM>
__global__ void __launch_bounds__(256)
    mlp_train_kernel(const uint16_t *__restrict__ feats, const uint8_t *__restrict__ labels, int64_t n,
                     const float *__restrict__ w, float *__restrict__ grad, float *__restrict__ loss,
                     float pos_weight, float inv_batch, uint64_t seed, int64_t step) {
  using M = MlpShape<DIM>;
  using L = TrainSmem<DIM>;
  extern __shared__ float sm[];
  float *W = sm + L::W, *X = sm + L::X, *Z1 = sm + L::Z1, *Z2 = sm + L::Z2, *H1 = sm + L::H1, *H2 = sm + L::H2;
  float *D1 = sm + L::D1, *D2 = sm + L::D2, *DY = sm + L::DY, *LB = sm + L::LB;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int t = tid; t < M::NW; t += nt) W[t] = w[t];
  for (int t = tid; t < kTrainB * M::NI; t += nt) {
    const int s = t / M::NI, i = t % M::NI;
    const int64_t idx = (int64_t)(mix64(seed ^ mix64((uint64_t)step * 1315423911ull + blockIdx.x * kTrainB + s)) %
                                  (uint64_t)n);
    X[t] = __bfloat162float(__ushort_as_bfloat16(feats[idx * M::NI + i]));
    if (i == 0) LB[s] = (float)labels[idx];
  }
  __syncthreads();
  for (int t = tid; t < kTrainB * M::NH; t += nt) {
    const int s = t / M::NH, h = t % M::NH;
    float z = W[M::B1 + h];
    const float *wr = W + M::W1 + h * M::NI, *x = X + s * M::NI;
    for (int i = 0; i < M::NI; i++) z = fmaf(wr[i], x[i], z);
    Z1[t] = z;
    H1[t] = gelu(z);
  }
  __syncthreads();
  for (int t = tid; t < kTrainB * M::NH; t += nt) {
    const int s = t / M::NH, h = t % M::NH;
    float z = W[M::B2 + h];
    const float *wr = W + M::W2 + h * M::NH, *x = H1 + s * M::NH;
#pragma unroll 8
    for (int i = 0; i < M::NH; i++) z = fmaf(wr[i], x[i], z);
    Z2[t] = z;
    H2[t] = gelu(z);
  }
  __syncthreads();
  if (tid < kTrainB) {
    float z = W[M::B3];
    const float *x = H2 + tid * M::NH;
#pragma unroll 8
    for (int i = 0; i < M::NH; i++) z = fmaf(W[M::W3 + i], x[i], z);
    const float y = LB[tid], wt = y > 0.5f ? pos_weight : 1.0f;
    const float p = 1.0f / (1.0f + expf(-z));
    // weighted BCE on the logit: wt (softplus(z) - y z)
    const float sp = z > 0.0f ? z + log1pf(expf(-z)) : log1pf(expf(z));
    atomicAdd(loss, wt * (sp - y * z) * inv_batch);
    DY[tid] = wt * (p - y) * inv_batch;
  }
  __syncthreads();
  for (int t = tid; t < kTrainB * M::NH; t += nt) {
    const int h = t % M::NH;
    D2[t] = DY[t / M::NH] * W[M::W3 + h] * gelu_grad(Z2[t]);
  }
  __syncthreads();
  for (int t = tid; t < kTrainB * M::NH; t += nt) {
    const int s = t / M::NH, h = t % M::NH;
    float a = 0.0f;
#pragma unroll 8
    for (int o = 0; o < M::NH; o++) a = fmaf(W[M::W2 + o * M::NH + h], D2[s * M::NH + o], a);
    D1[t] = a * gelu_grad(Z1[t]);
  }
  __syncthreads();
  // parameter gradients, summed over the block's samples
  for (int t = tid; t < M::NW; t += nt) {
    float a = 0.0f;
    if (t < M::B1) {
      const int h = t / M::NI, i = t % M::NI;
      for (int s = 0; s < kTrainB; s++) a = fmaf(D1[s * M::NH + h], X[s * M::NI + i], a);
    } else if (t < M::W2) {
      for (int s = 0; s < kTrainB; s++) a += D1[s * M::NH + (t - M::B1)];
    } else if (t < M::B2) {
      const int o = (t - M::W2) / M::NH, h = (t - M::W2) % M::NH;
      for (int s = 0; s < kTrainB; s++) a = fmaf(D2[s * M::NH + o], H1[s * M::NH + h], a);
    } else if (t < M::W3) {
      for (int s = 0; s < kTrainB; s++) a += D2[s * M::NH + (t - M::B2)];
    } else if (t < M::B3) {
      for (int s = 0; s < kTrainB; s++) a = fmaf(DY[s], H2[s * M::NH + (t - M::W3)], a);
    } else {
      for (int s = 0; s < kTrainB; s++) a += DY[s];
    }
    atomicAdd(grad + t, a);
  }
}

// Adam on the FP32 master weights; the forward passes use their BF16 rounding
__global__ void __launch_bounds__(256)
    mlp_adam_kernel(float *__restrict__ master, float *__restrict__ m, float *__restrict__ v,
                    float *__restrict__ grad, float *__restrict__ wq, uint16_t *__restrict__ wb, int nw, float lr,
                    float c1, float c2) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nw) return;
  const float gr = grad[t];
  grad[t] = 0.0f;
  const float mt = 0.9f * m[t] + 0.1f * gr, vt = 0.999f * v[t] + 0.001f * gr * gr;
  m[t] = mt;
  v[t] = vt;
  const float x = master[t] - lr * (mt * c1) / (sqrtf(vt * c2) + 1e-8f);
  master[t] = x;
  const __nv_bfloat16 b = __float2bfloat16_rn(x);
  wb[t] = __bfloat16_as_ushort(b);
  wq[t] = __bfloat162float(b);
}

// ---------------------------------------------------------------------------
// Inference with the first layer on the tcgen05 tensor cores: per block of 128
// cells (two threads per cell = per row of the tile) the BF16 feature rows form
// A [128 x KP], W1^T in BF16 forms B [KP x 32], and D = A B accumulates in FP32
// in 32 TMEM columns (M128 N32 K16 MMAs, kind::f16).  The features are written
// in halves of K into one shared-memory buffer (two blocks fit an SM).  Then
// bias + GELU, the 32 x 32 second layer and the output on the CUDA cores in FP32
// (as in training).  Every mbarrier wait is bounded; on timeout the block sets
// DevScalars::fault and returns after freeing its TMEM.
constexpr int kMlpThreads = 256;

template <int DIM>
struct MlpTc {
  using M = MlpShape<DIM>;
  using Tl = MlpTile<DIM>;
  static constexpr int KP = (M::NI + 15) / 16 * 16;        // K padded to the MMA K of 16
  static constexpr int NCH = KP / 8;                       // 16-byte chunks of 8 BF16
  static constexpr int HALVES = DIM == 3 ? 2 : 1;
  static constexpr int NCHH = NCH / HALVES;                // chunks per half
  static constexpr int A_CH = 128 * 16;
  static constexpr int B_CH = 32 * 16;
  static constexpr int OFF_B = NCHH * A_CH;                // A: one half
  static constexpr int OFF_TILE = OFF_B + NCH * B_CH;      // B: all of W1^T
  static constexpr int OFF_H = OFF_TILE + (2 * Tl::N * 4 + 15) / 16 * 16; // H1 [128][33] floats
  static constexpr int OFF_W = OFF_H + 128 * 33 * 4;       // b1, W2, b2, w3, b3 (floats)
  static constexpr int NW2 = M::NW - M::B1;
  static constexpr int OFF_SC = OFF_W + (NW2 + 3) / 4 * 16; // centers and scales [128][4] floats
  static constexpr int OFF_OFS = OFF_SC + 128 * 4 * 4;     // patch offsets [P] int
  static constexpr int OFF_BAR = OFF_OFS + (M::P + 3) / 4 * 16;
  static constexpr int SMEM = OFF_BAR + 16;
  static_assert(NCH % HALVES == 0 && NCHH % 2 == 0, "K halves of whole MMA steps");
  static_assert(SMEM <= 113 * 1024, "two blocks per SM");
};

template <int DIM>
__global__ void __launch_bounds__(256) mlp_pack_kernel(const uint16_t *__restrict__ wb, uint16_t *__restrict__ img) {
  using M = MlpShape<DIM>;
  using C = MlpTc<DIM>;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 32 * C::KP) return;
  const int n = t / C::KP, k = t % C::KP;
  img[(k / 8) * 256 + n * 8 + (k % 8)] = k < M::NI ? wb[M::W1 + n * M::NI + k] : (uint16_t)0;
}

// mode 0: flags (+ prediction, flagged count); mode 1: probabilities
template <int DIM, int EQ, int MODE>
__global__ void __launch_bounds__(kMlpThreads, 2)
    mlp_tc_kernel(const double *__restrict__ U, Grid g, const uint16_t *__restrict__ wb,
                  const uint16_t *__restrict__ w1img, const double *__restrict__ theta, uint8_t *__restrict__ flag,
                  uint8_t *__restrict__ pred, float *__restrict__ prob, DevScalars *__restrict__ sc, float logit_thr) {
  using M = MlpShape<DIM>;
  using Tl = MlpTile<DIM>;
  using C = MlpTc<DIM>;
  extern __shared__ __align__(128) uint8_t msm[];
  float(*tile)[Tl::N] = reinterpret_cast<float(*)[Tl::N]>(msm + C::OFF_TILE);
  float(*sH)[33] = reinterpret_cast<float(*)[33]>(msm + C::OFF_H);
  float *sW = reinterpret_cast<float *>(msm + C::OFF_W);   // layout of the flat weights from B1 on
  float(*sSc)[4] = reinterpret_cast<float(*)[4]>(msm + C::OFF_SC);
  int *sOfs = reinterpret_cast<int *>(msm + C::OFF_OFS);
  uint64_t *bar = reinterpret_cast<uint64_t *>(msm + C::OFF_BAR);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(msm + C::OFF_BAR + 8);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int quarter = warp & 3, part = warp >> 2;
  const int row = quarter * 32 + lane;
  const int64_t i0 = blockIdx.x * (int64_t)kBlockX, j0 = blockIdx.y * (int64_t)kBlockY, k = blockIdx.z;
  const int64_t i = i0 + lane, j = j0 + quarter;
  const bool live = i < g.nx && j < g.ny;
  const uint32_t barA = smem_u32(bar);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(32u)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(barA) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  {
    const uint4 *src = reinterpret_cast<const uint4 *>(w1img);
    uint4 *dst = reinterpret_cast<uint4 *>(msm + C::OFF_B);
    for (int t = tid; t < C::NCH * C::B_CH / 16; t += kMlpThreads) dst[t] = src[t];
    for (int t = tid; t < C::NW2; t += kMlpThreads) sW[t] = __bfloat162float(__ushort_as_bfloat16(wb[M::B1 + t]));
    constexpr int ZR = DIM == 3 ? Tl::R : 0;
    for (int q = tid; q < M::P; q += kMlpThreads) {
      const int dx = q % M::SIDE - Tl::R, dy = (q / M::SIDE) % M::SIDE - Tl::R, dz = q / (M::SIDE * M::SIDE) - ZR;
      sOfs[q] = (dz * Tl::TY + dy) * Tl::TX + dx;
    }
  }
  for (int t = tid; t < Tl::N; t += kMlpThreads) {
    const int a = t % Tl::TX, b = (t / Tl::TX) % Tl::TY, cz = t / (Tl::TX * Tl::TY);
    const int64_t gi = i0 - Tl::R + a, gj = j0 - Tl::R + b, gk = k - (DIM == 3 ? Tl::R : 0) + cz;
    if (gi > g.nx + Tl::R - 1 || gj > g.ny + Tl::R - 1) continue;
    const double *Uq = U + pidx(g, gi, gj, gk);
    double u[Eos<EQ>::NV];
#pragma unroll
    for (int v = 0; v < Eos<EQ>::NV; v++) u[v] = Uq[v * g.pvol];
    tile[0][t] = (float)u[DENS];
    tile[1][t] = (float)Eos<EQ>::pres(g.gamma, u);
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  // scales of the two patches: part 0 density, part 1 pressure
  constexpr int ZR = DIM == 3 ? Tl::R : 0;
  const int c0 = (ZR * Tl::TY + quarter + Tl::R) * Tl::TX + lane + Tl::R;
  {
    const float ref = tile[part][c0];
    float mx = 0.0f;
    for (int q = 0; q < M::P; q++) mx = fmaxf(mx, fabsf(__fsub_rn(tile[part][c0 + sOfs[q]], ref)));
    sSc[row][part] = ref;
    sSc[row][2 + part] = mlp_scale(mx, ref);
  }
  __syncthreads();
  const float rc = sSc[row][0], pc = sSc[row][1], sr = sSc[row][2], sp = sSc[row][3];
  const uint32_t aB = smem_u32(msm), bB = smem_u32(msm + C::OFF_B);
  constexpr uint32_t idesc = bf16_idesc<32>();
  bool ok = true;
#pragma unroll 1
  for (int h = 0; h < C::HALVES; h++) {
    // this thread's chunks of the half: features k = 8 ch .. 8 ch + 7
    for (int cl = part; cl < C::NCHH; cl += 2) {
      const int ch = h * C::NCHH + cl;
      uint32_t pk[4];
#pragma unroll
      for (int t = 0; t < 4; t++) {
        float x2[2];
#pragma unroll
        for (int e = 0; e < 2; e++) {
          const int kk = ch * 8 + 2 * t + e;
          float x = 0.0f;
          if (kk < M::P) x = mlp_feature(tile[0][c0 + sOfs[kk]], rc, sr);
          else if (kk < M::NI) x = mlp_feature(tile[1][c0 + sOfs[kk - M::P]], pc, sp);
          x2[e] = live ? x : 0.0f;
        }
        const __nv_bfloat162 b2 = __floats2bfloat162_rn(x2[0], x2[1]); // .x low half, .y high half
        pk[t] = *reinterpret_cast<const uint32_t *>(&b2);
      }
      st_shared_v4(aB + cl * C::A_CH + row * 16, pk);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll 1
      for (int s = 0; s < C::NCHH / 2; s++) {
        const uint64_t ad = umma_desc(aB + 2 * s * C::A_CH, C::A_CH, 128);
        const uint64_t bd = umma_desc(bB + (h * C::NCHH + 2 * s) * C::B_CH, C::B_CH, 128);
        mma_bf16(tmem, ad, bd, idesc, (h > 0 || s > 0) ? 1 : 0);
      }
      mma_commit(barA);
    }
    ok = mbar_wait(barA, (uint32_t)h & 1u);
    if (!__syncthreads_and(ok)) break;
  }
  if (__syncthreads_and(ok)) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // first layer: bias + GELU of this part's 16 hidden units
    const uint32_t lanes = (uint32_t)(quarter * 32) << 16;
    float z[16];
    tmem_ld8(tmem + lanes + (uint32_t)(16 * part), *reinterpret_cast<float(*)[8]>(z));
    tmem_ld8(tmem + lanes + (uint32_t)(16 * part + 8), *reinterpret_cast<float(*)[8]>(z + 8));
#pragma unroll
    for (int t = 0; t < 16; t++) sH[row][16 * part + t] = gelu(z[t] + sW[16 * part + t]);
    __syncthreads();
    // second layer and output on the CUDA cores, 16 outputs per part
    float acc = 0.0f;
#pragma unroll 4
    for (int o = 16 * part; o < 16 * part + 16; o++) {
      float a = sW[M::B2 - M::B1 + o];
      const float *wr = sW + (M::W2 - M::B1) + o * M::NH;
#pragma unroll
      for (int hh = 0; hh < M::NH; hh++) a = fmaf(wr[hh], sH[row][hh], a);
      acc = fmaf(sW[M::W3 - M::B1 + o], gelu(a), acc);
    }
    __syncthreads();
    if (part == 1) sH[row][32] = acc;   // the second half's sum, read by part 0
    __syncthreads();
    if (part == 0 && live) {
      const float logit = sW[M::B3 - M::B1] + acc + sH[row][32];
      const int64_t c = (k * g.ny + j) * g.nx + i;
      if (MODE == 0) {
        const bool p = logit > logit_thr;
        pred[c] = p ? 1 : 0;
        const bool f = p || theta[c] < 1.0;
        flag[c] = f ? 1 : 0;
      } else {
        prob[c] = 1.0f / (1.0f + expf(-logit));
      }
    }
    if (MODE == 0 && part == 0) {
      bool f = false;
      if (live) f = flag[(k * g.ny + j) * g.nx + i] != 0;
      const unsigned ball = __ballot_sync(0xffffffffu, f);
      if (lane == 0 && ball) atomicAdd(&sc->nflag, (unsigned)__popc(ball));
    }
  } else if (tid == 0) {
    atomicExch(&sc->fault, 1u);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(32u) : "memory");
}

// ---------------------------------------------------------------------------
// host launchers
static dim3 mlp_cell_grid(const Grid &g) {
  return dim3((unsigned)((g.nx + kBlockX - 1) / kBlockX), (unsigned)((g.ny + kBlockY - 1) / kBlockY),
              (unsigned)g.nz);
}

int mlp_num_weights(int dim) { return dim == 2 ? MlpShape<2>::NW : MlpShape<3>::NW; }
int mlp_num_inputs(int dim) { return dim == 2 ? MlpShape<2>::NI : MlpShape<3>::NI; }

template <int DIM, int EQ>
static cudaError_t collect_t(const double *U, const Grid &g, const DevStencil *S, double tau, double keep,
                             uint64_t seed, uint16_t *feats, uint8_t *labels, int64_t *cells,
                             unsigned long long *count, int64_t cap, cudaStream_t s) {
  mlp_collect_kernel<DIM, EQ><<<mlp_cell_grid(g), dim3(kBlockX, kBlockY), 0, s>>>(U, g, S, tau, keep, seed, feats,
                                                                                   labels, cells, count, cap);
  return cudaGetLastError();
}

template <int DIM, int EQ, int MODE>
static cudaError_t tc_t(const double *U, const Grid &g, const uint16_t *wb, const uint16_t *img, const double *theta,
                        uint8_t *flag, uint8_t *pred, float *prob, DevScalars *sc, float thr, cudaStream_t s) {
  using C = MlpTc<DIM>;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(mlp_tc_kernel<DIM, EQ, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         C::SMEM);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  mlp_tc_kernel<DIM, EQ, MODE><<<mlp_cell_grid(g), kMlpThreads, C::SMEM, s>>>(U, g, wb, img, theta, flag, pred, prob,
                                                                            sc, thr);
  return cudaGetLastError();
}

template <int DIM, int EQ>
static cudaError_t flag_t(const double *U, const Grid &g, const uint16_t *wb, const uint16_t *img,
                          const double *theta, uint8_t *flag, uint8_t *pred, DevScalars *sc, float thr, cudaStream_t s) {
  return tc_t<DIM, EQ, 0>(U, g, wb, img, theta, flag, pred, nullptr, sc, thr, s);
}

template <int DIM, int EQ>
static cudaError_t prob_t(const double *U, const Grid &g, const uint16_t *wb, const uint16_t *img, float *out,
                          DevScalars *sc, cudaStream_t s) {
  return tc_t<DIM, EQ, 1>(U, g, wb, img, nullptr, nullptr, nullptr, out, sc, 0.0f, s);
}

#define KFVM_MLP_DISPATCH(DIM_, EQ_, FN, ...)                                      \
  do {                                                                           \
    if ((DIM_) == 2 && (EQ_) == EQ_HYDRO) return FN<2, EQ_HYDRO>(__VA_ARGS__);   \
    if ((DIM_) == 3 && (EQ_) == EQ_HYDRO) return FN<3, EQ_HYDRO>(__VA_ARGS__);   \
    if ((DIM_) == 2 && (EQ_) == EQ_NS) return FN<2, EQ_NS>(__VA_ARGS__);         \
    if ((DIM_) == 3 && (EQ_) == EQ_NS) return FN<3, EQ_NS>(__VA_ARGS__);         \
    if ((DIM_) == 2 && (EQ_) == EQ_GLM) return FN<2, EQ_GLM>(__VA_ARGS__);       \
    if ((DIM_) == 3 && (EQ_) == EQ_GLM) return FN<3, EQ_GLM>(__VA_ARGS__);       \
    return cudaErrorInvalidValue;                                                \
  } while (0)

cudaError_t launch_mlp_collect(int dim, int eq, const double *U, const Grid &g, const DevStencil *S, double tau,
                               double keep, uint64_t seed, uint16_t *feats, uint8_t *labels, int64_t *cells,
                               unsigned long long *count, int64_t cap, cudaStream_t s) {
  KFVM_MLP_DISPATCH(dim, eq, collect_t, U, g, S, tau, keep, seed, feats, labels, cells, count, cap, s);
}

cudaError_t launch_mlp_flag(int dim, int eq, const double *U, const Grid &g, const uint16_t *wb,
                            const uint16_t *w1img, const double *theta, uint8_t *flag, uint8_t *pred, DevScalars *sc,
                            float logit_thr, cudaStream_t s) {
  KFVM_MLP_DISPATCH(dim, eq, flag_t, U, g, wb, w1img, theta, flag, pred, sc, logit_thr, s);
}

cudaError_t launch_mlp_prob(int dim, int eq, const double *U, const Grid &g, const uint16_t *wb,
                            const uint16_t *w1img, float *out, DevScalars *sc, cudaStream_t s) {
  KFVM_MLP_DISPATCH(dim, eq, prob_t, U, g, wb, w1img, out, sc, s);
}

int mlp_w1_image_size(int dim) { return dim == 2 ? 32 * MlpTc<2>::KP : 32 * MlpTc<3>::KP; }

cudaError_t launch_mlp_pack(int dim, const uint16_t *wb, uint16_t *img, cudaStream_t s) {
  const int n = mlp_w1_image_size(dim);
  if (dim == 2) mlp_pack_kernel<2><<<(n + 255) / 256, 256, 0, s>>>(wb, img);
  else mlp_pack_kernel<3><<<(n + 255) / 256, 256, 0, s>>>(wb, img);
  return cudaGetLastError();
}

cudaError_t launch_mlp_train_step(int dim, const uint16_t *feats, const uint8_t *labels, int64_t n, int batch,
                                  float *master, float *m, float *v, float *grad, float *wq, uint16_t *wb,
                                  float *loss, float pos_weight, float lr, int t, uint64_t seed, cudaStream_t s) {
  const int blocks = (batch + kTrainB - 1) / kTrainB;
  const float inv = 1.0f / (float)(blocks * kTrainB);
  cudaError_t e;
  if (dim == 2) {
    static bool attr = false;
    if (!attr && (e = cudaFuncSetAttribute(mlp_train_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)TrainSmem<2>::BYTES)) != cudaSuccess)
      return e;
    attr = true;
    mlp_train_kernel<2><<<blocks, 256, TrainSmem<2>::BYTES, s>>>(feats, labels, n, wq, grad, loss, pos_weight, inv,
                                                                 seed, t);
  } else {
    static bool attr = false;
    if (!attr && (e = cudaFuncSetAttribute(mlp_train_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)TrainSmem<3>::BYTES)) != cudaSuccess)
      return e;
    attr = true;
    mlp_train_kernel<3><<<blocks, 256, TrainSmem<3>::BYTES, s>>>(feats, labels, n, wq, grad, loss, pos_weight, inv,
                                                                 seed, t);
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  const int nw = mlp_num_weights(dim);
  const float c1 = 1.0f / (1.0f - powf(0.9f, (float)t)), c2 = 1.0f / (1.0f - powf(0.999f, (float)t));
  mlp_adam_kernel<<<(nw + 255) / 256, 256, 0, s>>>(master, m, v, grad, wq, wb, nw, lr, c1, c2);
  return cudaGetLastError();
}

} // namespace kfvm
