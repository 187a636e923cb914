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

#include <thrust/iterator/counting_iterator.h>

#include <algorithm>
#include <cstdint>
#include <cub/device/device_select.cuh>

#include "kernels.cuh"
#include "launch.h"
#include "mlp.cuh"
#include "tcgen05.cuh"
#include "tma.cuh"

namespace kfvm {

// ---------------------------------------------------------------------------
// sample collection, in a fixed order: (1) every cell's label and keep decision
// (positives always kept, negatives with probability keep_frac by a hash of the
// cell); (2) the kept cells compacted in cell order (a stable select); (3) their
// features from the (density, pressure) pairs, stored as BF16.  The set and its
// order repeat exactly, so training on it does too.
template <int DIM, int EQ>
__global__ void __launch_bounds__(256)
    mlp_label_kernel(const double *__restrict__ U, Grid g, const DevStencil *__restrict__ S, double tau,
                     double keep_frac, uint64_t seed, uint8_t *__restrict__ flags) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= g.n) return;
  const int64_t i = c % g.nx, j = (c / g.nx) % g.ny, k = c / (g.nx * g.ny);
  const double dep = weno_departure<DIM, EQ>(U + pidx(g, i, j, k), g, S);
  const bool pos = dep > tau;
  const bool keep = pos || unit_hash(seed, (uint64_t)c) < keep_frac;
  flags[c] = keep ? (pos ? 3 : 1) : 0;
}

template <int DIM>
__global__ void __launch_bounds__(128)
    mlp_feature_kernel(const float2 *__restrict__ rp, int64_t rpx, Grid g, const int64_t *__restrict__ sel,
                       int64_t count, const uint8_t *__restrict__ flags, uint16_t *__restrict__ feats,
                       uint8_t *__restrict__ labels, int64_t *__restrict__ cells) {
  using M = MlpShape<DIM>;
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= count) return;
  const int64_t c = sel[t];
  const int64_t i = c % g.nx, j = (c / g.nx) % g.ny, k = c / (g.nx * g.ny);
  const float2 *p0 = rp + ((k + g.rz) * g.py + j + kRad) * rpx + i + kRad;
  constexpr int R = M::R, ZR = DIM == 3 ? R : 0;
  const float rc = p0->x, pc = p0->y;
  float mr = 0.0f, mp = 0.0f;
  for (int dz = -ZR; dz <= ZR; dz++)
    for (int dy = -R; dy <= R; dy++)
      for (int dx = -R; dx <= R; dx++) {
        const float2 q = p0[(dz * g.py + dy) * rpx + dx];
        mr = fmaxf(mr, fabsf(__fsub_rn(q.x, rc)));
        mp = fmaxf(mp, fabsf(__fsub_rn(q.y, pc)));
      }
  const float sr = mlp_scale(mr, rc), sp = mlp_scale(mp, pc);
  uint16_t *x = feats + t * M::NI;
  int q = 0;
  for (int dz = -ZR; dz <= ZR; dz++)
    for (int dy = -R; dy <= R; dy++)
      for (int dx = -R; dx <= R; dx++, q++) {
        const float2 v = p0[(dz * g.py + dy) * rpx + dx];
        x[q] = __bfloat16_as_ushort(__float2bfloat16_rn(mlp_feature(v.x, rc, sr)));
        x[M::P + q] = __bfloat16_as_ushort(__float2bfloat16_rn(mlp_feature(v.y, pc, sp)));
      }
  labels[t] = flags[c] >> 1;
  cells[t] = c;
}

// ---------------------------------------------------------------------------
// training: one block = kTrainB samples drawn uniformly (with replacement) from
// the collected set; forward and backward in FP32 with the BF16-rounded weights;
// the block's gradient of the weighted binary cross entropy goes to its own row
// of gpart and its loss to lpart (summed in block order by the Adam kernel, so a
// training run repeats bit for bit)
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
                     const float *__restrict__ w, float *__restrict__ gpart, float *__restrict__ lpart,
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
    LB[tid] = wt * (sp - y * z) * inv_batch;   // the label is not read again
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
    gpart[(int64_t)blockIdx.x * M::NW + t] = a;
  }
  if (tid == 0) {
    float l = 0.0f;
    for (int q = 0; q < kTrainB; q++) l += LB[q];
    lpart[blockIdx.x] = l;
  }
}

// Adam on the FP32 master weights with the gradient summed over the blocks'
// rows in block order; the forward passes use the weights' BF16 rounding
__global__ void __launch_bounds__(256)
    mlp_adam_kernel(float *__restrict__ master, float *__restrict__ m, float *__restrict__ v,
                    const float *__restrict__ gpart, const float *__restrict__ lpart, int blocks,
                    float *__restrict__ loss, float *__restrict__ wq, uint16_t *__restrict__ wb, int nw, float lr,
                    float c1, float c2) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0) {
    float l = 0.0f;
    for (int b = 0; b < blocks; b++) l += lpart[b];
    *loss += l;
  }
  if (t >= nw) return;
  float gr = 0.0f;
  for (int b = 0; b < blocks; b++) gr += gpart[(int64_t)b * nw + t];
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
// Density and pressure of every padded cell as an FP32 pair (the values the
// features are made of), row pitch rpx (even, so that rows of 8-byte pairs start
// on 16-byte boundaries for the TMA loads of the inference kernel).  Computed
// once per evaluation; every block of the inference kernel then loads its
// 36 x 8 x 5 halo tile of pairs (11.5 KB) instead of five FP64 variables.
template <int EQ>
__global__ void __launch_bounds__(256)
    mlp_rp_kernel(const double *__restrict__ U, Grid g, int64_t planes, int64_t rpx, float2 *__restrict__ rp) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= g.px * g.py * planes) return;
  const int64_t a = t % g.px, r = t / g.px;   // r = plane * py + row
  double u[Eos<EQ>::NV];
#pragma unroll
  for (int v = 0; v < Eos<EQ>::NV; v++) u[v] = U[v * g.pvol + t];
  rp[r * rpx + a] = make_float2((float)u[DENS], (float)Eos<EQ>::pres(g.gamma, u));
}

// ---------------------------------------------------------------------------
// Inference with both matrix layers on the tcgen05 tensor cores, per block of 128
// cells (two threads per cell = per row of the tiles, part 0 and part 1):
//   layer 1  D1 = A1 B1, A1 [128 x KP] the BF16 features, B1 = W1^T in BF16,
//            M128 N32 K16 MMAs (kind::f16), FP32 accumulation in TMEM columns 0-31.
//            The GEMM places density feature q in column q and pressure feature q
//            in column PAD + q (PAD = 32 in 2D, 128 in 3D), so that one 8-byte
//            read of the (density, pressure) pair of a patch cell gives both.
//   layer 2  D2 = A2 B2, A2 [128 x 32] = H1 = gelu(D1 + b1) split as tf32 hi + lo,
//            B2 = W2^T (BF16 values, exact in TF32), M128 N32 K8 MMAs (kind::tf32,
//            two per K step: hi and lo), FP32 accumulation in TMEM columns 32-63;
//            the product carries about 21 bits of H1, as the FP32 layer of
//            training does.
//   output   gelu(D2 + b2) . w3 + b3, each part summing 16 hidden units.
// Each cell block's halo tile of pairs arrives by one TMA load, issued while the
// previous cell block is processed.  Every mbarrier wait is bounded; on timeout
// the block sets DevScalars::fault, waits (bounded) for the loads it has in
// flight, frees its TMEM and returns.
constexpr int kMlpThreads = 256;

template <int DIM>
struct MlpTc {
  using M = MlpShape<DIM>;
  using Tl = MlpTile<DIM>;
  static constexpr int PAD = DIM == 2 ? 32 : 128;          // GEMM column of the first pressure feature
  static constexpr int KP = 2 * PAD;                       // layer-1 K
  static constexpr int NCH = KP / 8;                       // 16-byte chunks of 8 BF16 along K
  static constexpr int NQC = PAD / 8;                      // chunks of one quantity
  static constexpr int A_CH = 128 * 16;                    // one K chunk of a 128-row operand
  static constexpr int B_CH = 32 * 16;                     // one K chunk of a 32-row operand
  static constexpr int A1 = NCH * A_CH;
  static constexpr int A2 = 2 * 8 * A_CH;                  // H1 hi and lo: 32 K = 8 chunks of 4 tf32
  // the weight image in global memory (launch_mlp_pack), copied as two bulk loads:
  //   W1^T [k / 8][n][k % 8] BF16 | W2^T [k / 4][n][k % 4] FP32 | b1 b2 w3 b3 (+ 3 pad) FP32
  static constexpr int W1B = NCH * B_CH;
  static constexpr int W2B = 8 * B_CH;
  static constexpr int PRMB = 100 * 4;
  static constexpr int IMG_BYTES = W1B + W2B + PRMB;
  static constexpr int OFF_B1 = A1 > A2 ? A1 : A2;         // A1, then A2 in the same bytes
  static constexpr int OFF_B2 = OFF_B1 + W1B;
  static constexpr int OFF_W = OFF_B2 + W2B;
  static constexpr int OFF_TILE = (OFF_W + PRMB + 127) / 128 * 128;
  static constexpr int TILE_BYTES = (Tl::N * 8 + 127) / 128 * 128;   // one of the two tile buffers
  static constexpr int OFF_SUM = OFF_TILE + 2 * TILE_BYTES; // part 1's share of the output sum [128]
  static constexpr int OFF_BAR = OFF_SUM + 128 * 4;
  // scratch of the window extrema, in the A1 bytes before the features are written
  static constexpr int EXT_BYTES = (Tl::TY + kBlockY) * Tl::TX * 16;
  static constexpr int SMEM = OFF_BAR + 48;                // 4 barriers (MMA, weights, 2 tiles), TMEM slot
  static_assert(M::P <= PAD && NQC % 2 == 0, "pressure features start past the density ones");
  static_assert(OFF_TILE % 128 == 0 && OFF_B1 % 16 == 0 && OFF_B2 % 16 == 0, "TMA destination alignment");
  static_assert((W2B + PRMB) % 16 == 0 && W1B % 16 == 0, "bulk copy sizes");
  static_assert((Tl::TX * 8) % 16 == 0, "TMA box inner extent");
  static_assert(SMEM <= 113 * 1024, "two blocks per SM");
  static_assert(EXT_BYTES <= A1, "extrema scratch inside the A1 bytes");
};

// (max, min) of density and pressure: (max rho, min rho, max p, min p)
__device__ __forceinline__ float4 ext_of(float2 v) { return make_float4(v.x, v.x, v.y, v.y); }
__device__ __forceinline__ float4 ext_merge(float4 e, float4 f) {
  return make_float4(fmaxf(e.x, f.x), fminf(e.y, f.y), fmaxf(e.z, f.z), fminf(e.w, f.w));
}

// a (density, pressure) feature pair (q - q_c) s, both components at once: the
// packed FP32 sub.rn / mul.rn round each component as __fsub_rn / __fmul_rn do
__device__ __forceinline__ float2 mlp_feature2(float2 v, float2 c, float2 s) {
  uint64_t d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(*reinterpret_cast<const uint64_t *>(&v)),
      "l"(*reinterpret_cast<const uint64_t *>(&c)));
  asm("mul.rn.f32x2 %0, %0, %1;" : "+l"(d) : "l"(*reinterpret_cast<const uint64_t *>(&s)));
  return *reinterpret_cast<const float2 *>(&d);
}

// the layer-1 operand rows of one cell, chunks cq = PART, PART + 2, ...: every loop
// is unrolled, so each patch offset is a constant of the shared-memory load
template <int DIM, int PART>
__device__ __forceinline__ void mlp_features(const float2 *__restrict__ tc, float2 ref, float2 scl, bool live,
                                             uint32_t aB, int row) {
  using M = MlpShape<DIM>;
  using Tl = MlpTile<DIM>;
  using C = MlpTc<DIM>;
  constexpr int ZR = DIM == 3 ? Tl::R : 0;
#pragma unroll
  for (int cq = PART; cq < C::NQC; cq += 2) {
    uint32_t pr[4], pp[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      float2 x[2];
#pragma unroll
      for (int e = 0; e < 2; e++) {
        const int q = cq * 8 + 2 * u + e;
        x[e] = make_float2(0.0f, 0.0f);
        if (q < M::P) {
          const int dx = q % M::SIDE - Tl::R, dy = (q / M::SIDE) % M::SIDE - Tl::R,
                    dz = q / (M::SIDE * M::SIDE) - ZR;
          x[e] = mlp_feature2(tc[(dz * Tl::TY + dy) * Tl::TX + dx], ref, scl);
        }
      }
      const __nv_bfloat162 br = __floats2bfloat162_rn(x[0].x, x[1].x); // .x low half, .y high half
      const __nv_bfloat162 bp = __floats2bfloat162_rn(x[0].y, x[1].y);
      pr[u] = live ? *reinterpret_cast<const uint32_t *>(&br) : 0u;
      pp[u] = live ? *reinterpret_cast<const uint32_t *>(&bp) : 0u;
    }
    st_shared_v4(aB + cq * C::A_CH + row * 16, pr);
    st_shared_v4(aB + (C::NQC + cq) * C::A_CH + row * 16, pp);
  }
}

// the weight image of the inference kernel: W1^T in the layer-1 B layout
// [k / 8][n][k % 8] (k the GEMM column), then W2^T as FP32 in the layer-2 B layout
// [k / 4][n][k % 4], then b1, b2, w3, b3 as FP32
template <int DIM>
__global__ void __launch_bounds__(256)
    mlp_pack_kernel(const uint16_t *__restrict__ wb, const float *__restrict__ wq, uint8_t *__restrict__ img) {
  using M = MlpShape<DIM>;
  using C = MlpTc<DIM>;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < 32 * C::KP) {
    const int n = t / C::KP, k = t % C::KP;
    const int q = k < C::PAD ? k : k - C::PAD;
    const int f = k < C::PAD ? q : M::P + q;               // network input of this column
    reinterpret_cast<uint16_t *>(img)[(k / 8) * 256 + n * 8 + (k % 8)] =
        q < M::P ? wb[M::W1 + n * M::NI + f] : (uint16_t)0;
  }
  float *w2 = reinterpret_cast<float *>(img + C::W1B);
  if (t < M::NH * M::NH) {
    const int n = t / M::NH, kk = t % M::NH;
    w2[(kk / 4) * 128 + n * 4 + (kk % 4)] = wq[M::W2 + n * M::NH + kk];
  }
  float *prm = reinterpret_cast<float *>(img + C::W1B + C::W2B);
  if (t < 32) {
    prm[t] = wq[M::B1 + t];
    prm[32 + t] = wq[M::B2 + t];
    prm[64 + t] = wq[M::W3 + t];
  }
  if (t < 4) prm[96 + t] = t == 0 ? wq[M::B3] : 0.0f;
}

// mode 0: flags (+ prediction, flagged count); mode 1: probabilities.
// Persistent: each block allocates its TMEM and loads the weight image once, then
// takes the cell blocks b = blockIdx.x, blockIdx.x + gridDim.x, ... (nbx x nby x nz
// of them, x fastest), with the next one's halo tile already on its way by TMA
// into the other tile buffer.
template <int DIM, int EQ, int MODE>
__global__ void __launch_bounds__(kMlpThreads, DIM == 2 ? 4 : 2)
    mlp_tc_kernel(const __grid_constant__ CUtensorMap rpMap, Grid g, const uint8_t *__restrict__ img,
                  const double *__restrict__ theta, uint8_t *__restrict__ flag, uint8_t *__restrict__ pred,
                  float *__restrict__ prob, DevScalars *__restrict__ sc, float logit_thr, int nbx, int nby,
                  int nblk) {
  using M = MlpShape<DIM>;
  using Tl = MlpTile<DIM>;
  using C = MlpTc<DIM>;
  extern __shared__ __align__(128) uint8_t msm[];
  const float *sW = reinterpret_cast<const float *>(msm + C::OFF_W);   // b1 [32], b2 [32], w3 [32], b3
  float *sSum = reinterpret_cast<float *>(msm + C::OFF_SUM);
  uint64_t *bar = reinterpret_cast<uint64_t *>(msm + C::OFF_BAR);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(msm + C::OFF_BAR + 32);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int quarter = warp & 3, part = warp >> 2;
  const int row = quarter * 32 + lane;
  // barriers: MMA completion, weight image, tile buffer 0, tile buffer 1
  const uint32_t barA = smem_u32(bar), barW = barA + 8, barT0 = barA + 16;
  constexpr uint32_t kTileBytes = (uint32_t)(Tl::N * sizeof(float2));
  auto tile_load = [&](int b, int buf) {   // thread 0: the halo tile of cell block b
    const int bx = b % nbx, by = (b / nbx) % nby, bz = b / (nbx * nby);
    const uint32_t tb = barT0 + 8u * (uint32_t)buf;
    mbar_arrive_expect_tx(tb, kTileBytes);
    // padded coordinates of the tile's first cell: i0 - R, j0 - R, k - R in cells
    tma_load_3d(smem_u32(msm + C::OFF_TILE + buf * C::TILE_BYTES), &rpMap, bx * kBlockX, by * kBlockY, bz, tb);
  };
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(64u)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  // loads in flight per tile buffer and the parity of each buffer's next phase
  // (kept by thread 0, which issues the loads, for the exit path)
  uint32_t inflight = 0u, tpar = 0u;   // bit q: buffer q
  if (tid == 0) {
    mbar_init(barA, 1);
    mbar_init(barW, 1);
    mbar_init(barT0, 1);
    mbar_init(barT0 + 8, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    mbar_arrive_expect_tx(barW, (uint32_t)C::IMG_BYTES);
    bulk_load(smem_u32(msm + C::OFF_B1), img, C::W1B, barW);
    bulk_load(smem_u32(msm + C::OFF_B2), img + C::W1B, C::W2B + C::PRMB, barW);
    if ((int)blockIdx.x < nblk) {
      tile_load(blockIdx.x, 0);
      inflight = 1u;
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  bool ok = __syncthreads_and(mbar_wait(barW, 0u));
  constexpr int ZR = DIM == 3 ? Tl::R : 0;
  const int c0 = (ZR * Tl::TY + quarter + Tl::R) * Tl::TX + lane + Tl::R;
  const uint32_t aB = smem_u32(msm), b1B = smem_u32(msm + C::OFF_B1), b2B = smem_u32(msm + C::OFF_B2);
  const uint32_t lanes = (uint32_t)(quarter * 32) << 16;
  int it = 0;
  for (int b = blockIdx.x; ok && b < nblk; b += gridDim.x, it++) {
    const int buf = it & 1;
    // the next cell block's tile goes into the other buffer, whose last reads ended
    // before the closing barrier of the previous iteration
    if (tid == 0 && b + (int)gridDim.x < nblk) {
      tile_load(b + gridDim.x, buf ^ 1);
      inflight |= 1u << (buf ^ 1);
    }
    const bool got = mbar_wait(barT0 + 8u * (uint32_t)buf, (uint32_t)((it >> 1) & 1));
    if (tid == 0 && got) {
      inflight &= ~(1u << buf);
      tpar ^= 1u << buf;
    }
    ok = __syncthreads_and(got);
    if (!ok) break;
    // the cell block's halo tile of (density, pressure) pairs, [z][y][x] as the TMA box lands
    const float2 *tile = reinterpret_cast<const float2 *>(msm + C::OFF_TILE + buf * C::TILE_BYTES);
    const int bx = b % nbx, by = (b / nbx) % nby, bz = b / (nbx * nby);
    const int64_t i = (int64_t)bx * kBlockX + lane, j = (int64_t)by * kBlockY + quarter, k = bz;
    const bool live = i < g.nx && j < g.ny;
    const int64_t c = (k * g.ny + j) * g.nx + i;
    // the positivity history of the cell, read now so that the load overlaps the features
    const double th = MODE == 0 && part == 0 && live ? theta[c] : 1.0;
    // window extrema of the patches, separably along z, y and x, in scratch that
    // the A1 bytes hold until the features are written
    float4 *ez = reinterpret_cast<float4 *>(msm);           // [TY][TX] after z
    float4 *ey = ez + Tl::TY * Tl::TX;                      // [kBlockY][TX] after y
    if (DIM == 3) {
      for (int n = tid; n < Tl::TY * Tl::TX; n += kMlpThreads) {
        float4 e = ext_of(tile[n]);
#pragma unroll
        for (int dz = 1; dz < Tl::TZ; dz++) e = ext_merge(e, ext_of(tile[dz * Tl::TY * Tl::TX + n]));
        ez[n] = e;
      }
      __syncthreads();
    }
    for (int n = tid; n < kBlockY * Tl::TX; n += kMlpThreads) {
      float4 e = DIM == 3 ? ez[n] : ext_of(tile[n]);
#pragma unroll
      for (int dy = 1; dy < MlpShape<DIM>::SIDE; dy++)
        e = ext_merge(e, DIM == 3 ? ez[dy * Tl::TX + n] : ext_of(tile[dy * Tl::TX + n]));
      ey[n] = e;
    }
    __syncthreads();
    const float2 ref = tile[c0];
    float2 scl;
    {
      float4 e = ey[quarter * Tl::TX + lane];
#pragma unroll
      for (int dx = 1; dx < MlpShape<DIM>::SIDE; dx++) e = ext_merge(e, ey[quarter * Tl::TX + lane + dx]);
      // rounding is monotonic, so max_k |fl(q_k - q_c)| = max(fl(max q - q_c), fl(q_c - min q))
      scl.x = mlp_scale(fmaxf(__fsub_rn(e.x, ref.x), __fsub_rn(ref.x, e.y)), ref.x);
      scl.y = mlp_scale(fmaxf(__fsub_rn(e.z, ref.y), __fsub_rn(ref.y, e.w)), ref.y);
    }
    __syncthreads();   // the scratch is overwritten by the features
    // features: chunk cq of 8 patch cells gives density chunk cq and pressure
    // chunk NQC + cq; the parts take alternate chunks
    if (part == 0)
      mlp_features<DIM, 0>(tile + c0, ref, scl, live, aB, row);
    else
      mlp_features<DIM, 1>(tile + c0, ref, scl, live, aB, row);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      constexpr uint32_t idesc1 = bf16_idesc<32>();
#pragma unroll 1
      for (int s = 0; s < C::NCH / 2; s++) {
        const uint64_t ad = umma_desc(aB + 2 * s * C::A_CH, C::A_CH, 128);
        const uint64_t bd = umma_desc(b1B + 2 * s * C::B_CH, C::B_CH, 128);
        mma_bf16(tmem, ad, bd, idesc1, s > 0 ? 1 : 0);
      }
      mma_commit(barA);
    }
    ok = __syncthreads_and(mbar_wait(barA, 0u));   // two commits per cell block: parity 0, then 1
    if (!ok) break;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    {
      // H1 = gelu(D1 + b1) of this part's 16 hidden units, split hi + lo into A2
      float z[16];
      tmem_ld8(tmem + lanes + (uint32_t)(16 * part), *reinterpret_cast<float(*)[8]>(z));
      tmem_ld8(tmem + lanes + (uint32_t)(16 * part + 8), *reinterpret_cast<float(*)[8]>(z + 8));
      const uint32_t aHi = aB, aLo = aB + 8 * C::A_CH;
#pragma unroll
      for (int c = 0; c < 4; c++) {
        uint32_t hi[4], lo[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const int h = 16 * part + 4 * c + u;
          const float x = gelu(z[4 * c + u] + sW[h]);
          hi[u] = to_tf32(x);
          lo[u] = to_tf32(x - __uint_as_float(hi[u]));
        }
        st_shared_v4(aHi + (4 * part + c) * C::A_CH + row * 16, hi);
        st_shared_v4(aLo + (4 * part + c) * C::A_CH + row * 16, lo);
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      constexpr uint32_t idesc2 = tf32_idesc<32>();
      const uint32_t aHi = aB, aLo = aB + 8 * C::A_CH;
#pragma unroll
      for (int s = 0; s < 4; s++) {
        const uint64_t bd = umma_desc(b2B + 2 * s * C::B_CH, C::B_CH, 128);
        mma_tf32(tmem + 32, umma_desc(aLo + 2 * s * C::A_CH, C::A_CH, 128), bd, idesc2, s > 0 ? 1 : 0);
        mma_tf32(tmem + 32, umma_desc(aHi + 2 * s * C::A_CH, C::A_CH, 128), bd, idesc2, 1);
      }
      mma_commit(barA);
    }
    ok = __syncthreads_and(mbar_wait(barA, 1u));
    if (!ok) break;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    float z[16];
    tmem_ld8(tmem + lanes + (uint32_t)(32 + 16 * part), *reinterpret_cast<float(*)[8]>(z));
    tmem_ld8(tmem + lanes + (uint32_t)(32 + 16 * part + 8), *reinterpret_cast<float(*)[8]>(z + 8));
    float acc = 0.0f;
#pragma unroll
    for (int u = 0; u < 16; u++) {
      const int o = 16 * part + u;
      acc = fmaf(sW[64 + o], gelu(z[u] + sW[32 + o]), acc);
    }
    if (part == 1) sSum[row] = acc;
    __syncthreads();
    if (part == 0) {
      bool f = false;
      if (live) {
        const float logit = sW[96] + acc + sSum[row];
        if (MODE == 0) {
          const bool p = logit > logit_thr;
          pred[c] = p ? 1 : 0;
          f = p || th < 1.0;
          flag[c] = f ? 1 : 0;
        } else {
          prob[c] = 1.0f / (1.0f + expf(-logit));
        }
      }
      if (MODE == 0) {
        const unsigned ball = __ballot_sync(0xffffffffu, f);
        if (lane == 0 && ball) atomicAdd(&sc->nflag, (unsigned)__popc(ball));
      }
    }
    // the tile buffer, the A bytes, sSum and TMEM are reused by the next cell block
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
  }
  if (!ok && tid == 0) {
    atomicExch(&sc->fault, 1u);
    // the weight image and tile loads still in flight land before the block leaves
    // (bounded waits; a completed phase returns at once)
    mbar_wait(barW, 0u);
    for (int q = 0; q < 2; q++)
      if ((inflight >> q) & 1u) mbar_wait(barT0 + 8u * (uint32_t)q, (tpar >> q) & 1u);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(64u) : "memory");
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
static cudaError_t label_t(const double *U, const Grid &g, const DevStencil *S, double tau, double keep,
                           uint64_t seed, uint8_t *flags, cudaStream_t s) {
  mlp_label_kernel<DIM, EQ><<<(unsigned)((g.n + 255) / 256), 256, 0, s>>>(U, g, S, tau, keep, seed, flags);
  return cudaGetLastError();
}

template <int DIM, int EQ>
static cudaError_t rp_t(const double *U, const Grid &g, float2 *rp, int64_t rpx, cudaStream_t s) {
  const int64_t planes = DIM == 3 ? g.nz + 2 * kRad : 1;
  const int64_t np = g.px * g.py * planes;
  mlp_rp_kernel<EQ><<<(unsigned)((np + 255) / 256), 256, 0, s>>>(U, g, planes, rpx, rp);
  return cudaGetLastError();
}

template <int DIM, int EQ, int MODE>
static cudaError_t tc_t(const double *U, const Grid &g, float2 *rp, int64_t rpx, const CUtensorMap &map,
                        const uint8_t *img, const double *theta, uint8_t *flag, uint8_t *pred, float *prob,
                        DevScalars *sc, float thr, cudaStream_t s) {
  using C = MlpTc<DIM>;
  // set once per process (a function-local static is initialised once, also when
  // several host threads drive solvers)
  static const cudaError_t attr =
      cudaFuncSetAttribute(mlp_tc_kernel<DIM, EQ, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM);
  if (attr != cudaSuccess) return attr;
  const int64_t planes = DIM == 3 ? g.nz + 2 * kRad : 1;
  const int64_t np = g.px * g.py * planes;
  mlp_rp_kernel<EQ><<<(unsigned)((np + 255) / 256), 256, 0, s>>>(U, g, planes, rpx, rp);
  const dim3 cb = mlp_cell_grid(g);
  const int nblk = (int)(cb.x * cb.y * cb.z);
  // as many blocks as are resident at once: the SM's shared memory and registers
  // divided by one block's (2 per SM in 3D, by shared memory; 4 in 2D); computed from
  // the device's limits with the largest shared-memory carveout requested
  static const int per_sm = [] {
    cudaFuncAttributes fa;
    int dev = 0, smem_sm = 0, smem_rsv = 0, regs_sm = 0;
    if (cudaFuncSetAttribute(mlp_tc_kernel<DIM, EQ, MODE>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             (int)cudaSharedmemCarveoutMaxShared) != cudaSuccess ||
        cudaFuncGetAttributes(&fa, mlp_tc_kernel<DIM, EQ, MODE>) != cudaSuccess || cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&smem_rsv, cudaDevAttrReservedSharedMemoryPerBlock, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev) != cudaSuccess)
      return 0;
    const int warp_regs = (fa.numRegs * 32 + 255) / 256 * 256;   // allocated per warp in units of 256
    const int by_smem = smem_sm / (C::SMEM + (int)fa.sharedSizeBytes + smem_rsv);
    const int by_regs = regs_sm / (warp_regs * (kMlpThreads / 32));
    return std::min(by_smem, by_regs);
  }();
  static const int nsm = [] {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      return 0;
    return n;
  }();
  if (per_sm <= 0 || nsm <= 0) return cudaErrorInvalidConfiguration;
  const int grid = std::min(nblk, per_sm * nsm);
  mlp_tc_kernel<DIM, EQ, MODE><<<grid, kMlpThreads, C::SMEM, s>>>(map, g, img, theta, flag, pred, prob, sc, thr,
                                                                 (int)cb.x, (int)cb.y, nblk);
  return cudaGetLastError();
}

template <int DIM, int EQ>
static cudaError_t flag_t(const double *U, const Grid &g, float2 *rp, int64_t rpx, const CUtensorMap &map,
                          const uint8_t *img, const double *theta, uint8_t *flag, uint8_t *pred, DevScalars *sc,
                          float thr, cudaStream_t s) {
  return tc_t<DIM, EQ, 0>(U, g, rp, rpx, map, img, theta, flag, pred, nullptr, sc, thr, s);
}

template <int DIM, int EQ>
static cudaError_t prob_t(const double *U, const Grid &g, float2 *rp, int64_t rpx, const CUtensorMap &map,
                          const uint8_t *img, float *out, DevScalars *sc, cudaStream_t s) {
  return tc_t<DIM, EQ, 1>(U, g, rp, rpx, map, img, nullptr, nullptr, nullptr, out, sc, 0.0f, s);
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

size_t mlp_select_temp_bytes(int64_t n) {
  size_t bytes = 0;
  cub::DeviceSelect::Flagged(nullptr, bytes, thrust::counting_iterator<int64_t>(0), (const uint8_t *)nullptr,
                             (int64_t *)nullptr, (int64_t *)nullptr, n);
  return bytes;
}

cudaError_t launch_mlp_select(int dim, int eq, const double *U, const Grid &g, const DevStencil *S, double tau,
                              double keep, uint64_t seed, const MlpTileBuf &tb, uint8_t *flags, int64_t *sel,
                              int64_t *nsel, void *temp, size_t temp_bytes, cudaStream_t s) {
  cudaError_t e;
  auto labels = [&]() -> cudaError_t { KFVM_MLP_DISPATCH(dim, eq, label_t, U, g, S, tau, keep, seed, flags, s); };
  auto pairs = [&]() -> cudaError_t { KFVM_MLP_DISPATCH(dim, eq, rp_t, U, g, tb.rp, tb.rpx, s); };
  if ((e = labels()) != cudaSuccess || (e = pairs()) != cudaSuccess) return e;
  return cub::DeviceSelect::Flagged(temp, temp_bytes, thrust::counting_iterator<int64_t>(0), flags, sel, nsel, g.n,
                                    s);
}

cudaError_t launch_mlp_features(int dim, const Grid &g, const MlpTileBuf &tb, const int64_t *sel, int64_t count,
                                const uint8_t *flags, uint16_t *feats, uint8_t *labels, int64_t *cells,
                                cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  const unsigned blocks = (unsigned)((count + 127) / 128);
  if (dim == 2) mlp_feature_kernel<2><<<blocks, 128, 0, s>>>(tb.rp, tb.rpx, g, sel, count, flags, feats, labels, cells);
  else mlp_feature_kernel<3><<<blocks, 128, 0, s>>>(tb.rp, tb.rpx, g, sel, count, flags, feats, labels, cells);
  return cudaGetLastError();
}

cudaError_t launch_mlp_flag(int dim, int eq, const double *U, const Grid &g, const MlpTileBuf &tb, const uint8_t *img,
                            const double *theta, uint8_t *flag, uint8_t *pred, DevScalars *sc, float logit_thr,
                            cudaStream_t s) {
  KFVM_MLP_DISPATCH(dim, eq, flag_t, U, g, tb.rp, tb.rpx, tb.map, img, theta, flag, pred, sc, logit_thr, s);
}

cudaError_t launch_mlp_prob(int dim, int eq, const double *U, const Grid &g, const MlpTileBuf &tb, const uint8_t *img,
                            float *out, DevScalars *sc, cudaStream_t s) {
  KFVM_MLP_DISPATCH(dim, eq, prob_t, U, g, tb.rp, tb.rpx, tb.map, img, out, sc, s);
}

// ---------------------------------------------------------------------------
// the (density, pressure) pair array and the tensor map of its halo tiles
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

int encode_tensor_map_8b(CUtensorMap *map, const void *base, int rank, const uint64_t *dims,
                         const uint64_t *strides_bytes, const uint32_t *box) {
  // looked up once (a function-local static is initialised once, also when several
  // host threads drive solvers)
  static const EncodeTiledFn fn = []() -> EncodeTiledFn {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return nullptr;
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  if (!fn) return -1;
  if (reinterpret_cast<uintptr_t>(base) % 16 != 0) return -2;
  cuuint64_t d[5], st[4];
  cuuint32_t bx[5], es[5];
  for (int r = 0; r < rank; r++) {
    d[r] = dims[r];
    bx[r] = box[r];
    es[r] = 1;
    if (r > 0) {
      if (strides_bytes[r - 1] % 16 != 0) return -3;
      st[r - 1] = strides_bytes[r - 1];
    }
  }
  if ((box[0] * 8) % 16 != 0) return -4;
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, (cuuint32_t)rank, const_cast<void *>(base), d, st, bx,
                        es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : -5;
}

cudaError_t mlp_tile_buf_init(int dim, const Grid &g, MlpTileBuf &tb) {
  const int64_t planes = dim == 3 ? g.nz + 2 * kRad : 1;
  tb.rpx = (g.px + 1) / 2 * 2;  // even: every row starts on a 16-byte boundary
  cudaError_t e = cudaMalloc((void **)&tb.rp, (size_t)(tb.rpx * g.py * planes) * sizeof(float2));
  if (e != cudaSuccess) return e;
  const uint64_t dims[3] = {(uint64_t)g.px, (uint64_t)g.py, (uint64_t)planes};
  const uint64_t strides[2] = {(uint64_t)(tb.rpx * 8), (uint64_t)(tb.rpx * g.py * 8)};
  const uint32_t box[3] = {dim == 3 ? (uint32_t)MlpTile<3>::TX : (uint32_t)MlpTile<2>::TX,
                           dim == 3 ? (uint32_t)MlpTile<3>::TY : (uint32_t)MlpTile<2>::TY,
                           dim == 3 ? (uint32_t)MlpTile<3>::TZ : (uint32_t)MlpTile<2>::TZ};
  if (encode_tensor_map_8b(&tb.map, tb.rp, 3, dims, strides, box) != 0) return cudaErrorInvalidValue;
  return cudaSuccess;
}

int mlp_image_bytes(int dim) { return dim == 2 ? MlpTc<2>::IMG_BYTES : MlpTc<3>::IMG_BYTES; }

cudaError_t launch_mlp_pack(int dim, const uint16_t *wb, const float *wq, uint8_t *img, cudaStream_t s) {
  const int n = dim == 2 ? 32 * MlpTc<2>::KP : 32 * MlpTc<3>::KP;   // at least the 1024 W2 entries
  if (dim == 2) mlp_pack_kernel<2><<<(n + 255) / 256, 256, 0, s>>>(wb, wq, img);
  else mlp_pack_kernel<3><<<(n + 255) / 256, 256, 0, s>>>(wb, wq, img);
  return cudaGetLastError();
}

cudaError_t launch_mlp_train_step(int dim, const uint16_t *feats, const uint8_t *labels, int64_t n, int batch,
                                  float *master, float *m, float *v, float *gpart, float *lpart, float *wq,
                                  uint16_t *wb, float *loss, float pos_weight, float lr, int t, uint64_t seed,
                                  cudaStream_t s) {
  const int blocks = mlp_train_blocks(batch);
  const float inv = 1.0f / (float)(blocks * kTrainB);
  cudaError_t e;
  if (dim == 2) {
    static const cudaError_t attr = cudaFuncSetAttribute(
        mlp_train_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TrainSmem<2>::BYTES);
    if (attr != cudaSuccess) return attr;
    mlp_train_kernel<2><<<blocks, 256, TrainSmem<2>::BYTES, s>>>(feats, labels, n, wq, gpart, lpart, pos_weight,
                                                                 inv, seed, t);
  } else {
    static const cudaError_t attr = cudaFuncSetAttribute(
        mlp_train_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TrainSmem<3>::BYTES);
    if (attr != cudaSuccess) return attr;
    mlp_train_kernel<3><<<blocks, 256, TrainSmem<3>::BYTES, s>>>(feats, labels, n, wq, gpart, lpart, pos_weight,
                                                                 inv, seed, t);
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  const int nw = mlp_num_weights(dim);
  const float c1 = 1.0f / (1.0f - powf(0.9f, (float)t)), c2 = 1.0f / (1.0f - powf(0.999f, (float)t));
  mlp_adam_kernel<<<(nw + 255) / 256, 256, 0, s>>>(master, m, v, gpart, lpart, blocks, loss, wq, wb, nw, lr, c1,
                                                   c2);
  return cudaGetLastError();
}

int mlp_train_blocks(int batch) { return (batch + kTrainB - 1) / kTrainB; }

} // namespace kfvm
