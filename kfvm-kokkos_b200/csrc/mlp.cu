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
  __shared__ double tile[2][Tl::N];
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
  double rc, pc, sr, sp;
  mlp_scales<DIM>(tile, threadIdx.x, threadIdx.y, rc, pc, sr, sp);
  constexpr int R = Tl::R, ZR = DIM == 3 ? R : 0;
  const int c0 = (ZR * Tl::TY + threadIdx.y + R) * Tl::TX + threadIdx.x + R;
  uint16_t *x = feats + (int64_t)idx * M::NI;
  int q = 0;
  for (int dz = -ZR; dz <= ZR; dz++)
    for (int dy = -R; dy <= R; dy++)
      for (int dx = -R; dx <= R; dx++, q++) {
        const int n = c0 + (dz * Tl::TY + dy) * Tl::TX + dx;
        x[q] = __bfloat16_as_ushort(__float2bfloat16_rn((float)((tile[0][n] - rc) * sr)));
        x[M::P + q] = __bfloat16_as_ushort(__float2bfloat16_rn((float)((tile[1][n] - pc) * sp)));
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

// BF16 weights -> FP32, W1 transposed to [input][hidden] for the per-cell pass
template <int DIM>
__device__ __forceinline__ void mlp_stage_weights(const uint16_t *__restrict__ wb, float *__restrict__ sw) {
  using M = MlpShape<DIM>;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x, nt = blockDim.x * blockDim.y;
  for (int t = tid; t < M::NW; t += nt) {
    const float x = __bfloat162float(__ushort_as_bfloat16(wb[t]));
    if (t < M::B1) sw[(t % M::NI) * M::NH + t / M::NI] = x;
    else sw[t] = x;
  }
}

// network logit of the cell at block position (tx, ty), features from the tile;
// the first layer sums the density inputs, then the pressure inputs, in order
template <int DIM>
__device__ __forceinline__ float mlp_cell_logit(const double (*t)[MlpTile<DIM>::N], int tx, int ty,
                                                const float *__restrict__ sw) {
  using M = MlpShape<DIM>;
  using Tl = MlpTile<DIM>;
  constexpr int R = Tl::R, ZR = DIM == 3 ? R : 0;
  double rc, pc, sr, sp;
  mlp_scales<DIM>(t, tx, ty, rc, pc, sr, sp);
  const int c0 = (ZR * Tl::TY + ty + R) * Tl::TX + tx + R;
  float z[M::NH];
#pragma unroll
  for (int h = 0; h < M::NH; h++) z[h] = sw[M::B1 + h];
#pragma unroll 1
  for (int a = 0; a < 2; a++) {
    const double ref = a == 0 ? rc : pc, sc = a == 0 ? sr : sp;
    int q = a * M::P;
    for (int dz = -ZR; dz <= ZR; dz++)
      for (int dy = -R; dy <= R; dy++)
#pragma unroll
        for (int dx = -R; dx <= R; dx++, q++) {
          const float x = (float)((t[a][c0 + (dz * Tl::TY + dy) * Tl::TX + dx] - ref) * sc);
          const float4 *wr = reinterpret_cast<const float4 *>(sw + q * M::NH);
#pragma unroll
          for (int h4 = 0; h4 < M::NH / 4; h4++) {
            const float4 wv = wr[h4];
            z[4 * h4 + 0] = fmaf(wv.x, x, z[4 * h4 + 0]);
            z[4 * h4 + 1] = fmaf(wv.y, x, z[4 * h4 + 1]);
            z[4 * h4 + 2] = fmaf(wv.z, x, z[4 * h4 + 2]);
            z[4 * h4 + 3] = fmaf(wv.w, x, z[4 * h4 + 3]);
          }
        }
  }
#pragma unroll
  for (int h = 0; h < M::NH; h++) z[h] = gelu(z[h]);
  float out = sw[M::B3];
#pragma unroll 4
  for (int o = 0; o < M::NH; o++) {
    float a = sw[M::B2 + o];
    const float *wr = sw + M::W2 + o * M::NH;
#pragma unroll
    for (int h = 0; h < M::NH; h++) a = fmaf(wr[h], z[h], a);
    out = fmaf(sw[M::W3 + o], gelu(a), out);
  }
  return out;
}

template <int DIM>
struct FlagSmem {
  static constexpr size_t TILE = 2 * MlpTile<DIM>::N * sizeof(double);
  static constexpr size_t BYTES = TILE + MlpShape<DIM>::NW * sizeof(float);
};

// inference in the stage: flag = network says troubled, or theta < 1 (the
// positivity history rule of WenoSelect_K); pred keeps the network's answer for
// the judge; the flagged count feeds the flag-set semantics as in flag_kernel
template <int DIM, int EQ>
__global__ void __launch_bounds__(128)
    mlp_flag_kernel(const double *__restrict__ U, Grid g, const uint16_t *__restrict__ wb,
                    const double *__restrict__ theta, uint8_t *__restrict__ flag, uint8_t *__restrict__ pred,
                    DevScalars *__restrict__ sc, float logit_thr) {
  using Tl = MlpTile<DIM>;
  extern __shared__ __align__(16) unsigned char fsm[];
  double(*tile)[Tl::N] = reinterpret_cast<double(*)[Tl::N]>(fsm);
  float *sw = reinterpret_cast<float *>(fsm + FlagSmem<DIM>::TILE);
  const int64_t i0 = blockIdx.x * (int64_t)kBlockX, j0 = blockIdx.y * (int64_t)kBlockY, k = blockIdx.z;
  mlp_stage_weights<DIM>(wb, sw);
  mlp_tile_fill<DIM, EQ>(U, g, i0, j0, k, tile);
  __syncthreads();
  const int64_t i = i0 + threadIdx.x, j = j0 + threadIdx.y;
  bool f = false;
  if (i < g.nx && j < g.ny) {
    const int64_t c = (k * g.ny + j) * g.nx + i;
    const bool p = mlp_cell_logit<DIM>(tile, threadIdx.x, threadIdx.y, sw) > logit_thr;
    pred[c] = p ? 1 : 0;
    f = p || theta[c] < 1.0;
    flag[c] = f ? 1 : 0;
  }
  const unsigned ball = __ballot_sync(0xffffffffu, f);
  if ((threadIdx.x & 31) == 0 && ball) atomicAdd(&sc->nflag, (unsigned)__popc(ball));
}

// probability of every cell (inspection and tests)
template <int DIM, int EQ>
__global__ void __launch_bounds__(128)
    mlp_prob_kernel(const double *__restrict__ U, Grid g, const uint16_t *__restrict__ wb, float *__restrict__ out) {
  using Tl = MlpTile<DIM>;
  extern __shared__ __align__(16) unsigned char fsm[];
  double(*tile)[Tl::N] = reinterpret_cast<double(*)[Tl::N]>(fsm);
  float *sw = reinterpret_cast<float *>(fsm + FlagSmem<DIM>::TILE);
  const int64_t i0 = blockIdx.x * (int64_t)kBlockX, j0 = blockIdx.y * (int64_t)kBlockY, k = blockIdx.z;
  mlp_stage_weights<DIM>(wb, sw);
  mlp_tile_fill<DIM, EQ>(U, g, i0, j0, k, tile);
  __syncthreads();
  const int64_t i = i0 + threadIdx.x, j = j0 + threadIdx.y;
  if (i >= g.nx || j >= g.ny) return;
  const float z = mlp_cell_logit<DIM>(tile, threadIdx.x, threadIdx.y, sw);
  out[(k * g.ny + j) * g.nx + i] = 1.0f / (1.0f + expf(-z));
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

template <int DIM, int EQ>
static cudaError_t flag_t(const double *U, const Grid &g, const uint16_t *wb, const double *theta, uint8_t *flag,
                          uint8_t *pred, DevScalars *sc, float thr, cudaStream_t s) {
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(mlp_flag_kernel<DIM, EQ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)FlagSmem<DIM>::BYTES);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  mlp_flag_kernel<DIM, EQ><<<mlp_cell_grid(g), dim3(kBlockX, kBlockY), FlagSmem<DIM>::BYTES, s>>>(
      U, g, wb, theta, flag, pred, sc, thr);
  return cudaGetLastError();
}

template <int DIM, int EQ>
static cudaError_t prob_t(const double *U, const Grid &g, const uint16_t *wb, float *out, cudaStream_t s) {
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(mlp_prob_kernel<DIM, EQ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)FlagSmem<DIM>::BYTES);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  mlp_prob_kernel<DIM, EQ><<<mlp_cell_grid(g), dim3(kBlockX, kBlockY), FlagSmem<DIM>::BYTES, s>>>(U, g, wb, out);
  return cudaGetLastError();
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
                            const double *theta, uint8_t *flag, uint8_t *pred, DevScalars *sc, float logit_thr,
                            cudaStream_t s) {
  KFVM_MLP_DISPATCH(dim, eq, flag_t, U, g, wb, theta, flag, pred, sc, logit_thr, s);
}

cudaError_t launch_mlp_prob(int dim, int eq, const double *U, const Grid &g, const uint16_t *wb, float *out,
                            cudaStream_t s) {
  KFVM_MLP_DISPATCH(dim, eq, prob_t, U, g, wb, out, s);
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
