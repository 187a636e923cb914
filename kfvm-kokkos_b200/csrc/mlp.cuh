// mlp.cuh -- the learned troubled-cell indicator: shapes, weight layout and the
// per-block density / pressure tile its features are read from.
//
// Input: the normalised (2r+1)^d patch (r = 2) of density and pressure around a
// cell, giving 50 inputs in 2D and 250 in 3D (density first, patch cells in
// (z, y, x) order, x fastest).  With q = rho or p (computed in FP64, rounded to
// FP32) and every operation below in FP32:
//   d_k = q_k - q_c,  s = 1 / (max_k |d_k| + 1e-4 |q_c|),  x_k = d_k s,
// then rounded to BF16, the operand type of the network.  Network: NI -> 32 -> 32 -> 1, GELU (tanh
// approximation, gelu below) after both hidden layers, sigmoid output.  Weights are BF16 (raw uint16 at the C ABI), every sum
// accumulates in FP32.  Weight layout (one flat array):
//   W1 [32][NI], b1 [32], W2 [32][32], b2 [32], w3 [32], b3
#pragma once

#include <cuda_bf16.h>

#include <cstdint>

#include "kernels.cuh"

namespace kfvm {

template <int DIM>
struct MlpShape {
  static constexpr int R = 2;
  static constexpr int SIDE = 2 * R + 1;
  static constexpr int P = DIM == 2 ? SIDE * SIDE : SIDE * SIDE * SIDE;
  static constexpr int NI = 2 * P;
  static constexpr int NH = 32;
  static constexpr int W1 = 0, B1 = NH * NI, W2 = B1 + NH, B2 = W2 + NH * NH, W3 = B2 + NH, B3 = W3 + NH;
  static constexpr int NW = B3 + 1;
};

// density / pressure of the block's cells plus a halo of R (padded array indices)
template <int DIM>
struct MlpTile {
  static constexpr int R = MlpShape<DIM>::R;
  static constexpr int TX = kBlockX + 2 * R, TY = kBlockY + 2 * R, TZ = DIM == 3 ? 2 * R + 1 : 1;
  static constexpr int N = TX * TY * TZ;
};

// GELU in its tanh approximation (Hendrycks and Gimpel), written as
// x sigma(2 sqrt(2/pi) (x + 0.044715 x^3)): one exponential and one approximate
// division instead of erf.  Inference and training use the same function.
constexpr float kGeluC0 = 1.5957691216057308f;   // 2 sqrt(2 / pi)
constexpr float kGeluC1 = 0.07135481627260025f;    // 2 sqrt(2 / pi) 0.044715

// sigma(2 sqrt(2/pi) (x + 0.044715 x^3)); the exponent is capped so that the
// denominator stays below the range where __fdividef returns 0
__device__ __forceinline__ float gelu_sig(float x) {
  const float y = x * fmaf(kGeluC1, x * x, kGeluC0);
  return __fdividef(1.0f, 1.0f + __expf(fminf(-y, 80.0f)));
}

__device__ __forceinline__ float gelu(float x) { return x * gelu_sig(x); }

__device__ __forceinline__ float gelu_grad(float x) {
  const float s = gelu_sig(x);
  return s + x * s * (1.0f - s) * fmaf(3.0f * kGeluC1, x * x, kGeluC0);
}

template <int DIM, int EQ>
__device__ __forceinline__ void mlp_tile_fill(const double *__restrict__ U, const Grid &g, int64_t i0, int64_t j0,
                                              int64_t k, float (*t)[MlpTile<DIM>::N]) {
  using Tl = MlpTile<DIM>;
  using E = Eos<EQ>;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  for (int n = tid; n < Tl::N; n += blockDim.x * blockDim.y) {
    const int a = n % Tl::TX, b = (n / Tl::TX) % Tl::TY, cz = n / (Tl::TX * Tl::TY);
    const int64_t gi = i0 - Tl::R + a, gj = j0 - Tl::R + b, gk = k - (DIM == 3 ? Tl::R : 0) + cz;
    if (gi > g.nx + Tl::R - 1 || gj > g.ny + Tl::R - 1) continue; // beyond the padded array
    const double *Uc = U + pidx(g, gi, gj, gk);
    double u[E::NV];
#pragma unroll
    for (int v = 0; v < E::NV; v++) u[v] = Uc[v * g.pvol];
    t[0][n] = (float)u[DENS];
    t[1][n] = (float)E::pres(g.gamma, u);
  }
}

// 1 / (m + 1e-4 |q_c|), every operation rounded on its own (no contraction), so
// the value is reproducible off the GPU
__device__ __forceinline__ float mlp_scale(float m, float qc) {
  return __fdiv_rn(1.0f, __fadd_rn(__fadd_rn(m, __fmul_rn(1e-4f, fabsf(qc))), 1e-30f));
}

// a feature: (q - q_c) s
__device__ __forceinline__ float mlp_feature(float q, float qc, float s) { return __fmul_rn(__fsub_rn(q, qc), s); }

// center values and scale factors of the two patches of a cell at block position (tx, ty)
template <int DIM>
__device__ __forceinline__ void mlp_scales(const float (*t)[MlpTile<DIM>::N], int tx, int ty, float &rc,
                                           float &pc, float &sr, float &sp) {
  using Tl = MlpTile<DIM>;
  constexpr int R = Tl::R, ZR = DIM == 3 ? R : 0;
  const int c0 = (ZR * Tl::TY + ty + R) * Tl::TX + tx + R;
  rc = t[0][c0];
  pc = t[1][c0];
  float mr = 0.0f, mp = 0.0f;
  for (int dz = -ZR; dz <= ZR; dz++)
    for (int dy = -R; dy <= R; dy++)
#pragma unroll
      for (int dx = -R; dx <= R; dx++) {
        const int n = c0 + (dz * Tl::TY + dy) * Tl::TX + dx;
        mr = fmaxf(mr, fabsf(__fsub_rn(t[0][n], rc)));
        mp = fmaxf(mp, fabsf(__fsub_rn(t[1][n], pc)));
      }
  sr = mlp_scale(mr, rc);
  sp = mlp_scale(mp, pc);
}

} // namespace kfvm
