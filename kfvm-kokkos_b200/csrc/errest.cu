// errest.cu -- the embedded RK error estimate and positivity check over a state
// pair (RKFSAL_ErrEst_K, src/numeric/Numeric_K.H:262-290 of slug-cfd/kfvm-kokkos):
//   err    = sum over cells and variables of ((u - uhat) / (atol + rtol max(|u|,|uhat|)))^2
//   posmin = min over cells of EOS::positivity(u), or -1 where u holds a NaN
// Deterministic two-level reduction: one partial per block of kErrBlock cells,
// then a fixed-order sum in one block.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/kfvm_b200.h"
#include "kernels.cuh"
#include "launch.h"

namespace kfvm {

constexpr int kErrBlock = 256;

template <int EQ>
__global__ void __launch_bounds__(kErrBlock)
    errest_kernel(const double *__restrict__ u, const double *__restrict__ uhat, int64_t n,
                  double atol, double rtol, double *__restrict__ part) {
  using E = Eos<EQ>;
  constexpr int NV = E::NV;
  const int64_t c = blockIdx.x * (int64_t)kErrBlock + threadIdx.x;
  double err = 0.0, pos = 1.0;
  if (c < n) {
    bool hasNan = false;
    double st[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) {
      const double a = u[v * n + c], b = uhat[v * n + c];
      st[v] = a;
      hasNan = hasNan || isnan(a);
      const double e = (a - b) / (atol + rtol * fmax(fabs(a), fabs(b)));
      err += e * e;
    }
    pos = hasNan ? -1.0 : E::positivity(st);
  }
  __shared__ double se[kErrBlock / 32], sp[kErrBlock / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    err += __shfl_xor_sync(0xffffffffu, err, o);
    pos = fmin(pos, __shfl_xor_sync(0xffffffffu, pos, o));
  }
  if ((threadIdx.x & 31) == 0) {
    se[threadIdx.x >> 5] = err;
    sp[threadIdx.x >> 5] = pos;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 1.0;
    for (int w = 0; w < kErrBlock / 32; w++) {
      a += se[w];
      b = b > sp[w] ? sp[w] : b;
    }
    part[2 * blockIdx.x] = a;
    part[2 * blockIdx.x + 1] = b;
  }
}

// fixed-order combination of the block partials into out[0] (sum) and out[1] (min)
__global__ void __launch_bounds__(1024) errest_finalize(const double *__restrict__ part, int64_t nblk,
                                                        double *__restrict__ out) {
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
    out[0] = se[0];
    out[1] = sp[0];
  }
}

int64_t errest_blocks(int64_t n) { return (n + kErrBlock - 1) / kErrBlock; }

cudaError_t launch_errest(int eq, const double *u, const double *uhat, int64_t n, double atol,
                          double rtol, double *part, double *out, cudaStream_t s) {
  const int64_t nblk = errest_blocks(n);
  if (nblk <= 0) return cudaErrorInvalidValue;
  if (eq == EQ_GLM) errest_kernel<EQ_GLM><<<(unsigned)nblk, kErrBlock, 0, s>>>(u, uhat, n, atol, rtol, part);
  else if (eq == EQ_SR) errest_kernel<EQ_SR><<<(unsigned)nblk, kErrBlock, 0, s>>>(u, uhat, n, atol, rtol, part);
  else errest_kernel<EQ_HYDRO><<<(unsigned)nblk, kErrBlock, 0, s>>>(u, uhat, n, atol, rtol, part);
  errest_finalize<<<1, 1024, 0, s>>>(part, nblk, out);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Scratch of kfvm_err_est_noalloc: one (sum, min) pair per block of kErrBlock
// cells, for up to KFVM_NOALLOC_MAX_CELLS cells (1 MiB).  It is a file-scope
// device array, so every GPU that loads the library holds it until exit, and all
// calls share it.  Every block overwrites its own pair before the finalize kernel
// reads it, so nothing has to be cleared between calls.
static __device__ __align__(256) double g_noalloc_part[2 * (KFVM_NOALLOC_MAX_CELLS / kErrBlock)];

namespace {
// Device address of g_noalloc_part on the current device.  In host code the
// symbol names a host-side stand-in, so the address comes from
// cudaGetSymbolAddress with the device current.  It is looked up on every call
// (a host-side query, no device work): after a cudaDeviceReset the module is
// loaded again and the array may move, so a cached address could go stale.
cudaError_t noalloc_scratch(double **ptr) {
  void *p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_part);
  if (e != cudaSuccess) return e;
  *ptr = static_cast<double *>(p);
  return cudaSuccess;
}
} // namespace

} // namespace kfvm

extern "C" int kfvm_err_est_noalloc(int32_t eq, const double *u_dev, const double *uhat_dev,
                                    int64_t n, double atol, double rtol, double *out_dev,
                                    void *stream) {
  if (!u_dev || !uhat_dev || !out_dev)
    return kfvm::set_last_error(KFVM_ERR_ARG, "kfvm_err_est_noalloc: null pointer");
  if (eq < KFVM_EQ_HYDRO || eq > KFVM_EQ_SRHYDRO)
    return kfvm::set_last_error(KFVM_ERR_ARG, "kfvm_err_est_noalloc: unknown equation type");
  if (n <= 0 || n > KFVM_NOALLOC_MAX_CELLS)
    return kfvm::set_last_error(KFVM_ERR_ARG,
                                "kfvm_err_est_noalloc: n must be in [1, " +
                                    std::to_string((long long)KFVM_NOALLOC_MAX_CELLS) +
                                    "], the capacity of its fixed scratch array");
  double *part = nullptr;
  cudaError_t e = kfvm::noalloc_scratch(&part);
  if (e != cudaSuccess)
    return kfvm::set_last_error(KFVM_ERR_CUDA, std::string("kfvm_err_est_noalloc: cudaGetSymbolAddress: ") +
                                                   cudaGetErrorString(e));
  e = kfvm::launch_errest(eq, u_dev, uhat_dev, n, atol, rtol, part, out_dev,
                          static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess)
    return kfvm::set_last_error(KFVM_ERR_CUDA, std::string("kfvm_err_est_noalloc: ") + cudaGetErrorString(e));
  return KFVM_OK;
}
