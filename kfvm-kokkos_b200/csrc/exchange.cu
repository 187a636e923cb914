// exchange.cu -- the boundary communication of a decomposed domain on the device:
// the axis-by-axis halo fill and the pack / unpack of cell slabs and boundary
// face states that the exchange callbacks carry between ranks
// (src/Solver.cpp:744-1460, src/BoundaryData.cpp of the reference).
//
// Halo (setCellBCs order): axis x over the interior y, z rows, then axis y over
// all x (the x halo included) and interior z, then axis z over all x and y.  Per
// axis, the r = 2 layers along an exchange face come from the neighbour (packed
// there from its interior layers), the other faces are filled from this block as
// the one-domain fill does (periodic wrap or wall mirror of that axis only, with
// the face's sign flips).  Every cell of the padded block then holds what the
// whole domain's padded array holds at the same place.
//
// Face states (setFaceBCs): on an exchange face the outer slot (the neighbour's
// reconstruction) is received into the face array itself, slot 0 at the low
// face and slot 1 at the high face; the kernels that read boundary faces take it
// from there.  Per face point: the NV states, then (for the KXRCF selector) the
// FP32 indicator.
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.cuh"
#include "launch.h"

namespace kfvm {

// extents of the halo slab of axis d: layers (2r: r low, r high), then the two
// other axes in increasing order (padded for axes below d, interior above)
struct Slab {
  int64_t e1, e2, lo1, lo2;  // extents and first index of the other two axes
  int a1, a2;                // which axes they are
};

__host__ __device__ inline Slab slab_of(const Grid &g, int dim, int d) {
  const int64_t n[3] = {g.nx, g.ny, dim == 3 ? g.nz : 1};
  Slab s;
  s.a1 = d == 0 ? 1 : 0;
  s.a2 = d == 2 ? 1 : 2;
  const bool pad1 = s.a1 < d, pad2 = s.a2 < d && dim == 3;
  s.lo1 = pad1 ? -kRad : 0;
  s.e1 = n[s.a1] + (pad1 ? 2 * kRad : 0);
  s.lo2 = pad2 ? -kRad : 0;
  s.e2 = (s.a2 == 2 && dim == 2) ? 1 : n[s.a2] + (pad2 ? 2 * kRad : 0);
  return s;
}

// (layer index h in [0, r), slab position t) -> padded coordinates; side 0 = low
__device__ inline void slab_cell(const Grid &g, int dim, int d, const Slab &s, int side, bool halo, int64_t h,
                                 int64_t t, int64_t &i, int64_t &j, int64_t &k) {
  const int64_t n[3] = {g.nx, g.ny, dim == 3 ? g.nz : 1};
  int64_t c[3];
  // along d: halo layers -r..-1 / n..n+r-1, interior layers 0..r-1 / n-r..n-1
  c[d] = halo ? (side == 0 ? h - kRad : n[d] + h) : (side == 0 ? h : n[d] - kRad + h);
  c[s.a1] = s.lo1 + t % s.e1;
  c[s.a2] = s.lo2 + t / s.e1;
  i = c[0];
  j = c[1];
  k = dim == 3 ? c[2] : 0;
}

template <int DIM, int NV>
__global__ void __launch_bounds__(256) bc_axis_kernel(double *__restrict__ U, Grid g, int d) {
  const Slab s = slab_of(g, DIM, d);
  const int64_t per = s.e1 * s.e2, total = 2 * kRad * per;
  const int64_t n[3] = {g.nx, g.ny, DIM == 3 ? g.nz : 1};
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t layer = t / per, q = t % per;
    const int side = layer < kRad ? 0 : 1;
    const int f = 2 * d + side;
    if (g.bc[f] == KFVM_BC_EXCHANGE || g.bc[f] == KFVM_BC_USER) continue;  // from the neighbour / the user
    int64_t i, j, k;
    slab_cell(g, DIM, d, s, side, true, side == 0 ? layer : layer - kRad, q, i, j, k);
    int64_t c[3] = {i, j, k};
    const int64_t m = c[d];
    // periodic wrap or mirror along d only; the other coordinates stay (their
    // halos were filled by the earlier axes)
    if (m < 0) c[d] = g.bc[2 * d] == KFVM_BC_PERIODIC ? m + n[d] : -m - 1;
    else c[d] = g.bc[2 * d + 1] == KFVM_BC_PERIODIC ? m - n[d] : 2 * n[d] - m - 1;
    const int64_t dst = pidx(g, i, j, k), src = pidx(g, c[0], c[1], c[2]);
    const unsigned flip = g.bflip[f];
#pragma unroll
    for (int v = 0; v < NV; v++) {
      const double x = U[v * g.pvol + src];
      U[v * g.pvol + dst] = (flip >> v) & 1u ? -x : x;
    }
  }
}

// cells of one side's slab <-> buffer [v][layer][position]
template <int DIM, bool PACK>
__global__ void __launch_bounds__(256)
    cell_slab_kernel(double *__restrict__ U, Grid g, int nv, int d, int side, double *__restrict__ buf) {
  const Slab s = slab_of(g, DIM, d);
  const int64_t per = s.e1 * s.e2, total = kRad * per;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t i, j, k;
    slab_cell(g, DIM, d, s, side, !PACK, t / per, t % per, i, j, k);
    const int64_t p = pidx(g, i, j, k);
    for (int v = 0; v < nv; v++) {
      if (PACK) buf[v * total + t] = U[v * g.pvol + p];
      else U[v * g.pvol + p] = buf[v * total + t];
    }
  }
}

// boundary face plane of axis d at the low (side 0) or high face: this block's own
// slot (1 at the low face, 0 at the high face) packed, or the outer slot unpacked;
// buffer [q][v][face of the plane] then, with W, [q][face] as floats
template <bool PACK>
__global__ void __launch_bounds__(256)
    face_plane_kernel(double *__restrict__ F, float *__restrict__ W, Grid g, int nqf, int nv, int d, int side,
                      double *__restrict__ buf) {
  const int64_t fx = g.fdim[d][0], fy = g.fdim[d][1], fz = g.fdim[d][2];
  const int64_t e1 = d == 0 ? fy : fx, e2 = d == 2 ? fy : fz;
  const int64_t per = e1 * e2, nf = g.nface[d];
  const int64_t m = side == 0 ? 0 : (d == 0 ? g.nx : (d == 1 ? g.ny : g.nz));
  const int slot = PACK ? (side == 0 ? 1 : 0) : (side == 0 ? 0 : 1);
  float *wbuf = reinterpret_cast<float *>(buf + (int64_t)nqf * nv * per);
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < per; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t a = t % e1, b = t / e1;
    const int64_t fi = d == 0 ? m : a, fj = d == 0 ? a : (d == 1 ? m : b), fk = d == 2 ? m : b;
    const int64_t fidx = (fk * fy + fj) * fx + fi;
    for (int q = 0; q < nqf; q++) {
      for (int v = 0; v < nv; v++) {
        double *x = F + ((int64_t)(slot * nqf + q) * nv + v) * nf + fidx;
        double *y = buf + ((int64_t)q * nv + v) * per + t;
        if (PACK) *y = *x;
        else *x = *y;
      }
      if (W) {
        float *x = W + (int64_t)(slot * nqf + q) * nf + fidx;
        float *y = wbuf + (int64_t)q * per + t;
        if (PACK) *y = *x;
        else *x = *y;
      }
    }
  }
}

// the FP32 KXRCF indicator of the outer slot of one boundary face plane, from the
// outer states a user boundary condition wrote there (the value the reconstruction
// stores for an inner state: Eos::weno_store, or D rounded for SR)
template <int DIM, int EQ>
__global__ void __launch_bounds__(256)
    face_indicator_kernel(const double *__restrict__ F, float *__restrict__ W, Grid g, int nqf, int d, int side) {
  constexpr int NV = Eos<EQ>::NV;
  const int64_t fx = g.fdim[d][0], fy = g.fdim[d][1], fz = g.fdim[d][2];
  const int64_t e1 = d == 0 ? fy : fx, e2 = d == 2 ? fy : fz;
  const int64_t per = e1 * e2, nf = g.nface[d];
  const int64_t m = side == 0 ? 0 : (d == 0 ? g.nx : (d == 1 ? g.ny : g.nz));
  const int slot = side == 0 ? 0 : 1;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < per * nqf;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int q = (int)(t / per);
    const int64_t p = t % per, a = p % e1, b = p / e1;
    const int64_t fi = d == 0 ? m : a, fj = d == 0 ? a : (d == 1 ? m : b), fk = d == 2 ? m : b;
    const int64_t fidx = (fk * fy + fj) * fx + fi;
    double st[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) st[v] = F[((int64_t)(slot * nqf + q) * NV + v) * nf + fidx];
    float w;
    if constexpr (EQ == EQ_SR) w = __double2float_rn(st[DENS]);
    else w = Eos<EQ>::template weno_store<DIM>(g.gamma, st[DENS], (g.gamma - 1.0) * Eos<EQ>::eint(st));
    W[(int64_t)(slot * nqf + q) * nf + fidx] = w;
  }
}

static unsigned blocks_for(int64_t n) { return (unsigned)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096); }

int64_t cell_slab_values(const Grid &g, int dim, int nv, int d) {
  const Slab s = slab_of(g, dim, d);
  return (int64_t)kRad * s.e1 * s.e2 * nv;
}

int64_t face_plane_bytes(const Grid &g, int nqf, int nv, int d, bool withW) {
  const int64_t e1 = d == 0 ? g.fdim[d][1] : g.fdim[d][0], e2 = d == 2 ? g.fdim[d][1] : g.fdim[d][2];
  const int64_t per = e1 * e2;
  return per * nqf * nv * (int64_t)sizeof(double) + (withW ? per * nqf * (int64_t)sizeof(float) : 0);
}

cudaError_t launch_bc_axis(int dim, int nv, double *U, const Grid &g, int d, cudaStream_t s) {
  const Slab sl = slab_of(g, dim, d);
  const unsigned nb = blocks_for(2 * kRad * sl.e1 * sl.e2);
  if (dim == 2 && nv == 5) bc_axis_kernel<2, 5><<<nb, 256, 0, s>>>(U, g, d);
  else if (dim == 3 && nv == 5) bc_axis_kernel<3, 5><<<nb, 256, 0, s>>>(U, g, d);
  else if (dim == 2) bc_axis_kernel<2, 9><<<nb, 256, 0, s>>>(U, g, d);
  else bc_axis_kernel<3, 9><<<nb, 256, 0, s>>>(U, g, d);
  return cudaGetLastError();
}

cudaError_t launch_cell_slab(int dim, int nv, double *U, const Grid &g, int d, int side, bool pack, double *buf,
                             cudaStream_t s) {
  const Slab sl = slab_of(g, dim, d);
  const unsigned nb = blocks_for(kRad * sl.e1 * sl.e2);
  if (dim == 2) {
    if (pack) cell_slab_kernel<2, true><<<nb, 256, 0, s>>>(U, g, nv, d, side, buf);
    else cell_slab_kernel<2, false><<<nb, 256, 0, s>>>(U, g, nv, d, side, buf);
  } else {
    if (pack) cell_slab_kernel<3, true><<<nb, 256, 0, s>>>(U, g, nv, d, side, buf);
    else cell_slab_kernel<3, false><<<nb, 256, 0, s>>>(U, g, nv, d, side, buf);
  }
  return cudaGetLastError();
}

cudaError_t launch_face_plane(double *F, float *W, const Grid &g, int nqf, int nv, int d, int side, bool pack,
                              double *buf, cudaStream_t s) {
  const int64_t e1 = d == 0 ? g.fdim[d][1] : g.fdim[d][0], e2 = d == 2 ? g.fdim[d][1] : g.fdim[d][2];
  const unsigned nb = blocks_for(e1 * e2);
  if (pack) face_plane_kernel<true><<<nb, 256, 0, s>>>(F, W, g, nqf, nv, d, side, buf);
  else face_plane_kernel<false><<<nb, 256, 0, s>>>(F, W, g, nqf, nv, d, side, buf);
  return cudaGetLastError();
}

cudaError_t launch_face_indicator(int dim, int eq, const double *F, float *W, const Grid &g, int nqf, int d,
                                  int side, cudaStream_t s) {
  const int64_t e1 = d == 0 ? g.fdim[d][1] : g.fdim[d][0], e2 = d == 2 ? g.fdim[d][1] : g.fdim[d][2];
  const unsigned nb = blocks_for(e1 * e2 * nqf);
#define KFVM_FI(D, E) face_indicator_kernel<D, E><<<nb, 256, 0, s>>>(F, W, g, nqf, d, side)
  if (dim == 2) {
    if (eq == EQ_GLM) KFVM_FI(2, EQ_GLM);
    else if (eq == EQ_SR) KFVM_FI(2, EQ_SR);
    else if (eq == EQ_NS) KFVM_FI(2, EQ_NS);
    else KFVM_FI(2, EQ_HYDRO);
  } else {
    if (eq == EQ_GLM) KFVM_FI(3, EQ_GLM);
    else if (eq == EQ_SR) KFVM_FI(3, EQ_SR);
    else if (eq == EQ_NS) KFVM_FI(3, EQ_NS);
    else KFVM_FI(3, EQ_HYDRO);
  }
#undef KFVM_FI
  return cudaGetLastError();
}

} // namespace kfvm
