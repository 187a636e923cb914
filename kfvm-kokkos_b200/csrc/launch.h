// launch.h -- host-side entry points of the kernels in kernels.cu
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "kernels.cuh"

namespace kfvm {

struct StageArgs {
  const double *U;     // stage state (padded, halo filled)
  double *Unext;       // next stage state (padded), STAGE_UPDATE only
  const double *Uprev; // state at the start of the step (padded)
  double *Uhat, *Utmp, *K;
  double *const *G;    // per-direction face fluxes
  double *const *F;    // per-direction face states (GLM sources)
  const double *src;   // interior point values (GLM)
  const double *theta;
  int mode;            // enum StageMode
  StageCoef co;
  double Re, Pr, atol, rtol;
  double *part;        // block partials of the error estimate
  DevScalars *sc;
};

int64_t stage_blocks(const Grid &g);
cudaError_t launch_bc(int dim, int eq, double *U, const Grid &g, cudaStream_t s);
// decomposed domains (exchange.cu): the halo fill of one axis (its non-exchange
// faces), and the pack (pack = true) / unpack of one side's r cell layers of an
// axis ([v][layer][position], cell_slab_values values) and of one boundary face
// plane (this block's slot packed, the outer slot unpacked; face_plane_bytes,
// the FP32 indicator after the states when W is given)
cudaError_t launch_bc_axis(int dim, int nv, double *U, const Grid &g, int d, cudaStream_t s);
int64_t cell_slab_values(const Grid &g, int dim, int nv, int d);
int64_t face_plane_bytes(const Grid &g, int nqf, int nv, int d, bool withW);
cudaError_t launch_cell_slab(int dim, int nv, double *U, const Grid &g, int d, int side, bool pack, double *buf,
                             cudaStream_t s);
cudaError_t launch_face_plane(double *F, float *W, const Grid &g, int nqf, int nv, int d, int side, bool pack,
                              double *buf, cudaStream_t s);
// the FP32 KXRCF indicator of one face plane's outer slot from its states (user faces)
cudaError_t launch_face_indicator(int dim, int eq, const double *F, float *W, const Grid &g, int nqf, int d,
                                  int side, cudaStream_t s);
// interior state between the host order (variable, k, j, i) in a flat device
// buffer and the padded layout; one launch for all variables
cudaError_t launch_interior(double *Up, double *flat, const Grid &g, int nv, bool toPadded, cudaStream_t s);
cudaError_t launch_fill(double *p, int64_t n, double val, cudaStream_t s);
// rcp_nr accuracy probe: out[0] = max ulp distance to 1/y, out[1] = bits of the
// largest relative difference of x * rcp_nr(y) from x / y
cudaError_t launch_rcp_probe(int64_t n, uint64_t seed, unsigned long long *out, cudaStream_t s);
// FP64 tensor-pipe probe: blocks x 4 warps, each iters x 8 m8n8k4 MMAs
cudaError_t launch_dmma_peak(int blocks, int iters, double *out, cudaStream_t s);
// limiter bounds of every cell, [minDens | maxDens | minEint][cell] (the pre-pass
// of the reconstruction kernels, which read them)
cudaError_t launch_bounds(int dim, int eq, const double *U, const Grid &g, double *bnd, cudaStream_t s);
// stage front end: linear states + KXRCF indicator + limiter bound status,
// KXRCF flags, WENO decision / heavy-list compaction, heavy cells
// bnd: the limiter bounds of every cell from launch_bounds
// (the FP64 form computes the limiter bounds itself and writes them to bnd).  umap
// (recon_dmma_state_map of U; five variables, or GLM-MHD in 2D) stages the halo tiles by TMA;
// null reads the state with plain global loads; a block whose wait gave up sets
// sc->fault
cudaError_t launch_recon(int dim, int eq, const double *U, const CUtensorMap *umap, const Grid &g,
                         const DevStencil *S, int wantInd, double *const *F, float *const *W, double *src,
                         uint8_t *status, double2 *lamvel, double *bnd, DevScalars *sc, cudaStream_t s);
int recon_dmma_state_map(CUtensorMap *map, const double *U, const Grid &g, int dim, int nv);
// the same outputs with the stencil sum on the tcgen05 tensor cores (3xTF32);
// umap (recon_tc_state_map of U) stages the halo tiles by TMA, null loads them
// with plain global loads; a block whose wait gave up sets sc->fault
cudaError_t launch_recon_tc(int dim, int eq, const double *U, const CUtensorMap *umap, const Grid &g,
                            const DevStencil *S, int wantInd, double *const *F, float *const *W, double *src,
                            uint8_t *status, double2 *lamvel, double *bnd, DevScalars *sc, cudaStream_t s);
int recon_tc_state_map(CUtensorMap *map, const double *U, const Grid &g, int dim, int nv);
// self-test of the bounded mbarrier wait: out[0] = gave up, out[1] = ns waited
cudaError_t launch_wait_probe(uint64_t limit_ns, unsigned long long *out, cudaStream_t s);
// host: split the [cell][row] linear weights of S into the TF32 B-operand tables
void fill_tc_weights(DevStencil &S, int dim, int nrows);
// host: the same weights as FP64 MMA B fragments
void fill_dmma_weights(DevStencil &S, int nrows);
cudaError_t launch_flag(int dim, int eq, const double *U, const Grid &g, float *const *W, double *const *F,
                        const double *theta, uint8_t *flag, DevScalars *sc, double thr,
                        cudaStream_t s);
cudaError_t launch_compact(int dim, int eq, const Grid &g, int mode, const uint8_t *flag, uint8_t *wset,
                           const uint8_t *status, uint8_t *applied, double *theta, uint32_t *heavy,
                           const double2 *lamvel, DevScalars *sc, const JudgeArgs &jd, cudaStream_t s);
// bnd: the reconstruction's limiter bounds, or null (full-WENO evaluations, where
// no reconstruction pass ran) to compute them from the state
cudaError_t launch_heavy(int dim, int eq, const double *U, const Grid &g, const DevStencil *S,
                         double *theta, double *const *F, double *src, const uint32_t *heavy,
                         const double *bnd, DevScalars *sc, const JudgeArgs &jd, int heavy_blocks,
                         cudaStream_t s);
// same: the equal-state variant of the Riemann kernels
cudaError_t launch_riemann(int dim, int eq, double *const *F, double *const *G, const Grid &g,
                           DevScalars *sc, bool same, cudaStream_t s);
cudaError_t launch_stage(int dim, int eq, const StageArgs &a, const Grid &g, cudaStream_t s);

// learned troubled-cell indicator (mlp.cu)
int mlp_num_weights(int dim);
int mlp_num_inputs(int dim);
// sample collection in cell order: labels and keep decisions of every cell into
// flags, the (density, pressure) pairs into tb, and the kept cells' indices
// compacted into sel (*nsel of them; temp: mlp_select_temp_bytes(g.n) bytes of
// device scratch); then the features of the first `count` of them
size_t mlp_select_temp_bytes(int64_t n);
struct MlpTileBuf;
cudaError_t launch_mlp_select(int dim, int eq, const double *U, const Grid &g, const DevStencil *S, double tau,
                              double keep, uint64_t seed, const MlpTileBuf &tb, uint8_t *flags, int64_t *sel,
                              int64_t *nsel, void *temp, size_t temp_bytes, cudaStream_t s);
cudaError_t launch_mlp_features(int dim, const Grid &g, const MlpTileBuf &tb, const int64_t *sel, int64_t count,
                                const uint8_t *flags, uint16_t *feats, uint8_t *labels, int64_t *cells,
                                cudaStream_t s);
// inference: the (density, pressure) pairs of every padded cell (one kernel), then
// per block a TMA load of its halo tile of pairs plus bulk loads of the weight image,
// and the network with both matrix layers on tcgen05 (layer 1 BF16, layer 2 split
// TF32; FP32 accumulation), bias, GELU and output in FP32 (a second kernel)
struct MlpTileBuf {
  CUtensorMap map;         // halo tiles of rp (TMA box TX x TY x TZ of 8-byte pairs)
  float2 *rp = nullptr;    // [plane][row][x] pairs, row pitch rpx
  int64_t rpx = 0;
};
cudaError_t mlp_tile_buf_init(int dim, const Grid &g, MlpTileBuf &tb);
// img: the weight image of launch_mlp_pack
cudaError_t launch_mlp_flag(int dim, int eq, const double *U, const Grid &g, const MlpTileBuf &tb, const uint8_t *img,
                            const double *theta, uint8_t *flag, uint8_t *pred, DevScalars *sc, float logit_thr,
                            cudaStream_t s);
cudaError_t launch_mlp_prob(int dim, int eq, const double *U, const Grid &g, const MlpTileBuf &tb, const uint8_t *img,
                            float *out, DevScalars *sc, cudaStream_t s);
// the inference kernel's weight image (W1^T BF16, W2^T FP32, biases) from the BF16
// weights wb and their FP32 values wq, after every change of the weights
int mlp_image_bytes(int dim);
cudaError_t launch_mlp_pack(int dim, const uint16_t *wb, const float *wq, uint8_t *img, cudaStream_t s);
// one training step: per-block gradient rows in gpart (mlp_train_blocks(batch) x
// weights) and losses in lpart, summed in block order by the Adam update
int mlp_train_blocks(int batch);
cudaError_t launch_mlp_train_step(int dim, const uint16_t *feats, const uint8_t *labels, int64_t n, int batch,
                                  float *master, float *m, float *v, float *gpart, float *lpart, float *wq,
                                  uint16_t *wb, float *loss, float pos_weight, float lr, int t, uint64_t seed,
                                  cudaStream_t s);
cudaError_t launch_stage_pre(int dim, int eq, double *U1, const double *Uprev, double *Uhat,
                             double *Utmp, const double *K, const Grid &g, double betaDt,
                             double bhatDt, int use_tmp, cudaStream_t s);
cudaError_t launch_copy(int dim, int eq, double *dst, const double *src, const Grid &g,
                        cudaStream_t s);
cudaError_t launch_ic(int dim, int eq, int ic_kind, uint64_t seed, const kfvm_config &cfg,
                      double *U, const Grid &g, cudaStream_t s);

// error estimate of a state pair: block partials into part (2 per block of 256
// cells), fixed-order sum into out[0] (err) and out[1] (positivity minimum)
int64_t errest_blocks(int64_t n);

// flow statistics (stats.cu): 3 partials per block, the sums into out[0..2]
int64_t stats_blocks(const Grid &g);
int stats_count(int eq);
cudaError_t launch_stats(int dim, int eq, const double *U, const Grid &g, double ifac, double *part, double *out,
                         cudaStream_t s);

// random forcing (forcing.cu): mode table on the host, integrals and kick on the device
int forcing_num_modes(int dim);
void forcing_draw(int dim, uint32_t seed32, double *modes);
int64_t forcing_blocks(const Grid &g);
cudaError_t launch_forcing_integrate(int dim, const double *U, const Grid &g, const double *modes, int nm,
                                     double ratio, const double lo[3], double *part, double *sums,
                                     cudaStream_t s);
cudaError_t launch_forcing_apply(int dim, double *U, const Grid &g, const double *modes, int nm, double ratio,
                                 double str, const double lo[3], cudaStream_t s);
cudaError_t launch_errest(int eq, const double *u, const double *uhat, int64_t n, double atol,
                          double rtol, double *part, double *out, cudaStream_t s);

int build_stencil(const kfvm_config *cfg, kfvm_stencil *st);

// records msg as the calling thread's kfvm_last_error() and returns code
int set_last_error(int code, const std::string &msg);

} // namespace kfvm
