// capi.cu -- the C ABI (include/kfvm_b200.h): solver context, device memory,
// the per-stage launch sequence (Solver::evalRHS) and the adaptive FSAL time
// stepper (Solver::TakeStep) of slug-cfd/kfvm-kokkos, src/Solver.cpp:36-530.
//
// Host control flow stays on the host, as in the reference: one stream per
// solver, one device->host read per step attempt (max speed, error sum,
// positivity minimum) instead of the reference's per-stage reads.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/kfvm_b200.h"
#include "kernels.cuh"
#include "geometry.h"
#include "launch.h"

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

#define CK(call)                                                                         \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return fail(KFVM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));    \
  } while (0)

// RK coefficient tables (src/numeric/Numeric.H:111-282)
struct RKTable {
  int nStages;
  double gam1[10], gam2[10], gam3[10], delta[10], beta[10], bhat[10], c[10];
  double bhatfsal, ep1, ep2;
  bool use_tmp;
};

bool rk_table(int rk, RKTable &r) {
  std::memset(&r, 0, sizeof(r));
  if (rk == KFVM_RK_SSP4_3_2) {
    // SSP(4,3) of Kraaijevanger with the embedded pair and PI values of Conde et al.
    r.nStages = 4;
    const double g1[] = {0.0, 1.0, 1.0 / 3.0, 1.0}, g3[] = {0.0, 0.0, 2.0 / 3.0, 0.0};
    const double be[] = {1.0 / 2.0, 1.0 / 2.0, 1.0 / 6.0, 1.0 / 2.0};
    const double cc[] = {0.0, 1.0 / 2.0, 1.0, 1.0 / 2.0};
    for (int i = 0; i < 4; i++) {
      r.gam1[i] = g1[i];
      r.gam3[i] = g3[i];
      r.beta[i] = be[i];
      r.bhat[i] = 1.0 / 4.0;
      r.c[i] = cc[i];
    }
    r.bhatfsal = 0.0;
    r.ep1 = 0.8 / 3.0;
    r.ep2 = -0.31 / 3.0;
  } else if (rk == KFVM_RK_THREESTARP) {
    // third-order adaptive method of Ranocha et al.
    r.nStages = 5;
    const double g1[] = {0.0, 2.587771979725733308135192812685323706e-01,
                         -1.324380360140723382965420909764953437e-01,
                         5.056033948190826045833606441415585735e-02,
                         5.670532000739313812633197158607642990e-01};
    const double g2[] = {0.0, 5.528354909301389892439698870483746541e-01,
                         6.731871608203061824849561782794643600e-01,
                         2.803103963297672407841316576323901761e-01,
                         5.521525447020610386070346724931300367e-01};
    const double g3[] = {0.0, 0.0, 0.0, 2.752563273304676380891217287572780582e-01,
                         -8.950526174674033822276061734289327568e-01};
    const double de[] = {1.0, 3.407655879334525365094815965895763636e-01,
                         3.414382655003386206551709871126405331e-01,
                         7.229275366787987419692007421895451953e-01, 0.0};
    const double be[] = {2.300298624518076223899418286314123354e-01,
                         3.021434166948288809034402119555380003e-01,
                         8.025606185416310937583009085873554681e-01,
                         4.362158943603440930655148245148766471e-01,
                         1.129272530455059129782111662594436580e-01};
    const double bh[] = {9.484166705035703392326247283838082847e-02,
                         1.726371339430353766966762629176676070e-01,
                         3.998243189084371024483169698618455770e-01,
                         1.718016807580178450618829007973835152e-01,
                         5.881914422155740300718268359027168467e-02};
    const double cc[] = {0.0, 2.300298624518076223899418286314123354e-01,
                         4.050046072094990912268498160116125481e-01,
                         8.947822893693433545220710894560512805e-01,
                         7.235136928826589010272834603680114769e-01};
    for (int i = 0; i < 5; i++) {
      r.gam1[i] = g1[i];
      r.gam2[i] = g2[i];
      r.gam3[i] = g3[i];
      r.delta[i] = de[i];
      r.beta[i] = be[i];
      r.bhat[i] = bh[i];
      r.c[i] = cc[i];
    }
    r.bhatfsal = 1.020760551185952388626787099944507877e-01;
    r.ep1 = 0.7 / 3.0;
    r.ep2 = -0.23 / 3.0;
  } else if (rk == KFVM_RK_SSP10_4_3) {
    // SSP(10,4) of Ketcheson with the embedded pair and PI values of Conde et al.
    r.nStages = 10;
    const double g1[] = {0.0, 1.0, 1.0, 1.0, 2.0 / 5.0, 1.0, 1.0, 1.0, 1.0, 3.0 / 5.0};
    const double g2[] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0};
    const double g3[] = {0.0, 0.0, 0.0, 0.0, 3.0 / 5.0, 0.0, 0.0, 0.0, 0.0, -3.0 / 2.0};
    const double de[] = {0.0, 0.0, 0.0, 0.0, 0.0, 9.0 / 10.0, 0.0, 0.0, 0.0, 0.0};
    const double be[] = {1.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0, 1.0 / 15.0,
                         1.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0, 1.0 / 10.0};
    const double bh[] = {0.0, 2.0 / 9.0, 0.0, 0.0, 5.0 / 18.0, 1.0 / 3.0, 0.0, 0.0, 0.0, 1.0 / 6.0};
    const double cc[] = {0.0, 1.0 / 6.0, 1.0 / 3.0, 1.0 / 2.0, 2.0 / 3.0, 1.0 / 3.0, 1.0 / 2.0, 2.0 / 3.0,
                         5.0 / 6.0, 1.0};
    for (int i = 0; i < 10; i++) {
      r.gam1[i] = g1[i];
      r.gam2[i] = g2[i];
      r.gam3[i] = g3[i];
      r.delta[i] = de[i];
      r.beta[i] = be[i];
      r.bhat[i] = bh[i];
      r.c[i] = cc[i];
    }
    r.bhatfsal = 0.0;
    r.ep1 = 0.8 / 3.0;
    r.ep2 = -0.31 / 3.0;
  } else if (rk == KFVM_RK_FOURSTARP) {
    // fourth-order adaptive method of Ranocha et al.
    r.nStages = 9;
    const double g1[] = {0.0,
                         -4.655641447335068552684422206224169103e+00,
                         -7.720265099645871829248487209517314217e-01,
                         -4.024436690519806086742256154738379161e+00,
                         -2.129676284018530966221583708648634733e-02,
                         -2.435022509790109546199372365866450709e+00,
                         1.985627297131987000579523283542615256e-02,
                         -2.810791146791038566946663374735713961e-01,
                         1.689434168754859644351230590422137972e-01};
    const double g2[] = {0.0,
                         2.499262792574495009336242992898153462e+00,
                         5.866820377718875577451517985847920081e-01,
                         1.205146086523094569925592464380295241e+00,
                         3.474793722186732780030762737753849272e-01,
                         1.321346060965113109321230804210670518e+00,
                         3.119636464694193615946633676950358444e-01,
                         4.351419539684379261368971206040518552e-01,
                         2.359698130028753572503744518147537768e-01};
    const double g3[] = {0.0,
                         0.0,
                         0.0,
                         7.621006678721315291614677352949377871e-01,
                         -1.981182504339400567765766904309673119e-01,
                         -6.228959218699007450469629366684127462e-01,
                         -3.752248380775956442989480369774937099e-01,
                         -3.355438309135169811915662336248989661e-01,
                         -4.560955005031121479972862973705108039e-02};
    const double de[] = {1.0,
                         1.262923876648114432874834923838556100e+00,
                         7.574967189685911558308119415539596711e-01,
                         5.163589453140728104667573195005629833e-01,
                         -2.746327421802609557034437892013640319e-02,
                         -4.382673178127944142238606608356542890e-01,
                         1.273587294602656522645691372699677063e+00,
                         -6.294740283927400326554066998751383342e-01,
                         0.0};
    const double be[] = {2.836343005184365275160654678626695428e-01,
                         9.736500104654741223716056170419660217e-01,
                         3.382359225242515288768487569778320563e-01,
                         -3.584943611106183357043212309791897386e-01,
                         -4.113944068471528211627210454497620358e-03,
                         1.427968894048586363415504654313371031e+00,
                         1.808470948394314017665968411915568633e-02,
                         1.605770645946802213926893453819236685e-01,
                         2.952227015964591648775833803635147962e-01};
    const double bh[] = {2.483675912451591196775756814283216443e-02,
                         1.866327774562103796990092260942180726e-01,
                         5.671080795936984495604436622517631183e-02,
                         -3.447695439149287702616943808570747099e-03,
                         3.602245056516636472203469198006404016e-03,
                         4.545570622145088936800484247980581766e-01,
                         -2.434665289427612407531544765622888855e-04,
                         6.642755361103549971517945063138312147e-02,
                         1.613697079523505006226025497715177578e-01};
    const double cc[] = {0.0,
                         2.836343005184365275160654678626695428e-01,
                         5.484076570002894365286665352032296535e-01,
                         3.687228761669438493478872632332010073e-01,
                         -6.806126440140844191258463830024463902e-01,
                         3.518526124230705801739919476290327750e-01,
                         1.665941994879593315477304663913129942e+00,
                         9.715279295934715835299192116436237065e-01,
                         9.051569840159589594903399929316959062e-01};
    for (int i = 0; i < 9; i++) {
      r.gam1[i] = g1[i];
      r.gam2[i] = g2[i];
      r.gam3[i] = g3[i];
      r.delta[i] = de[i];
      r.beta[i] = be[i];
      r.bhat[i] = bh[i];
      r.c[i] = cc[i];
    }
    r.bhatfsal = 4.955424859358438183052504342394102722e-02;
    r.ep1 = 0.38 / 4.0;
    r.ep2 = -0.18 / 4.0;
  } else {
    return false;
  }
  for (int i = 0; i < r.nStages; i++) r.use_tmp = r.use_tmp || r.delta[i] != 0.0 || r.gam2[i] != 0.0;
  return true;
}

} // namespace

struct kfvm_solver {
  kfvm_config cfg;
  kfvm::Grid g;
  int dim, eq, nv;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  kfvm::DevStencil *dS = nullptr;
  double *Ub[3] = {nullptr, nullptr, nullptr};
  int iPrev = 0; // buffer holding Uprev; the other two alternate within a step
  int iCur = 0;  // buffer holding the current state U
  double *Uhat = nullptr, *Utmp = nullptr, *K = nullptr;
  double *F[3] = {nullptr, nullptr, nullptr}, *G[3] = {nullptr, nullptr, nullptr};
  double *src = nullptr, *theta = nullptr, *part = nullptr;
  double *bnd = nullptr; // limiter bounds per cell from the reconstruction pass, 3 x n
  double *io = nullptr; // host-order interior state for set/get (allocated at first use)
  uint8_t *flag = nullptr, *wset = nullptr, *applied = nullptr;
  uint32_t *heavy = nullptr; // compacted WENO / limiter cell list (one slot per cell)
  float *W[3] = {nullptr, nullptr, nullptr};  // KXRCF indicator (FP32 approximation) per own face slot and point
  uint8_t *status = nullptr;                  // 1: all linear states inside the limiter bounds
  double2 *lamvel = nullptr;                  // GLM speed maxima of each cell's linear states
  int heavyBlocks = 0;
  kfvm::DevScalars *sc = nullptr;
  kfvm::DevScalars *hsc = nullptr; // pinned host copy
  RKTable rk;
  double time = 0.0, dt = 0.0, errEst = 1.0;
  bool lastTimeStep = false, useSparseWeno = true, primed = false;
  // equal-state Riemann variant: on while at least a quarter
  // of its sampled faces qualify; when off, probed again after kSameProbeSteps steps
  bool sameOn = true;
  int sameProbe = 0;
  unsigned long long sameSeen = 0, sampSeen = 0;
  // random forcing (kfvm_set_forcing): parameters, draws so far, device mode table
  // and integrals
  bool forcing = false;
  kfvm_forcing fpar{};
  uint64_t fdraws = 0;
  double *fmodes = nullptr, *fsums = nullptr;
  // flow statistics: block partials and the three sums
  double *spart = nullptr, *ssum = nullptr;
  double plotFreq = 0.0; // plot times for the step-size limit (kfvm_set_plot_freq)
  int32_t plotNum = 0;
  bool writePlot = false;
  int indicator = KFVM_IND_KXRCF;
  int precision = KFVM_PREC_FP64;
  // domain decomposition: this block has exchange faces; the transport callbacks
  // (kfvm_set_exchange) and their device buffers send_lo, recv_lo, send_hi, recv_hi
  bool decomposed = false;
  // user boundary conditions (kfvm_set_user_bc): some face is KFVM_BC_USER, the
  // callback, and the time of the RHS evaluation in progress
  bool hasUser = false;
  kfvm_user_bc_fn ufn = nullptr;
  void *uuser = nullptr;
  double tEval = 0.0;
  kfvm_exchange_fn xfn = nullptr;
  kfvm_allreduce_fn rfn = nullptr;
  void *xuser = nullptr;
  double *xbuf[4] = {nullptr, nullptr, nullptr, nullptr};
  // TMA maps of the three state buffers for the tensor-core reconstruction's halo
  // tiles (built when the FP32 form is selected; unused where the pitch is odd)
  CUtensorMap umap[3];
  bool umapOk = false;
  // and those of the FP64 reconstruction's halo tiles (five variables or 2D, even pitch)
  CUtensorMap dmap[3];
  bool dmapOk = false;
  int64_t nRhs = 0, nWenoLast = 0;
  int nTS = 1;
  double dmin = 0.0;
  float lastMs = 0.0f;
  // measurement: kernel launches, optional per-class event timing
  int64_t launches = 0;
  bool timing = false;
  struct Mark {
    int cls;
    cudaEvent_t a, b;
  };
  std::vector<Mark> marks;    // recorded since the last harvest
  std::vector<cudaEvent_t> evPool;
  double clsMs[KFVM_NUM_KCLASS] = {0};
  int64_t clsLaunches[KFVM_NUM_KCLASS] = {0};
  // learned troubled-cell indicator (buffers allocated by the kfvm_mlp_* calls)
  struct Mlp {
    bool ready = false;                 // weights set or initialised
    int nw = 0, ni = 0;
    uint16_t *wb = nullptr;             // BF16 weights used by inference
    uint8_t *img = nullptr;             // the inference kernel's weight image (tcgen05 B operands, biases)
    float *wq = nullptr;                // the same values as FP32 (training forward)
    float *master = nullptr, *m = nullptr, *v = nullptr, *loss = nullptr;
    int t = 0;                          // Adam steps taken
    uint8_t *pred = nullptr;            // per-cell prediction of the last evaluation
    kfvm::MlpTileBuf tiles;             // (density, pressure) pairs and their TMA tile map
    uint16_t *feats = nullptr;          // collected samples: features, labels, cells
    uint8_t *labels = nullptr;
    int64_t *cells = nullptr;
    unsigned long long *count = nullptr;
    int64_t cap = 0, nPos = 0, have = 0;
    uint8_t *flags = nullptr;           // collection scratch: per-cell keep / label flags,
    int64_t *sel = nullptr, *nsel = nullptr;  // the kept cells in cell order and their count
    void *selTemp = nullptr;            // device scratch of the stable select
    size_t selBytes = 0;
    float *gpart = nullptr, *lpart = nullptr;  // training: per-block gradient rows and losses
    int gpartBlocks = 0;
    double logitThr = 0.0, judgeFrac = 1.0 / 256.0, tau = 0.3, missLimit = 0.25;
    int fallbackSteps = 0;
    int64_t fallbackEvents = 0;
    unsigned long long lastPos = 0, lastMissed = 0;
  } mlp;
};

namespace {

const char *const kFaultMsg =
    "tensor-core reconstruction: a block gave up waiting for its MMA completion (bounded wait)";

// the -1 entries of the wall coefficient tables as a bit mask over the variables
// (src/physics/hydro/Hydro_BCCoeffs.H, navierstokes/NavierStokes_BCCoeffs.H,
// mhd_glm/MHD_GLM_BCCoeffs.H): reflecting negates the normal momentum (and the
// normal magnetic field), no-slip every momentum component (and the normal field)
unsigned wall_flip(int bc, int d, bool glm) {
  using namespace kfvm;
  const unsigned bn = glm ? 1u << (MAGX + d) : 0u;
  if (bc == KFVM_BC_REFLECTING) return (1u << (MOMX + d)) | bn;
  if (bc == KFVM_BC_NOSLIP) return (1u << MOMX) | (1u << MOMY) | (1u << MOMZ) | bn;
  return 0u;
}

int set_err_cuda(cudaError_t e, const char *what) {
  return fail(KFVM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

cudaEvent_t pool_event(kfvm_solver *s) {
  if (!s->evPool.empty()) {
    cudaEvent_t e = s->evPool.back();
    s->evPool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// run one launcher; count its kernels and, when timing, bracket it with events
template <class Fn>
cudaError_t run(kfvm_solver *s, int cls, int nKernels, Fn &&fn) {
  kfvm_solver::Mark m{cls, nullptr, nullptr};
  if (s->timing) {
    m.a = pool_event(s);
    m.b = pool_event(s);
    cudaEventRecord(m.a, s->stream);
  }
  cudaError_t e = fn();
  s->launches += nKernels;
  s->clsLaunches[cls] += nKernels;
  if (s->timing) {
    cudaEventRecord(m.b, s->stream);
    s->marks.push_back(m);
  }
  return e;
}

// accumulate the recorded kernel-class times (after the stream was synchronised)
void harvest(kfvm_solver *s) {
  for (auto &m : s->marks) {
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, m.a, m.b) == cudaSuccess) s->clsMs[m.cls] += ms;
    s->evPool.push_back(m.a);
    s->evPool.push_back(m.b);
  }
  s->marks.clear();
}

// Keeps the equal-state Riemann variant while at least a quarter of the faces it
// samples qualify (where few do, its heavier general path costs a few per cent);
// otherwise uses the plain variant and probes again after kSameProbeSteps steps.
constexpr int kSameProbeSteps = 4;
int reduce_all(kfvm_solver *s, int op, double *vals, int n);

int update_same_mode(kfvm_solver *s) {
  unsigned long long dS = s->hsc->nsame - s->sameSeen, dN = s->hsc->nsamp - s->sampSeen;
  s->sameSeen = s->hsc->nsame;
  s->sampSeen = s->hsc->nsamp;
  if (s->decomposed) {
    // every rank takes the same choice, from the counts of all ranks
    double c[2] = {(double)dS, (double)dN};
    if (int rc = reduce_all(s, KFVM_REDUCE_SUM, c, 2)) return rc;
    dS = (unsigned long long)c[0];
    dN = (unsigned long long)c[1];
  }
  if (s->sameOn) {
    if (dN > 0 && 4 * dS < dN) {
      s->sameOn = false;
      s->sameProbe = kSameProbeSteps;
    }
  } else if (--s->sameProbe <= 0) {
    s->sameOn = true;
  }
  return KFVM_OK;
}

// the reference's wenothresh sign switch: a positive threshold allows the sparse
// (selected-cells) WENO mode, for KXRCF and for the learned indicator alike
bool sparse_allowed(const kfvm_solver *s) {
  return s->cfg.weno_thresh > 0.0 && (s->indicator == KFVM_IND_KXRCF || s->indicator == KFVM_IND_MLP);
}

double bits_to_double(unsigned long long b) {
  double d;
  std::memcpy(&d, &b, sizeof(d));
  return d;
}

// ---------------------------------------------------------------------------
// boundary communication of a decomposed domain (Solver.cpp:744-1460)

// in-place reduction of n host doubles over all ranks (identity on one domain)
int reduce_all(kfvm_solver *s, int op, double *vals, int n) {
  if (!s->decomposed) return KFVM_OK;
  if (!s->rfn) return fail(KFVM_ERR_STATE, "exchange faces but no transport (kfvm_set_exchange)");
  if (s->rfn(s->xuser, op, vals, n) != 0) return fail(KFVM_ERR_STATE, "the allreduce callback failed");
  return KFVM_OK;
}

// the halo of buffer b: one launch on one domain; on a decomposed domain axis by
// axis, exchange faces from the neighbours, the others from this block
int fill_halo(kfvm_solver *s, int b) {
  using namespace kfvm;
  cudaStream_t st = s->stream;
  double *U = s->Ub[b];
  if (!s->decomposed && !s->hasUser) {
    cudaError_t e = run(s, KFVM_KCLASS_BC, 1, [&] { return launch_bc(s->dim, s->eq, U, s->g, st); });
    return e == cudaSuccess ? KFVM_OK : set_err_cuda(e, "bc");
  }
  if (s->decomposed && !s->xfn) return fail(KFVM_ERR_STATE, "exchange faces but no transport (kfvm_set_exchange)");
  if (s->hasUser && !s->ufn) return fail(KFVM_ERR_STATE, "user boundary faces but no kfvm_set_user_bc");
  for (int d = 0; d < s->dim; d++) {
    const bool lo = s->g.bc[2 * d] == KFVM_BC_EXCHANGE, hi = s->g.bc[2 * d + 1] == KFVM_BC_EXCHANGE;
    // user faces: the interior layers out, the halo layers back (CellBc*_K<user>)
    for (int side = 0; side < 2; side++) {
      if (s->g.bc[2 * d + side] != KFVM_BC_USER) continue;
      const int64_t vals = cell_slab_values(s->g, s->dim, s->nv, d);
      CK(launch_cell_slab(s->dim, s->nv, U, s->g, d, side, true, s->xbuf[0], st));
      CK(cudaStreamSynchronize(st));
      if (s->ufn(s->uuser, KFVM_USER_CELLS, 2 * d + side, s->tEval, s->xbuf[0], s->xbuf[1], vals / s->nv,
                 (void *)st) != 0)
        return fail(KFVM_ERR_STATE, "the user boundary callback failed");
      CK(launch_cell_slab(s->dim, s->nv, U, s->g, d, side, false, s->xbuf[1], st));
      s->launches += 2;
    }
    if (lo || hi) {
      const int64_t bytes = cell_slab_values(s->g, s->dim, s->nv, d) * (int64_t)sizeof(double);
      if (lo) CK(launch_cell_slab(s->dim, s->nv, U, s->g, d, 0, true, s->xbuf[0], st));
      if (hi) CK(launch_cell_slab(s->dim, s->nv, U, s->g, d, 1, true, s->xbuf[2], st));
      s->launches += (lo ? 1 : 0) + (hi ? 1 : 0);
      CK(cudaStreamSynchronize(st));
      if (s->xfn(s->xuser, d, lo ? s->xbuf[0] : nullptr, lo ? s->xbuf[1] : nullptr, hi ? s->xbuf[2] : nullptr,
                 hi ? s->xbuf[3] : nullptr, lo ? bytes : 0, hi ? bytes : 0) != 0)
        return fail(KFVM_ERR_STATE, "the halo exchange callback failed");
      if (lo) CK(launch_cell_slab(s->dim, s->nv, U, s->g, d, 0, false, s->xbuf[1], st));
      if (hi) CK(launch_cell_slab(s->dim, s->nv, U, s->g, d, 1, false, s->xbuf[3], st));
      s->launches += (lo ? 1 : 0) + (hi ? 1 : 0);
    }
    cudaError_t e = run(s, KFVM_KCLASS_BC, 1, [&] { return launch_bc_axis(s->dim, s->nv, U, s->g, d, st); });
    if (e != cudaSuccess) return set_err_cuda(e, "bc");
  }
  return KFVM_OK;
}

// the outer face states (and with W the KXRCF indicator) of every exchange face
int exchange_faces(kfvm_solver *s, bool withW) {
  using namespace kfvm;
  if (!s->decomposed && !s->hasUser) return KFVM_OK;
  cudaStream_t st = s->stream;
  const int nqf = s->dim == 2 ? s->g.nq : s->g.nq * s->g.nq;
  for (int d = 0; d < s->dim; d++) {
    // user faces: the inner states out, the outer states back (FaceBc*_K<user>),
    // then the outer indicator from them
    for (int side = 0; side < 2; side++) {
      if (s->g.bc[2 * d + side] != KFVM_BC_USER) continue;
      const int64_t pts = face_plane_bytes(s->g, nqf, s->nv, d, false) / (int64_t)(s->nv * sizeof(double));
      CK(launch_face_plane(s->F[d], nullptr, s->g, nqf, s->nv, d, side, true, s->xbuf[0], st));
      CK(cudaStreamSynchronize(st));
      if (s->ufn(s->uuser, KFVM_USER_FACES, 2 * d + side, s->tEval, s->xbuf[0], s->xbuf[1], pts, (void *)st) != 0)
        return fail(KFVM_ERR_STATE, "the user boundary callback failed");
      CK(launch_face_plane(s->F[d], nullptr, s->g, nqf, s->nv, d, side, false, s->xbuf[1], st));
      s->launches += 2;
      if (withW) {
        CK(launch_face_indicator(s->dim, s->eq, s->F[d], s->W[d], s->g, nqf, d, side, st));
        s->launches += 1;
      }
    }
    if (!s->decomposed) continue;
    const bool lo = s->g.bc[2 * d] == KFVM_BC_EXCHANGE, hi = s->g.bc[2 * d + 1] == KFVM_BC_EXCHANGE;
    if (!lo && !hi) continue;
    float *W = withW ? s->W[d] : nullptr;
    const int64_t bytes = face_plane_bytes(s->g, nqf, s->nv, d, withW);
    if (lo) CK(launch_face_plane(s->F[d], W, s->g, nqf, s->nv, d, 0, true, s->xbuf[0], st));
    if (hi) CK(launch_face_plane(s->F[d], W, s->g, nqf, s->nv, d, 1, true, s->xbuf[2], st));
    CK(cudaStreamSynchronize(st));
    if (s->xfn(s->xuser, 3 + d, lo ? s->xbuf[0] : nullptr, lo ? s->xbuf[1] : nullptr, hi ? s->xbuf[2] : nullptr,
               hi ? s->xbuf[3] : nullptr, lo ? bytes : 0, hi ? bytes : 0) != 0)
      return fail(KFVM_ERR_STATE, "the face exchange callback failed");
    if (lo) CK(launch_face_plane(s->F[d], W, s->g, nqf, s->nv, d, 0, false, s->xbuf[1], st));
    if (hi) CK(launch_face_plane(s->F[d], W, s->g, nqf, s->nv, d, 1, false, s->xbuf[3], st));
    s->launches += 2 * ((lo ? 1 : 0) + (hi ? 1 : 0));
  }
  return KFVM_OK;
}

// one RHS evaluation on buffer b: BCs, selection, reconstruction, Riemann fluxes.
// The caller launches the stage kernel that consumes the fluxes.
int eval_front(kfvm_solver *s, int b) {
  using namespace kfvm;
  s->nRhs++;
  cudaStream_t st = s->stream;
  const int dim = s->dim, eq = s->eq;
  cudaError_t e;
  if (int rc = fill_halo(s, b)) return rc;
  // reset the per-evaluation counters (nflag, napplied, nheavy) and the GLM maxima
  CK(cudaMemsetAsync(&s->sc->glm_lam_bits, 0, 2 * sizeof(unsigned long long) + 3 * sizeof(unsigned), st));
  int mode;
  if (s->indicator == KFVM_IND_NONE) {
    mode = RECON_LINEAR;
  } else if (s->useSparseWeno) {
    mode = RECON_SPARSE;
  } else {
    mode = RECON_FULL;
    // after a full-WENO evaluation the sparse mode is allowed again (Solver.cpp:439-443)
    s->useSparseWeno = sparse_allowed(s);
  }
  // the learned indicator selects the cells unless its judge has made the host
  // fall back to KXRCF for a few steps
  const bool mlpOn = s->indicator == KFVM_IND_MLP && s->mlp.fallbackSteps == 0;
  const bool wantInd = mode == RECON_SPARSE && !mlpOn;
  if (mode != RECON_FULL) {
    if ((e = run(s, KFVM_KCLASS_RECON, s->precision == KFVM_PREC_TF32X3 ? 2 : 1, [&] {
           if (s->precision == KFVM_PREC_TF32X3) {
             // the limiter bounds of every cell, then the linear states
             cudaError_t eb = launch_bounds(dim, eq, s->Ub[b], s->g, s->bnd, st);
             if (eb != cudaSuccess) return eb;
             return launch_recon_tc(dim, eq, s->Ub[b], s->umapOk ? &s->umap[b] : nullptr, s->g, s->dS, wantInd,
                                    s->F, s->W, s->src, s->status,
                                    s->lamvel, s->bnd, s->sc, st);
           }
           return launch_recon(dim, eq, s->Ub[b], s->dmapOk ? &s->dmap[b] : nullptr, s->g, s->dS, wantInd, s->F,
                               s->W, s->src, s->status, s->lamvel, s->bnd, s->sc, st);
         })) != cudaSuccess)
      return set_err_cuda(e, "recon");
  }
  // the first setFaceBCs of evalRHS: the selector reads the neighbours' states
  if (mode == RECON_SPARSE && !mlpOn)
    if (int rc = exchange_faces(s, wantInd)) return rc;
  if (mode == RECON_SPARSE) {
    const double thr = s->cfg.weno_thresh * std::pow(s->dmin, 1.5);
    if ((e = run(s, KFVM_KCLASS_FLAG, mlpOn ? 2 : 1, [&] {
           if (mlpOn)
             return launch_mlp_flag(dim, eq, s->Ub[b], s->g, s->mlp.tiles, s->mlp.img, s->theta,
                                    s->flag, s->mlp.pred, s->sc, (float)s->mlp.logitThr, st);
           return launch_flag(dim, eq, s->Ub[b], s->g, s->W, s->F, s->theta, s->flag, s->sc, thr, st);
         })) != cudaSuccess)
      return set_err_cuda(e, "flag");
  }
  JudgeArgs jd{0.0, 0, s->mlp.tau, s->mlp.pred};
  if (mlpOn && mode == RECON_SPARSE) {
    jd.frac = s->mlp.judgeFrac;
    jd.seed = 0x6a75646765ull ^ (uint64_t)s->nRhs;
  }
  if ((e = run(s, KFVM_KCLASS_SELECT, 1, [&] {
         return launch_compact(dim, eq, s->g, mode, s->flag, s->wset, s->status, s->applied, s->theta, s->heavy,
                               s->lamvel, s->sc, jd, st);
       })) != cudaSuccess)
    return set_err_cuda(e, "compact");
  if ((e = run(s, KFVM_KCLASS_HEAVY, 1, [&] {
         return launch_heavy(dim, eq, s->Ub[b], s->g, s->dS, s->theta, s->F, s->src, s->heavy,
                             mode == RECON_FULL ? nullptr : s->bnd, s->sc, jd, s->heavyBlocks, st);
       })) != cudaSuccess)
    return set_err_cuda(e, "heavy");
  if (s->decomposed || s->hasUser) {
    // the second setFaceBCs, and the GLM cleaning speed over all ranks (glmSpeedComm)
    if (int rc = exchange_faces(s, false)) return rc;
    if (eq == EQ_GLM && s->decomposed) {
      unsigned long long bits[2];
      CK(cudaMemcpyAsync(bits, &s->sc->glm_lam_bits, sizeof(bits), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      double v[2] = {bits_to_double(bits[0]), bits_to_double(bits[1])};
      if (int rc = reduce_all(s, KFVM_REDUCE_MAX, v, 2)) return rc;
      std::memcpy(bits, v, sizeof(bits));
      CK(cudaMemcpyAsync(&s->sc->glm_lam_bits, bits, sizeof(bits), cudaMemcpyHostToDevice, st));
      CK(cudaStreamSynchronize(st));
    }
  }
  if ((e = run(s, KFVM_KCLASS_RIEMANN, dim,
               [&] { return launch_riemann(dim, eq, s->F, s->G, s->g, s->sc, s->sameOn, st); })) !=
      cudaSuccess)
    return set_err_cuda(e, "riemann");
  return KFVM_OK;
}

kfvm::StageArgs stage_args(kfvm_solver *s, int bIn, int bOut, int mode) {
  kfvm::StageArgs a;
  std::memset(&a, 0, sizeof(a));
  a.U = s->Ub[bIn];
  a.Unext = bOut >= 0 ? s->Ub[bOut] : nullptr;
  a.Uprev = s->Ub[s->iPrev];
  a.Uhat = s->Uhat;
  a.Utmp = s->Utmp;
  a.K = s->K;
  a.G = s->G;
  a.F = s->F;
  a.src = s->src;
  a.theta = s->theta;
  a.mode = mode;
  a.Re = s->cfg.reynolds;
  a.Pr = s->cfg.prandtl;
  a.atol = s->cfg.atol;
  a.rtol = s->cfg.rtol;
  a.part = s->part;
  a.sc = s->sc;
  a.co.use_tmp = s->rk.use_tmp ? 1 : 0;
  return a;
}

// evalRHS(U_b) followed by K = RHS
int eval_into_K(kfvm_solver *s, int b) {
  int rc = eval_front(s, b);
  if (rc) return rc;
  kfvm::StageArgs a = stage_args(s, b, -1, kfvm::STAGE_EVAL);
  cudaError_t e = run(s, KFVM_KCLASS_STAGE, 1, [&] { return kfvm::launch_stage(s->dim, s->eq, a, s->g, s->stream); });
  if (e != cudaSuccess) return set_err_cuda(e, "stage");
  return KFVM_OK;
}

// tail of Solver::Solver: Uprev = U, prime FSAL, dt = 0.01 cfl dmin / maxVel
int prime(kfvm_solver *s) {
  s->iCur = s->iPrev;
  s->time = 0.0;
  s->errEst = 1.0;
  s->lastTimeStep = false;
  s->nTS = 1;
  s->useSparseWeno = sparse_allowed(s);
  s->mlp.fallbackSteps = 0;
  s->mlp.lastPos = s->mlp.lastMissed = 0;
  const int64_t n = s->g.n;
  CK(cudaMemsetAsync(s->wset, 0, n, s->stream));
  CK(cudaMemsetAsync(s->sc, 0, sizeof(kfvm::DevScalars), s->stream));
  CK(kfvm::launch_fill(s->theta, n, 1.0, s->stream));
  s->tEval = s->time;
  int rc = eval_into_K(s, s->iPrev);
  if (rc) return rc;
  CK(cudaMemcpyAsync(s->hsc, s->sc, sizeof(kfvm::DevScalars), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  if (s->hsc->fault) return fail(KFVM_ERR_CUDA, kFaultMsg);
  double maxVel = bits_to_double(s->hsc->maxvel_bits);
  if (int rc2 = reduce_all(s, KFVM_REDUCE_MAX, &maxVel, 1)) return rc2;  // rhsSpeedComm
  s->nWenoLast = s->hsc->napplied;
  s->dt = 0.01 * s->cfg.cfl * s->dmin / maxVel;
  s->primed = true;
  return KFVM_OK;
}

// Solver::TakeStep (Solver.cpp:188-343)
int take_step(kfvm_solver *s, kfvm_step_info *info) {
  using namespace kfvm;
  if (!s->primed) return fail(KFVM_ERR_STATE, "take_step before an initial condition was set");
  const RKTable &rk = s->rk;
  cudaStream_t st = s->stream;
  // limit dt to hit the final time or the next plot time (Solver.cpp:197-205)
  if (s->time + s->dt > s->cfg.final_time) {
    s->dt = s->cfg.final_time - s->time;
    s->lastTimeStep = true;
    s->writePlot = true;
  } else if (s->plotFreq > 0.0 && s->time + s->dt > s->plotNum * s->plotFreq) {
    s->dt = s->plotNum * s->plotFreq - s->time;
    s->writePlot = true;
  }
  bool accepted = false, firstUnphys = true;
  double maxVel = 0.0, errNew = 0.0, dtTaken = 0.0;
  int lStat = KFVM_TS_ACCEPTED, nT;
  const int bA = (s->iPrev + 1) % 3, bB = (s->iPrev + 2) % 3;
  CK(cudaEventRecord(s->ev0, st));
  for (nT = 0; nT < s->cfg.rejection_limit; nT++) {
    CK(cudaMemsetAsync(&s->sc->maxvel_bits, 0, sizeof(unsigned long long), st));
    if (nT > 0) {
      s->tEval = s->time;
      int rc = eval_into_K(s, s->iPrev);
      if (rc) return rc;
    }
    cudaError_t e = run(s, KFVM_KCLASS_OTHER, 1, [&] {
      return launch_stage_pre(s->dim, s->eq, s->Ub[bA], s->Ub[s->iPrev], s->Uhat, s->Utmp, s->K, s->g,
                              rk.beta[0] * s->dt, rk.bhat[0] * s->dt, rk.use_tmp ? 1 : 0, st);
    });
    if (e != cudaSuccess) return set_err_cuda(e, "stage_pre");
    int cur = bA, nxt = bB;
    for (int nS = 1; nS < rk.nStages; nS++) {
      s->tEval = s->time + rk.c[nS] * s->dt;
      int rc = eval_front(s, cur);
      if (rc) return rc;
      StageArgs a = stage_args(s, cur, nxt, STAGE_UPDATE);
      a.co.delta = rk.delta[nS];
      a.co.g1 = rk.gam1[nS];
      a.co.g2 = rk.gam2[nS];
      a.co.g3 = rk.gam3[nS];
      a.co.betaDt = rk.beta[nS] * s->dt;
      a.co.bhatDt = rk.bhat[nS] * s->dt;
      if ((e = run(s, KFVM_KCLASS_STAGE, 1, [&] { return launch_stage(s->dim, s->eq, a, s->g, st); })) !=
          cudaSuccess)
        return set_err_cuda(e, "stage");
      std::swap(cur, nxt);
    }
    // FSAL stage: K = RHS(U), Uhat += bhatfsal dt K, error estimate
    s->tEval = s->time + s->dt;
    int rc = eval_front(s, cur);
    if (rc) return rc;
    StageArgs a = stage_args(s, cur, -1, STAGE_FSAL);
    a.co.bhatDt = rk.bhatfsal * s->dt;
    if ((e = run(s, KFVM_KCLASS_STAGE, 2, [&] { return launch_stage(s->dim, s->eq, a, s->g, st); })) !=
        cudaSuccess)
      return set_err_cuda(e, "fsal");
    CK(cudaMemcpyAsync(s->hsc, s->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (s->hsc->fault) return fail(KFVM_ERR_CUDA, kFaultMsg);
    maxVel = bits_to_double(s->hsc->maxvel_bits);
    s->nWenoLast = s->hsc->napplied;
    if (int rc2 = update_same_mode(s)) return rc2;
    // over all ranks (rhsSpeedComm, timeStepErrEstComm, timeStepStatusComm): the
    // wave-speed maximum, the error sum over every degree of freedom of the domain
    // and the positivity minimum (the status follows from it and the error)
    double errSum = s->hsc->err, posFlag = s->hsc->posmin;
    if (s->decomposed) {
      if (int rc2 = reduce_all(s, KFVM_REDUCE_MAX, &maxVel, 1)) return rc2;
      if (int rc2 = reduce_all(s, KFVM_REDUCE_SUM, &errSum, 1)) return rc2;
      if (int rc2 = reduce_all(s, KFVM_REDUCE_MIN, &posFlag, 1)) return rc2;
    }
    const double nDofs = (double)(s->g.n * s->nv) * kfvm::cfg_nb(&s->cfg, 0) * kfvm::cfg_nb(&s->cfg, 1) *
                         kfvm::cfg_nb(&s->cfg, 2);
    errNew = 1.0 / std::sqrt(errSum / nDofs);
    double dtfac = std::pow(errNew, rk.ep1) * std::pow(s->errEst, rk.ep2);
    dtfac = std::isnan(dtfac) ? 1.2 : 1.0 + std::atan(dtfac - 1.0);
    if (posFlag < 0.0) lStat = KFVM_TS_UNPHYSICAL;
    else if (dtfac >= s->cfg.rejection_thresh) lStat = KFVM_TS_ACCEPTED;
    else lStat = KFVM_TS_TOLERANCE;

    if (lStat == KFVM_TS_UNPHYSICAL) {
      s->dt = firstUnphys ? std::fmin(0.25 * s->cfg.cfl * s->dmin / maxVel, s->dt / 4.0) : s->dt / 2.0;
      firstUnphys = false;
      s->useSparseWeno = false; // force full WENO on the retry
      if (s->lastTimeStep) {
        s->lastTimeStep = false;
        s->writePlot = false;
      }
    } else if (lStat == KFVM_TS_ACCEPTED) {
      accepted = true;
      dtTaken = s->dt;
      s->time += s->dt;
      const double dterr = s->dt * dtfac, dtcfl = s->cfg.cfl * s->dmin / maxVel;
      s->dt = std::fmin(dterr, dtcfl);
      s->errEst = errNew;
      // Uprev <- U by buffer rotation instead of a copy
      s->iPrev = cur;
      s->iCur = cur;
      // judge of the learned indicator: too many troubled cells missed in this step
      // sends the next steps to KXRCF
      if (s->indicator == KFVM_IND_MLP) {
        if (s->mlp.fallbackSteps > 0) s->mlp.fallbackSteps--;
        const unsigned long long dPos = s->hsc->mlp_pos - s->mlp.lastPos;
        const unsigned long long dMiss = s->hsc->mlp_missed - s->mlp.lastMissed;
        s->mlp.lastPos = s->hsc->mlp_pos;
        s->mlp.lastMissed = s->hsc->mlp_missed;
        if (dPos >= 8 && (double)dMiss > s->mlp.missLimit * (double)dPos) {
          s->mlp.fallbackSteps = 2;
          s->mlp.fallbackEvents++;
        }
      }
      nT++;
      break;
    } else {
      s->dt = s->dt * dtfac;
      if (s->lastTimeStep) {
        s->lastTimeStep = false;
        s->writePlot = false;
      }
    }
  }
  CK(cudaEventRecord(s->ev1, st));
  CK(cudaEventSynchronize(s->ev1));
  CK(cudaEventElapsedTime(&s->lastMs, s->ev0, s->ev1));
  harvest(s);
  if (!accepted) s->lastTimeStep = true;
  if (s->dt < s->cfg.min_dt) s->lastTimeStep = true;
  if (info) {
    info->time = s->time;
    info->dt = s->dt;
    info->dt_taken = dtTaken;
    info->max_vel = maxVel;
    info->err_est = errNew;
    info->status = lStat;
    info->attempts = nT;
    info->accepted = accepted ? 1 : 0;
    info->last_step = s->lastTimeStep ? 1 : 0;
    info->n_weno = s->nWenoLast;
    info->n_rhs = s->nRhs;
    info->write_plot = s->writePlot ? 1 : 0;
  }
  s->writePlot = false; // reported once
  return KFVM_OK;
}

// the host-order interior state (variable, k, j, i) travels as one contiguous copy
// through a device staging buffer; a kernel moves it to or from the padded layout
// (strided 3D copies of 2 KB rows ran at a fraction of the link bandwidth)
int ensure_io(kfvm_solver *s) {
  if (!s->io) CK(cudaMalloc(&s->io, (size_t)s->g.n * s->nv * sizeof(double)));
  return KFVM_OK;
}

int upload_state(kfvm_solver *s, int b, const double *u) {
  if (int rc = ensure_io(s)) return rc;
  CK(cudaMemcpyAsync(s->io, u, (size_t)s->g.n * s->nv * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  CK(kfvm::launch_interior(s->Ub[b], s->io, s->g, s->nv, true, s->stream));
  return KFVM_OK;
}

} // namespace

int kfvm::set_last_error(int code, const std::string &msg) { return fail(code, msg); }

extern "C" {

const char *kfvm_last_error(void) { return g_err.c_str(); }

void kfvm_default_config(kfvm_config *c) {
  std::memset(c, 0, sizeof(*c));
  c->dim = 2;
  c->eq = KFVM_EQ_HYDRO;
  c->rs = KFVM_RS_HLLC;
  c->rk = KFVM_RK_SSP4_3_2;
  c->nq = 2;
  c->indicator = KFVM_IND_KXRCF;
  c->nx = c->ny = c->nz = 1;
  c->xlo = c->ylo = c->zlo = 0.0;
  c->xup = c->yup = c->zup = 1.0;
  c->gamma = (double)1.4f;
  c->reynolds = 1.0;
  c->prandtl = (double)0.71f;
  c->weno_thresh = 10.0;
  c->lfac = 20.0;
  c->cfl = c->dim == 3 ? 0.5 : 0.75;
  c->atol = (double)1.e-4f;
  c->rtol = (double)1.e-4f;
  c->rejection_thresh = (double)0.8f;
  c->min_dt = (double)1.e-10f;
  c->final_time = 1.0;
  c->rejection_limit = 4;
  c->max_steps = 1000;
  c->nb[0] = c->nb[1] = c->nb[2] = 1;  // one block (mesh:numblocks 1 1 1)
}

int kfvm_stencil_build(const kfvm_config *cfg, kfvm_stencil *out) {
  if (!cfg || !out) return fail(KFVM_ERR_ARG, "null argument");
  const int rc = kfvm::build_stencil(cfg, out);
  if (rc) return fail(rc, "stencil weight precompute failed");
  return KFVM_OK;
}

int kfvm_create(const kfvm_config *cfg, kfvm_solver **out) {
  using namespace kfvm;
  if (!cfg || !out) return fail(KFVM_ERR_ARG, "null argument");
  *out = nullptr;
  if (cfg->dim != 2 && cfg->dim != 3) return fail(KFVM_ERR_ARG, "dim must be 2 or 3");
  if (!(cfg->nq == 2 || (cfg->nq == 3 && (cfg->dim == 2 || cfg->eq != KFVM_EQ_SRHYDRO))))
    return fail(KFVM_ERR_ARG, "the GPU path supports NUM_QUAD_PTS = 2, and 3 in 2D and for 3D Euler / Navier-Stokes / GLM-MHD");
  if (cfg->eq < KFVM_EQ_HYDRO || cfg->eq > KFVM_EQ_SRHYDRO) return fail(KFVM_ERR_ARG, "unknown equation type");
  if (cfg->rs < 0 || cfg->rs > 2) return fail(KFVM_ERR_ARG, "unknown Riemann solver");
  if (cfg->eq == KFVM_EQ_MHD_GLM && cfg->rs == KFVM_RS_HLLC)
    return fail(KFVM_ERR_ARG, "HLLC is not defined for MHD_GLM");
  if (cfg->eq == KFVM_EQ_SRHYDRO && cfg->rs == KFVM_RS_HLLC)
    return fail(KFVM_ERR_ARG, "the SRHydro Riemann solvers are HLL and LLF");
  if (cfg->eq == KFVM_EQ_SRHYDRO && cfg->indicator == KFVM_IND_MLP)
    return fail(KFVM_ERR_ARG, "the learned indicator is trained for the Euler / GLM-MHD paths");
  const int64_t nz = cfg->dim == 3 ? cfg->nz : 1;
  if (cfg->nx * cfg->ny * nz > (int64_t)kfvm::kHeavyCellMax + 1)
    return fail(KFVM_ERR_ARG, "more than 2^29 cells (the WENO cell list packs a cell index in 29 bits)");
  if (cfg->nx < 3 || cfg->ny < 3 || nz < (cfg->dim == 3 ? 3 : 1))
    return fail(KFVM_ERR_ARG, "grid too small for a radius-2 stencil");
  for (int d = 0; d < cfg->dim; d++) {
    if ((cfg->bc[2 * d] == KFVM_BC_PERIODIC) != (cfg->bc[2 * d + 1] == KFVM_BC_PERIODIC))
      return fail(KFVM_ERR_ARG, "periodic boundaries must come in pairs");
    for (int f = 2 * d; f < 2 * d + 2; f++)
      if (cfg->bc[f] < KFVM_BC_PERIODIC || cfg->bc[f] > KFVM_BC_EXCHANGE)
        return fail(KFVM_ERR_ARG, "unknown boundary condition (periodic, outflow, reflecting, noslip, exchange, user)");
  }
  for (int d = 0; d < 3; d++)
    if (cfg->nb[d] > 1 && (cfg->block[d] < 0 || cfg->block[d] >= cfg->nb[d]))
      return fail(KFVM_ERR_ARG, "block coordinate outside the block counts");
  kfvm_solver *s = new kfvm_solver();
  s->cfg = *cfg;
  s->cfg.nz = nz;
  s->dim = cfg->dim;
  s->eq = cfg->eq;
  s->nv = cfg->eq == KFVM_EQ_MHD_GLM ? 9 : 5;
  s->indicator = cfg->indicator;
  if (!rk_table(cfg->rk, s->rk)) {
    delete s;
    return fail(KFVM_ERR_ARG, "unsupported RK scheme");
  }
  Grid &g = s->g;
  std::memset(&g, 0, sizeof(g));
  g.nx = cfg->nx;
  g.ny = cfg->ny;
  g.nz = nz;
  g.n = g.nx * g.ny * g.nz;
  g.px = g.nx + 2 * kRad;
  g.py = g.ny + 2 * kRad;
  g.rz = cfg->dim == 3 ? kRad : 0;
  g.pvol = g.px * g.py * (cfg->dim == 3 ? nz + 2 * kRad : 1);
  for (int d = 0; d < 3; d++) {
    g.fdim[d][0] = g.nx + (d == 0);
    g.fdim[d][1] = g.ny + (d == 1);
    g.fdim[d][2] = g.nz + (d == 2);
    g.nface[d] = g.fdim[d][0] * g.fdim[d][1] * g.fdim[d][2];
  }
  // cell sizes and this block's global offset (Geometry.H:28-31; nb = 1: one domain)
  g.dx = cfg_dx(cfg, 0);
  g.dy = cfg_dx(cfg, 1);
  g.dz = cfg_dx(cfg, 2);
  for (int d = 0; d < 3; d++) {
    g.off[d] = cfg_offset(cfg, d);
    g.gn[d] = cfg_n(cfg, d) * cfg_nb(cfg, d);
  }
  g.rdx = 1.0 / g.dx;
  g.rdy = 1.0 / g.dy;
  g.rdz = 1.0 / g.dz;
  for (int f = 0; f < 6; f++) {
    g.bc[f] = cfg->bc[f];
    g.bflip[f] = wall_flip(cfg->bc[f], f / 2, cfg->eq == KFVM_EQ_MHD_GLM);
    if (f < 2 * cfg->dim && cfg->bc[f] == KFVM_BC_EXCHANGE) s->decomposed = true;
    if (f < 2 * cfg->dim && cfg->bc[f] == KFVM_BC_USER) s->hasUser = true;
  }
  g.gamma = cfg->gamma;
  g.rs = cfg->rs;
  g.nq = cfg->nq;
  s->dmin = cfg->dim == 2 ? std::fmin(g.dx, g.dy) : std::fmin(g.dx, std::fmin(g.dy, g.dz));

  DevStencil hS;
  std::memset(&hS, 0, sizeof(hS));
  int rc = build_stencil(&s->cfg, &hS.w);
  if (rc) {
    delete s;
    return fail(rc, "stencil weight precompute failed");
  }
  for (int c = 0; c < hS.w.n_cells; c++)
    hS.loff[c] = (hS.w.off[2][c] * g.py + hS.w.off[1][c]) * g.px + hS.w.off[0][c];
  for (int c = 0; c < hS.w.n_cells; c++) g.loff[c] = hS.loff[c];
  {
    // full-stencil linear weights as [cell][row]: face rows f*NQF+q, then interior rows
    const int C = hS.w.n_cells, nqf = hS.w.nqf, nf = 2 * cfg->dim;
    const int nrows = nf * nqf + (cfg->eq == KFVM_EQ_MHD_GLM ? hS.w.nqc : 0);
    for (int c = 0; c < C; c++) {
      int r = 0;
      for (int f = 0; f < nf; f++)
        for (int q = 0; q < nqf; q++) hS.lin[c * nrows + r++] = hS.w.face_w[0][f][q][c];
      if (cfg->eq == KFVM_EQ_MHD_GLM)
        for (int q = 0; q < hS.w.nqc; q++) hS.lin[c * nrows + r++] = hS.w.cell_w[0][q][c];
    }
    if (cfg->nq == 2) fill_tc_weights(hS, cfg->dim, nrows);  // the tensor-core form takes 2 points only
    fill_dmma_weights(hS, nrows);
  }

  auto cleanup = [&](cudaError_t e, const char *what) {
    kfvm_destroy(s);
    return set_err_cuda(e, what);
  };
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)) != cudaSuccess) return cleanup(e, "stream");
  if ((e = cudaEventCreate(&s->ev0)) != cudaSuccess) return cleanup(e, "event");
  if ((e = cudaEventCreate(&s->ev1)) != cudaSuccess) return cleanup(e, "event");
  const size_t nv = s->nv, n = g.n;
  const int nqf = cfg->dim == 2 ? cfg->nq : cfg->nq * cfg->nq;
  const int nqc = cfg->dim == 2 ? cfg->nq * cfg->nq : cfg->nq * cfg->nq * cfg->nq;
  auto dalloc = [&](void **p, size_t bytes) { return cudaMalloc(p, bytes); };
  if ((e = dalloc((void **)&s->dS, sizeof(DevStencil))) != cudaSuccess) return cleanup(e, "alloc");
  for (int b = 0; b < 3; b++)
    if ((e = dalloc((void **)&s->Ub[b], g.pvol * nv * sizeof(double))) != cudaSuccess) return cleanup(e, "alloc U");
  if ((e = dalloc((void **)&s->Uhat, n * nv * sizeof(double))) != cudaSuccess) return cleanup(e, "alloc");
  if ((e = dalloc((void **)&s->K, n * nv * sizeof(double))) != cudaSuccess) return cleanup(e, "alloc");
  if (s->rk.use_tmp && (e = dalloc((void **)&s->Utmp, n * nv * sizeof(double))) != cudaSuccess)
    return cleanup(e, "alloc");
  for (int d = 0; d < cfg->dim; d++) {
    if ((e = dalloc((void **)&s->F[d], 2 * nqf * nv * g.nface[d] * sizeof(double))) != cudaSuccess)
      return cleanup(e, "alloc faces");
    if ((e = dalloc((void **)&s->G[d], nv * g.nface[d] * sizeof(double))) != cudaSuccess)
      return cleanup(e, "alloc fluxes");
    if ((e = dalloc((void **)&s->W[d], 2 * nqf * g.nface[d] * sizeof(float))) != cudaSuccess)
      return cleanup(e, "alloc indicator");
  }
  if (cfg->eq == KFVM_EQ_MHD_GLM &&
      (e = dalloc((void **)&s->src, (size_t)nqc * nv * n * sizeof(double))) != cudaSuccess)
    return cleanup(e, "alloc");
  if ((e = dalloc((void **)&s->theta, n * sizeof(double))) != cudaSuccess) return cleanup(e, "alloc");
  if ((e = dalloc((void **)&s->bnd, 3 * n * sizeof(double))) != cudaSuccess) return cleanup(e, "alloc");
  if ((e = dalloc((void **)&s->flag, n)) != cudaSuccess) return cleanup(e, "alloc");
  if ((e = dalloc((void **)&s->wset, n)) != cudaSuccess) return cleanup(e, "alloc");
  if ((e = dalloc((void **)&s->applied, n)) != cudaSuccess) return cleanup(e, "alloc");
  if ((e = dalloc((void **)&s->heavy, n * sizeof(uint32_t))) != cudaSuccess) return cleanup(e, "alloc");
  if ((e = dalloc((void **)&s->status, n)) != cudaSuccess) return cleanup(e, "alloc");
  if (cfg->eq == KFVM_EQ_MHD_GLM && (e = dalloc((void **)&s->lamvel, n * sizeof(double2))) != cudaSuccess)
    return cleanup(e, "alloc");
  {
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    s->heavyBlocks = (nsm > 0 ? nsm : 148) * 4; // grid-stride over the device-side count
  }
  {
    const int64_t nb = std::max(std::max(stage_blocks(g), errest_blocks(g.n)), forcing_blocks(g));
    if ((e = dalloc((void **)&s->part, 2 * nb * sizeof(double))) != cudaSuccess) return cleanup(e, "alloc");
  }
  if ((e = dalloc((void **)&s->spart, 3 * stats_blocks(g) * sizeof(double))) != cudaSuccess) return cleanup(e, "alloc");
  if ((e = dalloc((void **)&s->ssum, 3 * sizeof(double))) != cudaSuccess) return cleanup(e, "alloc");
  if ((e = dalloc((void **)&s->sc, sizeof(DevScalars))) != cudaSuccess) return cleanup(e, "alloc");
  if ((e = cudaMallocHost((void **)&s->hsc, sizeof(DevScalars))) != cudaSuccess) return cleanup(e, "alloc host");
  for (int b = 0; b < 3; b++)
    if ((e = cudaMemsetAsync(s->Ub[b], 0, g.pvol * nv * sizeof(double), s->stream)) != cudaSuccess)
      return cleanup(e, "memset");
  if ((e = cudaMemcpyAsync(s->dS, &hS, sizeof(DevStencil), cudaMemcpyHostToDevice, s->stream)) != cudaSuccess)
    return cleanup(e, "upload stencil");
  if ((e = cudaMemsetAsync(s->sc, 0, sizeof(DevScalars), s->stream)) != cudaSuccess) return cleanup(e, "memset");

  if ((e = cudaStreamSynchronize(s->stream)) != cudaSuccess) return cleanup(e, "sync");
  // TMA maps of the FP64 reconstruction's halo tiles (five variables, or GLM-MHD in
  // 2D; even pitch; otherwise that kernel reads the state with plain loads)
  if (s->nv == 5 || s->dim == 2) {
    bool all = true;
    for (int b = 0; b < 3; b++) all = all && recon_dmma_state_map(&s->dmap[b], s->Ub[b], g, s->dim, s->nv) == 0;
    s->dmapOk = all;
  }
  *out = s;
  return KFVM_OK;
}

void kfvm_destroy(kfvm_solver *s) {
  if (!s) return;
  if (s->stream) cudaStreamSynchronize(s->stream);
  cudaFree(s->dS);
  for (int b = 0; b < 3; b++) cudaFree(s->Ub[b]);
  cudaFree(s->Uhat);
  cudaFree(s->Utmp);
  cudaFree(s->K);
  for (int d = 0; d < 3; d++) {
    cudaFree(s->F[d]);
    cudaFree(s->G[d]);
    cudaFree(s->W[d]);
  }
  cudaFree(s->status);
  cudaFree(s->lamvel);
  cudaFree(s->src);
  cudaFree(s->theta);
  cudaFree(s->bnd);
  cudaFree(s->io);
  cudaFree(s->flag);
  cudaFree(s->wset);
  cudaFree(s->applied);
  cudaFree(s->heavy);
  cudaFree(s->part);
  cudaFree(s->fmodes);
  cudaFree(s->spart);
  cudaFree(s->ssum);
  cudaFree(s->fsums);
  cudaFree(s->sc);
  for (int i = 0; i < 4; i++) cudaFree(s->xbuf[i]);
  if (s->hsc) cudaFreeHost(s->hsc);
  cudaFree(s->mlp.wb);
  cudaFree(s->mlp.wq);
  cudaFree(s->mlp.master);
  cudaFree(s->mlp.m);
  cudaFree(s->mlp.v);
  cudaFree(s->mlp.gpart);
  cudaFree(s->mlp.lpart);
  cudaFree(s->mlp.flags);
  cudaFree(s->mlp.sel);
  cudaFree(s->mlp.nsel);
  cudaFree(s->mlp.selTemp);
  cudaFree(s->mlp.loss);
  cudaFree(s->mlp.pred);
  cudaFree(s->mlp.img);
  cudaFree(s->mlp.tiles.rp);
  cudaFree(s->mlp.feats);
  cudaFree(s->mlp.labels);
  cudaFree(s->mlp.cells);
  cudaFree(s->mlp.count);
  if (s->ev0) cudaEventDestroy(s->ev0);
  if (s->ev1) cudaEventDestroy(s->ev1);
  for (auto &m : s->marks) {
    cudaEventDestroy(m.a);
    cudaEventDestroy(m.b);
  }
  for (auto e : s->evPool) cudaEventDestroy(e);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

int kfvm_init_ic(kfvm_solver *s, int32_t ic_kind, uint64_t seed) {
  if (!s) return fail(KFVM_ERR_ARG, "null solver");
  if (ic_kind < 0 || ic_kind > KFVM_IC_STIR_TURB) return fail(KFVM_ERR_ARG, "unknown initial condition");
  cudaError_t e = run(s, KFVM_KCLASS_OTHER, 1, [&] {
    return kfvm::launch_ic(s->dim, s->eq, ic_kind, seed, s->cfg, s->Ub[s->iPrev], s->g, s->stream);
  });
  if (e != cudaSuccess) return set_err_cuda(e, "ic");
  return prime(s);
}

int kfvm_set_state(kfvm_solver *s, const double *u) {
  if (!s || !u) return fail(KFVM_ERR_ARG, "null argument");
  int rc = upload_state(s, s->iPrev, u);
  if (rc) return rc;
  return prime(s);
}

int kfvm_get_state(kfvm_solver *s, double *u) {
  if (!s || !u) return fail(KFVM_ERR_ARG, "null argument");
  if (int rc = ensure_io(s)) return rc;
  CK(kfvm::launch_interior(s->Ub[s->iCur], s->io, s->g, s->nv, false, s->stream));
  CK(cudaMemcpyAsync(u, s->io, (size_t)s->g.n * s->nv * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return KFVM_OK;
}

int kfvm_eval_rhs(kfvm_solver *s, double t, double *rhs, double *max_vel) {
  if (!s) return fail(KFVM_ERR_ARG, "null solver");
  s->tEval = t;
  CK(cudaMemsetAsync(&s->sc->maxvel_bits, 0, sizeof(unsigned long long), s->stream));
  int rc = eval_into_K(s, s->iCur);
  if (rc) return rc;
  CK(cudaMemcpyAsync(s->hsc, s->sc, sizeof(kfvm::DevScalars), cudaMemcpyDeviceToHost, s->stream));
  if (rhs)
    CK(cudaMemcpyAsync(rhs, s->K, (size_t)s->g.n * s->nv * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  if (s->hsc->fault) return fail(KFVM_ERR_CUDA, kFaultMsg);
  s->nWenoLast = s->hsc->napplied;
  double mv = bits_to_double(s->hsc->maxvel_bits);
  if (int rc2 = reduce_all(s, KFVM_REDUCE_MAX, &mv, 1)) return rc2;  // rhsSpeedComm
  if (max_vel) *max_vel = mv;
  return KFVM_OK;
}

int kfvm_err_est(kfvm_solver *s, const double *u_dev, const double *uhat_dev, double *err,
                 double *posmin) {
  if (!s || !u_dev || !uhat_dev) return fail(KFVM_ERR_ARG, "null argument");
  cudaError_t e = run(s, KFVM_KCLASS_OTHER, 2, [&] {
    return kfvm::launch_errest(s->eq, u_dev, uhat_dev, s->g.n, s->cfg.atol, s->cfg.rtol, s->part, &s->sc->err,
                               s->stream);
  });
  if (e != cudaSuccess) return set_err_cuda(e, "err_est");
  CK(cudaMemcpyAsync(s->hsc, s->sc, sizeof(kfvm::DevScalars), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  if (err) *err = s->hsc->err;
  if (posmin) *posmin = s->hsc->posmin;
  return KFVM_OK;
}

int kfvm_take_step(kfvm_solver *s, kfvm_step_info *info) {
  if (!s) return fail(KFVM_ERR_ARG, "null solver");
  return take_step(s, info);
}

int kfvm_solve(kfvm_solver *s, int32_t max_steps, int64_t *n_steps_out, kfvm_step_info *last) {
  if (!s) return fail(KFVM_ERR_ARG, "null solver");
  kfvm_step_info info;
  std::memset(&info, 0, sizeof(info));
  int64_t acc = 0;
  for (; s->nTS < max_steps && !s->lastTimeStep; ++s->nTS) {
    // Solver::Solve (Solver.cpp:99-103): force before the step while time < t_off
    if (s->forcing && s->time < s->fpar.t_off) {
      int rc = kfvm_apply_forcing(s, nullptr, nullptr, nullptr);
      if (rc) return rc;
    }
    int rc = take_step(s, &info);
    if (rc) return rc;
    acc += info.accepted;
  }
  if (n_steps_out) *n_steps_out = acc;
  if (last) *last = info;
  return KFVM_OK;
}

int kfvm_get_time(kfvm_solver *s, double *time, double *dt) {
  if (!s) return fail(KFVM_ERR_ARG, "null solver");
  if (time) *time = s->time;
  if (dt) *dt = s->dt;
  return KFVM_OK;
}

int kfvm_set_time(kfvm_solver *s, double time, double dt) {
  if (!s || !(dt > 0.0)) return fail(KFVM_ERR_ARG, "bad argument");
  s->time = time;
  s->dt = dt;
  return KFVM_OK;
}

int kfvm_set_indicator(kfvm_solver *s, int32_t ind) {
  if (!s || ind < 0 || ind > KFVM_IND_MLP) return fail(KFVM_ERR_ARG, "bad indicator");
  if (ind == KFVM_IND_MLP && !s->mlp.ready)
    return fail(KFVM_ERR_STATE, "learned indicator: no weights (kfvm_mlp_set_weights or kfvm_mlp_init_weights + "
                                "kfvm_mlp_train)");
  if (ind == KFVM_IND_MLP && s->eq == KFVM_EQ_SRHYDRO)
    return fail(KFVM_ERR_ARG, "the learned indicator is trained for the Euler / GLM-MHD paths");
  s->indicator = ind;
  s->useSparseWeno = sparse_allowed(s);
  return KFVM_OK;
}

int kfvm_set_precision(kfvm_solver *s, int32_t precision) {
  if (!s || precision < KFVM_PREC_FP64 || precision > KFVM_PREC_TF32X3) return fail(KFVM_ERR_ARG, "bad precision");
  if (precision == KFVM_PREC_TF32X3) {
    // tcgen05 exists on compute capability 10.x only
    int dev = 0, major = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
    if (major != 10) return fail(KFVM_ERR_ARG, "the TF32 tensor-core form needs an sm_100 device");
    if (s->g.nq != 2) return fail(KFVM_ERR_ARG, "the TF32 tensor-core form is built for 2 Gauss points");
    if (s->eq == KFVM_EQ_SRHYDRO) return fail(KFVM_ERR_ARG, "the TF32 tensor-core form is built for the Euler / GLM-MHD paths");
    if (!s->umapOk) {
      bool all = true;
      for (int b = 0; b < 3; b++)
        all = all && kfvm::recon_tc_state_map(&s->umap[b], s->Ub[b], s->g, s->dim, s->nv) == 0;
      s->umapOk = all;
    }
  }
  s->precision = precision;
  return KFVM_OK;
}

// ---------------------------------------------------------------------------
// learned troubled-cell indicator
namespace {
uint16_t f2bf(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7fffffffu) > 0x7f800000u) return 0x7fc0; // NaN
  u += 0x7fffu + ((u >> 16) & 1u);                    // round to nearest even
  return (uint16_t)(u >> 16);
}
float bf2f(uint16_t b) {
  const uint32_t u = (uint32_t)b << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

int mlp_alloc(kfvm_solver *s) {
  auto &M = s->mlp;
  if (M.wb) return KFVM_OK;
  M.nw = kfvm::mlp_num_weights(s->dim);
  M.ni = kfvm::mlp_num_inputs(s->dim);
  cudaError_t e;
  if ((e = cudaMalloc((void **)&M.wb, M.nw * sizeof(uint16_t))) != cudaSuccess ||
      (e = cudaMalloc((void **)&M.wq, M.nw * sizeof(float))) != cudaSuccess ||
      (e = cudaMalloc((void **)&M.master, M.nw * sizeof(float))) != cudaSuccess ||
      (e = cudaMalloc((void **)&M.m, M.nw * sizeof(float))) != cudaSuccess ||
      (e = cudaMalloc((void **)&M.v, M.nw * sizeof(float))) != cudaSuccess ||
      (e = cudaMalloc((void **)&M.loss, 4 * sizeof(float))) != cudaSuccess ||
      (e = cudaMalloc((void **)&M.pred, s->g.n)) != cudaSuccess ||
      (e = cudaMalloc((void **)&M.img, kfvm::mlp_image_bytes(s->dim))) != cudaSuccess ||
      (e = kfvm::mlp_tile_buf_init(s->dim, s->g, M.tiles)) != cudaSuccess)
    return set_err_cuda(e, "learned indicator buffers");
  CK(cudaMemsetAsync(M.pred, 0, s->g.n, s->stream));
  return KFVM_OK;
}

// master = bf16 values, Adam state cleared
int mlp_load(kfvm_solver *s, const std::vector<float> &w) {
  auto &M = s->mlp;
  std::vector<uint16_t> b(M.nw);
  std::vector<float> q(M.nw);
  for (int i = 0; i < M.nw; i++) {
    b[i] = f2bf(w[i]);
    q[i] = bf2f(b[i]);
  }
  CK(cudaMemcpyAsync(M.wb, b.data(), M.nw * sizeof(uint16_t), cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemcpyAsync(M.wq, q.data(), M.nw * sizeof(float), cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemcpyAsync(M.master, q.data(), M.nw * sizeof(float), cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemsetAsync(M.m, 0, M.nw * sizeof(float), s->stream));
  CK(cudaMemsetAsync(M.v, 0, M.nw * sizeof(float), s->stream));
  cudaError_t e = kfvm::launch_mlp_pack(s->dim, M.wb, M.wq, M.img, s->stream);
  if (e != cudaSuccess) return set_err_cuda(e, "pack");
  CK(cudaStreamSynchronize(s->stream));
  M.t = 0;
  M.ready = true;
  return KFVM_OK;
}
} // namespace

int kfvm_mlp_num_weights(int32_t dim) {
  if (dim != 2 && dim != 3) return fail(KFVM_ERR_ARG, "dim must be 2 or 3");
  return kfvm::mlp_num_weights(dim);
}

int kfvm_mlp_init_weights(kfvm_solver *s, uint64_t seed) {
  if (!s) return fail(KFVM_ERR_ARG, "null solver");
  int rc = mlp_alloc(s);
  if (rc) return rc;
  const int ni = s->mlp.ni, nh = 32, nw = s->mlp.nw;
  std::vector<float> w(nw, 0.0f);
  std::mt19937_64 gen(seed);
  auto fill = [&](int off, int fanIn, int fanOut, int count) {
    const double a = std::sqrt(6.0 / (fanIn + fanOut)); // Glorot uniform
    std::uniform_real_distribution<double> u(-a, a);
    for (int i = 0; i < count; i++) w[off + i] = (float)u(gen);
  };
  fill(0, ni, nh, nh * ni);                            // W1
  fill(nh * ni + nh, nh, nh, nh * nh);                 // W2
  fill(nh * ni + nh + nh * nh + nh, nh, 1, nh);        // w3
  return mlp_load(s, w);
}

int kfvm_mlp_set_weights(kfvm_solver *s, const uint16_t *bf16, int64_t n) {
  if (!s || !bf16) return fail(KFVM_ERR_ARG, "null argument");
  int rc = mlp_alloc(s);
  if (rc) return rc;
  if (n != s->mlp.nw) return fail(KFVM_ERR_ARG, "wrong number of learned-indicator weights");
  std::vector<float> w(n);
  for (int64_t i = 0; i < n; i++) w[i] = bf2f(bf16[i]);
  return mlp_load(s, w);
}

int kfvm_mlp_get_weights(kfvm_solver *s, uint16_t *bf16, int64_t n) {
  if (!s || !bf16) return fail(KFVM_ERR_ARG, "null argument");
  if (!s->mlp.ready) return fail(KFVM_ERR_STATE, "learned indicator has no weights");
  if (n != s->mlp.nw) return fail(KFVM_ERR_ARG, "wrong number of learned-indicator weights");
  CK(cudaMemcpyAsync(bf16, s->mlp.wb, n * sizeof(uint16_t), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return KFVM_OK;
}

int kfvm_mlp_reserve(kfvm_solver *s, int64_t capacity) {
  if (!s || capacity <= 0) return fail(KFVM_ERR_ARG, "bad capacity");
  int rc = mlp_alloc(s);
  if (rc) return rc;
  auto &M = s->mlp;
  cudaFree(M.feats);
  cudaFree(M.labels);
  cudaFree(M.cells);
  M.feats = nullptr;
  M.labels = nullptr;
  M.cells = nullptr;
  cudaError_t e;
  if (!M.count && (e = cudaMalloc((void **)&M.count, sizeof(unsigned long long))) != cudaSuccess)
    return set_err_cuda(e, "sample counter");
  if ((e = cudaMalloc((void **)&M.feats, (size_t)capacity * M.ni * sizeof(uint16_t))) != cudaSuccess ||
      (e = cudaMalloc((void **)&M.labels, (size_t)capacity)) != cudaSuccess ||
      (e = cudaMalloc((void **)&M.cells, (size_t)capacity * sizeof(int64_t))) != cudaSuccess) {
    M.cap = 0;
    return set_err_cuda(e, "sample buffer");
  }
  if (!M.flags) {
    M.selBytes = kfvm::mlp_select_temp_bytes(s->g.n);
    if ((e = cudaMalloc((void **)&M.flags, (size_t)s->g.n)) != cudaSuccess ||
        (e = cudaMalloc((void **)&M.sel, (size_t)s->g.n * sizeof(int64_t))) != cudaSuccess ||
        (e = cudaMalloc((void **)&M.nsel, sizeof(int64_t))) != cudaSuccess ||
        (e = cudaMalloc(&M.selTemp, M.selBytes > 0 ? M.selBytes : 16)) != cudaSuccess)
      return set_err_cuda(e, "sample selection scratch");
  }
  M.cap = capacity;
  M.nPos = 0;
  M.have = 0;
  CK(cudaMemsetAsync(M.count, 0, sizeof(unsigned long long), s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return KFVM_OK;
}

int kfvm_mlp_collect(kfvm_solver *s, double tau, double keep_frac, uint64_t seed, int64_t *n_samples,
                     int64_t *n_positive) {
  if (!s) return fail(KFVM_ERR_ARG, "null solver");
  if (!s->primed) return fail(KFVM_ERR_STATE, "collect before an initial condition was set");
  auto &M = s->mlp;
  if (!M.cap) return fail(KFVM_ERR_STATE, "kfvm_mlp_reserve first");
  const int b = s->iCur;
  s->tEval = s->time;
  if (int rc = fill_halo(s, b)) return rc;
  cudaError_t e;
  // labels, pairs, then the kept cells in cell order (a stable select)
  e = run(s, KFVM_KCLASS_OTHER, 3, [&] {
    return kfvm::launch_mlp_select(s->dim, s->eq, s->Ub[b], s->g, s->dS, tau, keep_frac, seed, M.tiles, M.flags,
                                   M.sel, M.nsel, M.selTemp, M.selBytes, s->stream);
  });
  if (e != cudaSuccess) return set_err_cuda(e, "collect");
  int64_t nsel = 0;
  CK(cudaMemcpyAsync(&nsel, M.nsel, sizeof(nsel), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  // appended after the samples of earlier calls, up to the capacity
  const int64_t take = std::min<int64_t>(nsel, M.cap - M.have);
  e = run(s, KFVM_KCLASS_OTHER, 1, [&] {
    return kfvm::launch_mlp_features(s->dim, s->g, M.tiles, M.sel, take, M.flags, M.feats + M.have * M.ni,
                                     M.labels + M.have, M.cells + M.have, s->stream);
  });
  if (e != cudaSuccess) return set_err_cuda(e, "collect features");
  M.have += take;
  const unsigned long long cnt = (unsigned long long)M.have;
  CK(cudaMemcpyAsync(M.count, &cnt, sizeof(cnt), cudaMemcpyHostToDevice, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  const int64_t have = M.have;
  std::vector<uint8_t> lab(have);
  if (have) CK(cudaMemcpy(lab.data(), M.labels, have, cudaMemcpyDeviceToHost));
  int64_t pos = 0;
  for (auto l : lab) pos += l;
  M.nPos = pos;
  if (n_samples) *n_samples = have;
  if (n_positive) *n_positive = pos;
  return KFVM_OK;
}

int kfvm_mlp_get_samples(kfvm_solver *s, int64_t first, int64_t count, uint16_t *feats, uint8_t *labels,
                         int64_t *cells) {
  if (!s || first < 0 || count < 0) return fail(KFVM_ERR_ARG, "bad argument");
  auto &M = s->mlp;
  unsigned long long cnt = 0;
  if (M.count) CK(cudaMemcpy(&cnt, M.count, sizeof(cnt), cudaMemcpyDeviceToHost));
  const int64_t have = std::min<int64_t>((int64_t)cnt, M.cap);
  if (first + count > have) return fail(KFVM_ERR_ARG, "sample range beyond the collected samples");
  if (feats && count)
    CK(cudaMemcpy(feats, M.feats + first * M.ni, (size_t)count * M.ni * sizeof(uint16_t), cudaMemcpyDeviceToHost));
  if (labels && count) CK(cudaMemcpy(labels, M.labels + first, (size_t)count, cudaMemcpyDeviceToHost));
  if (cells && count) CK(cudaMemcpy(cells, M.cells + first, (size_t)count * sizeof(int64_t), cudaMemcpyDeviceToHost));
  return KFVM_OK;
}

int kfvm_mlp_train(kfvm_solver *s, int32_t steps, int32_t batch, double lr, double pos_weight, uint64_t seed,
                   double *loss_first, double *loss_last) {
  if (!s || steps <= 0 || batch <= 0 || !(lr > 0.0) || !(pos_weight > 0.0)) return fail(KFVM_ERR_ARG, "bad argument");
  auto &M = s->mlp;
  if (!M.ready) return fail(KFVM_ERR_STATE, "kfvm_mlp_init_weights or kfvm_mlp_set_weights first");
  unsigned long long cnt = 0;
  if (M.count) CK(cudaMemcpy(&cnt, M.count, sizeof(cnt), cudaMemcpyDeviceToHost));
  const int64_t n = std::min<int64_t>((int64_t)cnt, M.cap);
  if (n <= 0) return fail(KFVM_ERR_STATE, "no collected samples (kfvm_mlp_collect)");
  const int blocks = kfvm::mlp_train_blocks(batch);
  if (M.gpartBlocks < blocks) {
    cudaFree(M.gpart);
    cudaFree(M.lpart);
    M.gpart = M.lpart = nullptr;
    M.gpartBlocks = 0;
    cudaError_t ea;
    if ((ea = cudaMalloc((void **)&M.gpart, (size_t)blocks * M.nw * sizeof(float))) != cudaSuccess ||
        (ea = cudaMalloc((void **)&M.lpart, (size_t)blocks * sizeof(float))) != cudaSuccess)
      return set_err_cuda(ea, "training scratch");
    M.gpartBlocks = blocks;
  }
  // loss slots: [0] mean over the first 20 steps, [1] over the last 20, [2] the rest
  CK(cudaMemsetAsync(M.loss, 0, 4 * sizeof(float), s->stream));
  const int win = std::min(20, steps);
  for (int i = 0; i < steps; i++) {
    float *slot = i < win ? M.loss : (i >= steps - win ? M.loss + 1 : M.loss + 2);
    M.t++;
    cudaError_t e = run(s, KFVM_KCLASS_OTHER, 2, [&] {
      return kfvm::launch_mlp_train_step(s->dim, M.feats, M.labels, n, batch, M.master, M.m, M.v, M.gpart, M.lpart,
                                         M.wq, M.wb, slot, (float)pos_weight, (float)lr, M.t,
                                         seed ^ (uint64_t)M.t, s->stream);
    });
    if (e != cudaSuccess) return set_err_cuda(e, "train");
  }
  cudaError_t ep = kfvm::launch_mlp_pack(s->dim, M.wb, M.wq, M.img, s->stream);
  if (ep != cudaSuccess) return set_err_cuda(ep, "pack");
  float l[4];
  CK(cudaMemcpyAsync(l, M.loss, sizeof(l), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  harvest(s);
  if (loss_first) *loss_first = l[0] / win;
  if (loss_last) *loss_last = (steps > win ? l[1] : l[0]) / win;
  return KFVM_OK;
}

int kfvm_mlp_config(kfvm_solver *s, double prob_threshold, double judge_frac, double tau, double miss_limit) {
  if (!s || !(prob_threshold > 0.0 && prob_threshold < 1.0) || !(judge_frac >= 0.0 && judge_frac <= 1.0) ||
      !(tau >= 0.0) || !(miss_limit >= 0.0))
    return fail(KFVM_ERR_ARG, "bad learned-indicator parameter");
  s->mlp.logitThr = std::log(prob_threshold / (1.0 - prob_threshold));
  s->mlp.judgeFrac = judge_frac;
  s->mlp.tau = tau;
  s->mlp.missLimit = miss_limit;
  return KFVM_OK;
}

int kfvm_mlp_probability(kfvm_solver *s, float *out_host) {
  if (!s || !out_host) return fail(KFVM_ERR_ARG, "null argument");
  if (!s->mlp.ready) return fail(KFVM_ERR_STATE, "learned indicator has no weights");
  if (!s->primed) return fail(KFVM_ERR_STATE, "no state");
  float *d = nullptr;
  cudaError_t e;
  if ((e = cudaMalloc((void **)&d, s->g.n * sizeof(float))) != cudaSuccess) return set_err_cuda(e, "alloc");
  const int b = s->iCur;
  s->tEval = s->time;
  if (int rc = fill_halo(s, b)) {
    cudaFree(d);
    return rc;
  }
  e = kfvm::launch_mlp_prob(s->dim, s->eq, s->Ub[b], s->g, s->mlp.tiles, s->mlp.img, d, s->sc,
                              s->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out_host, d, s->g.n * sizeof(float), cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  cudaFree(d);
  if (e != cudaSuccess) return set_err_cuda(e, "probability");
  CK(cudaMemcpy(s->hsc, s->sc, sizeof(kfvm::DevScalars), cudaMemcpyDeviceToHost));
  if (s->hsc->fault) return fail(KFVM_ERR_CUDA, kFaultMsg);
  return KFVM_OK;
}

int kfvm_mlp_stats(kfvm_solver *s, int64_t *out6) {
  if (!s || !out6) return fail(KFVM_ERR_ARG, "null argument");
  CK(cudaMemcpyAsync(s->hsc, s->sc, sizeof(kfvm::DevScalars), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  out6[0] = (int64_t)s->hsc->mlp_judged;
  out6[1] = (int64_t)s->hsc->mlp_pos;
  out6[2] = (int64_t)s->hsc->mlp_missed;
  out6[3] = (int64_t)s->hsc->mlp_false;
  out6[4] = s->mlp.fallbackEvents;
  out6[5] = s->mlp.fallbackSteps;
  return KFVM_OK;
}

int kfvm_selftest_wait(double limit_s, int32_t *gave_up, double *waited_s) {
  if (!(limit_s > 0.0 && limit_s <= 1.0) || !gave_up || !waited_s) return fail(KFVM_ERR_ARG, "bad argument");
  unsigned long long *d = nullptr, h[2] = {0, 0};
  cudaError_t e = cudaMalloc((void **)&d, sizeof(h));
  if (e == cudaSuccess) e = kfvm::launch_wait_probe((uint64_t)(limit_s * 1e9), d, 0);
  if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return set_err_cuda(e, "wait probe");
  *gave_up = (int32_t)h[0];
  *waited_s = (double)h[1] * 1e-9;
  return KFVM_OK;
}

int kfvm_selftest_rcp(int64_t n, uint64_t seed, int64_t *max_ulp, double *max_rel_quot) {
  if (n <= 0 || n > ((int64_t)1 << 32) || !max_ulp || !max_rel_quot) return fail(KFVM_ERR_ARG, "bad argument");
  unsigned long long *d = nullptr, h[2] = {0, 0};
  cudaError_t e = cudaMalloc((void **)&d, sizeof(h));
  if (e == cudaSuccess) e = cudaMemset(d, 0, sizeof(h));
  if (e == cudaSuccess) e = kfvm::launch_rcp_probe(n, seed, d, 0);
  if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return set_err_cuda(e, "reciprocal probe");
  *max_ulp = (int64_t)h[0];
  double q;
  std::memcpy(&q, &h[1], sizeof(q));
  *max_rel_quot = q;
  return KFVM_OK;
}

int kfvm_get_faces(kfvm_solver *s, int32_t dir, double *out) {
  if (!s || !out || dir < 0 || dir >= s->dim) return fail(KFVM_ERR_ARG, "bad argument");
  const kfvm::Grid &g = s->g;
  const int nqf = s->dim == 2 ? s->g.nq : s->g.nq * s->g.nq, nv = s->nv;
  const int64_t nf = g.nface[dir];
  CK(cudaMemcpyAsync(out, s->F[dir], (size_t)2 * nqf * nv * nf * sizeof(double), cudaMemcpyDeviceToHost,
                     s->stream));
  CK(cudaStreamSynchronize(s->stream));
  // apply the face BCs to the boundary slots (setFaceBCs), as the kernels do on read
  const int64_t fx = g.fdim[dir][0], fy = g.fdim[dir][1], fz = g.fdim[dir][2];
  const int64_t nd = dir == 0 ? g.nx : (dir == 1 ? g.ny : g.nz);
  const int64_t stride = dir == 0 ? 1 : (dir == 1 ? fx : fx * fy);
  const bool per = g.bc[2 * dir] == KFVM_BC_PERIODIC;
  // an exchange or user face's outer slot already holds its outer states
  const bool xlo = kfvm::outer_in_face(g.bc[2 * dir]), xhi = kfvm::outer_in_face(g.bc[2 * dir + 1]);
  const unsigned flo = g.bflip[2 * dir], fhi = g.bflip[2 * dir + 1];
  for (int64_t k = 0; k < fz; k++)
    for (int64_t j = 0; j < fy; j++)
      for (int64_t i = 0; i < fx; i++) {
        const int64_t m = dir == 0 ? i : (dir == 1 ? j : k);
        if (m != 0) continue;
        const int64_t lo = (k * fy + j) * fx + i, hi = lo + nd * stride;
        for (int q = 0; q < nqf; q++)
          for (int v = 0; v < nv; v++) {
            const int64_t s0 = ((int64_t)(0 * nqf + q) * nv + v) * nf, s1 = ((int64_t)(1 * nqf + q) * nv + v) * nf;
            if (per) {
              out[s0 + lo] = out[s0 + hi];
              out[s1 + hi] = out[s1 + lo];
            } else {
              if (!xlo) out[s0 + lo] = (flo >> v) & 1u ? -out[s1 + lo] : out[s1 + lo];
              if (!xhi) out[s1 + hi] = (fhi >> v) & 1u ? -out[s0 + hi] : out[s0 + hi];
            }
          }
      }
  return KFVM_OK;
}

int kfvm_block_config(const kfvm_config *blocks, int32_t rank, kfvm_config *out, int32_t neighbors[6]) {
  if (!blocks || !out) return fail(KFVM_ERR_ARG, "null argument");
  const int dim = blocks->dim;
  if (dim != 2 && dim != 3) return fail(KFVM_ERR_ARG, "dim must be 2 or 3");
  int nb[3];
  for (int d = 0; d < 3; d++) {
    nb[d] = d < dim ? kfvm::cfg_nb(blocks, d) : 1;
    if (d >= dim && blocks->nb[d] > 1) return fail(KFVM_ERR_ARG, "blocks along z in a 2D domain");
  }
  const int64_t nranks = (int64_t)nb[0] * nb[1] * nb[2];
  if (rank < 0 || rank >= nranks) return fail(KFVM_ERR_ARG, "rank outside the block count");
  for (int f = 0; f < 2 * dim; f++)
    if (blocks->bc[f] == KFVM_BC_EXCHANGE) return fail(KFVM_ERR_ARG, "the domain's own faces cannot be exchange faces");
  kfvm_config c = *blocks;
  // MPI_Cart_create's row-major order: the last axis varies fastest
  int b[3];
  b[2] = rank % nb[2];
  b[1] = (rank / nb[2]) % nb[1];
  b[0] = rank / (nb[2] * nb[1]);
  int32_t nbr[6];
  for (int d = 0; d < 3; d++) {
    c.nb[d] = nb[d];
    c.block[d] = b[d];
    for (int side = 0; side < 2; side++) {
      const int f = 2 * d + side;
      nbr[f] = -1;
      if (d >= dim || nb[d] == 1) continue;
      const bool per = blocks->bc[f] == KFVM_BC_PERIODIC;
      int nbd = b[d] + (side == 0 ? -1 : 1);
      if (nbd < 0 || nbd >= nb[d]) {
        if (!per) continue;  // a physical face of the domain
        nbd = (nbd + nb[d]) % nb[d];
      }
      int q[3] = {b[0], b[1], b[2]};
      q[d] = nbd;
      nbr[f] = (q[0] * nb[1] + q[1]) * nb[2] + q[2];
      c.bc[f] = KFVM_BC_EXCHANGE;
    }
  }
  *out = c;
  if (neighbors)
    for (int f = 0; f < 6; f++) neighbors[f] = nbr[f];
  return KFVM_OK;
}

// the four buffers of the exchange and user-boundary callbacks, one size for every
// use: the largest cell slab or face plane (with the indicator) over the axes
int alloc_xbuf(kfvm_solver *s) {
  const int nqf = s->dim == 2 ? s->g.nq : s->g.nq * s->g.nq;
  int64_t bytes = 0;
  for (int d = 0; d < s->dim; d++) {
    bytes = std::max(bytes, kfvm::cell_slab_values(s->g, s->dim, s->nv, d) * (int64_t)sizeof(double));
    bytes = std::max(bytes, kfvm::face_plane_bytes(s->g, nqf, s->nv, d, true));
  }
  if (!s->xbuf[0]) {
    for (int i = 0; i < 4; i++) {
      cudaError_t e = cudaMalloc((void **)&s->xbuf[i], (size_t)bytes);
      if (e != cudaSuccess) {
        for (int k = 0; k <= i; k++) {
          cudaFree(s->xbuf[k]);
          s->xbuf[k] = nullptr;
        }
        return set_err_cuda(e, "alloc exchange buffers");
      }
    }
  }
  return KFVM_OK;
}

int kfvm_set_exchange(kfvm_solver *s, kfvm_exchange_fn ex, kfvm_allreduce_fn ar, void *user) {
  if (!s) return fail(KFVM_ERR_ARG, "null solver");
  if (!s->decomposed) return fail(KFVM_ERR_STATE, "no exchange faces in this solver's configuration");
  if (!ex || !ar) return fail(KFVM_ERR_ARG, "both callbacks are required");
  if (int rc = alloc_xbuf(s)) return rc;
  s->xfn = ex;
  s->rfn = ar;
  s->xuser = user;
  return KFVM_OK;
}

int kfvm_set_user_bc(kfvm_solver *s, kfvm_user_bc_fn fn, void *user) {
  if (!s) return fail(KFVM_ERR_ARG, "null solver");
  if (!s->hasUser) return fail(KFVM_ERR_STATE, "no user boundary faces in this solver's configuration");
  if (!fn) return fail(KFVM_ERR_ARG, "null callback");
  if (int rc = alloc_xbuf(s)) return rc;
  s->ufn = fn;
  s->uuser = user;
  return KFVM_OK;
}

int kfvm_get_flags(kfvm_solver *s, uint8_t *weno_applied, double *theta) {
  if (!s) return fail(KFVM_ERR_ARG, "null solver");
  if (weno_applied) CK(cudaMemcpyAsync(weno_applied, s->applied, s->g.n, cudaMemcpyDeviceToHost, s->stream));
  if (theta) CK(cudaMemcpyAsync(theta, s->theta, s->g.n * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return KFVM_OK;
}

int kfvm_set_plot_freq(kfvm_solver *s, double plot_freq, int32_t plot_num) {
  if (!s || !(plot_freq >= 0.0) || plot_num < 0) return fail(KFVM_ERR_ARG, "bad argument");
  s->plotFreq = plot_freq;
  s->plotNum = plot_num;
  return KFVM_OK;
}

int kfvm_write_plotfile(kfvm_solver *s, const char *dir, const char *base, int32_t num, int32_t ckpt,
                        int32_t time_step) {
  if (!s || !dir || !base) return fail(KFVM_ERR_ARG, "null argument");
  const int64_t n = s->g.n;
  std::vector<double> u((size_t)n * s->nv), th((size_t)n);
  std::vector<uint8_t> w((size_t)n);
  int rc = kfvm_get_state(s, u.data());
  if (rc) return rc;
  if ((rc = kfvm_get_flags(s, w.data(), th.data()))) return rc;
  return kfvm_plotfile_write(&s->cfg, dir, base, num, ckpt, time_step, s->time, s->dt, u.data(), w.data(),
                             th.data());
}

int kfvm_restart(kfvm_solver *s, const char *xmf_path, int32_t *time_step) {
  if (!s || !xmf_path || !time_step) return fail(KFVM_ERR_ARG, "null argument");
  const int64_t n = s->g.n;
  std::vector<double> u((size_t)n * s->nv), th((size_t)n);
  std::vector<uint8_t> w((size_t)n);
  double t = 0.0, h = 0.0;
  int32_t ts = 0;
  int rc = kfvm_plotfile_read(&s->cfg, xmf_path, u.data(), w.data(), th.data(), &ts, &t, &h);
  if (rc) return rc;
  if (!(h > 0.0)) return fail(KFVM_ERR_IO, "kfvm_restart: the file holds no time step size (a plot file?)");
  // state and both components of the WENO flag view, then the FSAL priming
  // evaluation; time, time step and step size come from the file (Solver.cpp:60-80)
  if ((rc = upload_state(s, s->iPrev, u.data()))) return rc;
  if ((rc = prime(s))) return rc;
  CK(cudaMemcpyAsync(s->theta, th.data(), n * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemcpyAsync(s->wset, w.data(), n, cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemcpyAsync(s->applied, w.data(), n, cudaMemcpyHostToDevice, s->stream));
  // the priming evaluation again, now with the restored flags, at the file's time
  CK(cudaMemsetAsync(&s->sc->maxvel_bits, 0, sizeof(unsigned long long), s->stream));
  s->tEval = t;
  if ((rc = eval_into_K(s, s->iPrev))) return rc;
  CK(cudaStreamSynchronize(s->stream));
  s->time = t;
  s->dt = h;
  s->nTS = ts + 1;
  *time_step = ts;
  return KFVM_OK;
}

int kfvm_flow_stats(kfvm_solver *s, double *stats, int32_t *n_stats) {
  using namespace kfvm;
  if (!s || !stats) return fail(KFVM_ERR_ARG, "null argument");
  if (!s->primed) return fail(KFVM_ERR_STATE, "no state yet (kfvm_init_ic / kfvm_set_state / kfvm_restart)");
  const kfvm_config &c = s->cfg;
  const double volume = s->dim == 2 ? (c.xup - c.xlo) * (c.yup - c.ylo)
                                    : (c.xup - c.xlo) * (c.yup - c.ylo) * (c.zup - c.zlo);
  const double dvol = s->dim == 2 ? s->g.dx * s->g.dy : s->g.dx * s->g.dy * s->g.dz;
  double *U = s->Ub[s->iCur];
  // the halo as the boundary conditions set it (the reference relies on the last
  // evaluation having set it; filling again gives the same values)
  s->tEval = s->time;
  if (int rc = fill_halo(s, s->iCur)) return rc;
  CK(launch_stats(s->dim, s->eq, U, s->g, dvol / volume, s->spart, s->ssum, s->stream));
  s->launches += s->eq == KFVM_EQ_SRHYDRO ? 1 : 3;
  double h[3];
  CK(cudaMemcpyAsync(h, s->ssum, sizeof(h), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  const int n = stats_count(s->eq);
  for (int q = 0; q < n; q++) stats[q] = h[q];
  if (n_stats) *n_stats = n;
  return KFVM_OK;
}

int kfvm_forcing_num_modes(int32_t dim) {
  const int n = kfvm::forcing_num_modes(dim);
  return n < 0 ? fail(KFVM_ERR_ARG, "dim must be 2 or 3") : n;
}

int kfvm_forcing_draw(int32_t dim, uint32_t seed32, double *modes) {
  if (!modes) return fail(KFVM_ERR_ARG, "null argument");
  if (dim != 2 && dim != 3) return fail(KFVM_ERR_ARG, "dim must be 2 or 3");
  kfvm::forcing_draw(dim, seed32, modes);
  return KFVM_OK;
}

int kfvm_set_forcing(kfvm_solver *s, const kfvm_forcing *f) {
  if (!s) return fail(KFVM_ERR_ARG, "null solver");
  if (!f) {
    s->forcing = false;
    return KFVM_OK;
  }
  if (s->eq == KFVM_EQ_SRHYDRO) return fail(KFVM_ERR_ARG, "random forcing acts on Newtonian momenta (Hydro, NS, GLM-MHD)");
  if (!(f->edot >= 0.0) || !std::isfinite(f->ratio)) return fail(KFVM_ERR_ARG, "forcing: edot >= 0 and a finite ratio");
  if (!s->fmodes) {
    CK(cudaMalloc((void **)&s->fmodes, KFVM_FORCING_MAX_MODES * 3 * 3 * sizeof(double)));
    CK(cudaMalloc((void **)&s->fsums, 2 * sizeof(double)));
  }
  s->fpar = *f;
  s->fdraws = 0;
  s->forcing = true;
  return KFVM_OK;
}

int kfvm_apply_forcing(kfvm_solver *s, const double *modes_in, double *modes_out, double *force_str) {
  using namespace kfvm;
  if (!s) return fail(KFVM_ERR_ARG, "null solver");
  if (!s->forcing || !s->fmodes) return fail(KFVM_ERR_STATE, "forcing not enabled (kfvm_set_forcing)");
  if (!s->primed) return fail(KFVM_ERR_STATE, "no state yet (kfvm_init_ic / kfvm_set_state / kfvm_restart)");
  const int nm = forcing_num_modes(s->dim);
  std::vector<double> m((size_t)nm * s->dim * 3);
  if (modes_in) {
    std::copy(modes_in, modes_in + m.size(), m.begin());
  } else {
    // a fresh generator per draw, as updateForcing makes one per call; its seed from
    // the solver's seed and the draw count (SplitMix64 finaliser)
    uint64_t x = s->fpar.seed + 0x9E3779B97F4A7C15ull * (++s->fdraws);
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    x ^= x >> 31;
    forcing_draw(s->dim, (uint32_t)(x >> 32), m.data());
  }
  const double lo[3] = {cfg_lo(&s->cfg, 0), cfg_lo(&s->cfg, 1), cfg_lo(&s->cfg, 2)};
  double *U = s->Ub[s->iCur];
  CK(cudaMemcpyAsync(s->fmodes, m.data(), m.size() * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  CK(launch_forcing_integrate(s->dim, U, s->g, s->fmodes, nm, s->fpar.ratio, lo, s->part, s->fsums, s->stream));
  s->launches += 2;
  double ab[2];
  CK(cudaMemcpyAsync(ab, s->fsums, sizeof(ab), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  // Solver::forceStrComm (Solver.cpp:395-409): the integrals summed over all ranks,
  // then the root of A s^2 + B s + C = 0 with C = -edot dt / dvol
  if (int rc = reduce_all(s, KFVM_REDUCE_SUM, ab, 2)) return rc;
  const double dvol = s->dim == 2 ? s->g.dx * s->g.dy : s->g.dx * s->g.dy * s->g.dz;
  const double A = ab[0], B = ab[1], C = -s->fpar.edot * s->dt / dvol;
  const double str = (-B + std::sqrt(std::fmax(0.0, B * B - 4.0 * A * C))) / (2.0 * A);
  CK(launch_forcing_apply(s->dim, U, s->g, s->fmodes, nm, s->fpar.ratio, str, lo, s->stream));
  s->launches += 1;
  CK(cudaStreamSynchronize(s->stream));
  if (modes_out) std::copy(m.begin(), m.end(), modes_out);
  if (force_str) *force_str = str;
  return KFVM_OK;
}

int kfvm_last_stage_ms(kfvm_solver *s, double *ms) {
  if (!s || !ms) return fail(KFVM_ERR_ARG, "null argument");
  *ms = s->lastMs;
  return KFVM_OK;
}

int kfvm_get_stream(kfvm_solver *s, void **stream) {
  if (!s || !stream) return fail(KFVM_ERR_ARG, "null argument");
  *stream = (void *)s->stream;
  return KFVM_OK;
}

int kfvm_set_timing(kfvm_solver *s, int32_t on) {
  if (!s) return fail(KFVM_ERR_ARG, "null solver");
  CK(cudaStreamSynchronize(s->stream));
  harvest(s);
  s->timing = on != 0;
  for (int c = 0; c < KFVM_NUM_KCLASS; c++) {
    s->clsMs[c] = 0.0;
    s->clsLaunches[c] = 0;
  }
  return KFVM_OK;
}

int kfvm_get_timing(kfvm_solver *s, double *ms, int64_t *launches) {
  if (!s) return fail(KFVM_ERR_ARG, "null solver");
  CK(cudaStreamSynchronize(s->stream));
  harvest(s);
  for (int c = 0; c < KFVM_NUM_KCLASS; c++) {
    if (ms) ms[c] = s->clsMs[c];
    if (launches) launches[c] = s->clsLaunches[c];
  }
  return KFVM_OK;
}

int kfvm_get_launch_count(kfvm_solver *s, int64_t *launches) {
  if (!s || !launches) return fail(KFVM_ERR_ARG, "null argument");
  *launches = s->launches;
  return KFVM_OK;
}

int kfvm_measure_fp64_mma(double *tflops) {
  if (!tflops) return fail(KFVM_ERR_ARG, "null argument");
  int dev = 0, sms = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  double *out = nullptr;
  cudaEvent_t a = nullptr, b = nullptr;
  cudaStream_t st = nullptr;
  CK(cudaMalloc((void **)&out, sizeof(double)));
  CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  const int blocks = 4 * sms, iters = 1 << 15;   // 16 warps per SM
  cudaError_t e = kfvm::launch_dmma_peak(blocks, 64, out, st);   // warm-up
  float ms = 0.0f;
  if (e == cudaSuccess) e = cudaEventRecord(a, st);
  if (e == cudaSuccess) e = kfvm::launch_dmma_peak(blocks, iters, out, st);
  if (e == cudaSuccess) e = cudaEventRecord(b, st);
  if (e == cudaSuccess) e = cudaEventSynchronize(b);
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaStreamDestroy(st);
  cudaFree(out);
  if (e != cudaSuccess) return set_err_cuda(e, "FP64 MMA probe");
  const double flops = (double)blocks * 4 * (double)iters * 8 * 512.0;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return KFVM_OK;
}

int kfvm_get_same_state(kfvm_solver *s, int32_t *on, int64_t *sampled, int64_t *equal) {
  if (!s) return fail(KFVM_ERR_ARG, "null solver");
  if (on) *on = s->sameOn ? 1 : 0;
  if (sampled) *sampled = (int64_t)s->sampSeen;
  if (equal) *equal = (int64_t)s->sameSeen;
  return KFVM_OK;
}

} // extern "C"
