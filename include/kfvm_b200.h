/*
 * kfvm_b200.h -- C ABI of the B200-native per-stage hot path of the KFVM
 * finite-volume solver (kernel-based WENO-AO reconstruction, HLLC/HLL Riemann
 * fluxes, flux divergence, low-storage SSP-RK stage update with the CFL
 * max-reduction), for one rank on one GPU.
 *
 * The reference has no FFI: its operator boundary is the C++ Solver class and
 * the Stencil weight object.  Each entry point below names the reference member
 * function it replaces (path within the reference project, file:line).  All
 * entry points take plain pointers and sizes, return 0 on success and a
 * negative KFVM_ERR_* code on failure, never abort, and never throw.
 *
 * State exchange format ("SoA interior"): double[NV][nz][ny][nx], x fastest,
 * interior cells only (no halo).  nz == 1 in 2D.  The conserved-variable order
 * is the reference's (src/physics/SimVar.H:12-66):
 *   Euler / Navier-Stokes / SRHydro: dens, momx, momy, momz, etot  (NV = 5;
 *                          SRHydro: D, Sx, Sy, Sz, E)
 *   GLM-MHD:               dens, momx, momy, momz, etot,
 *                          magx, magy, magz, psi                    (NV = 9)
 */
#ifndef KFVM_B200_H_
#define KFVM_B200_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- enumerations (values match the reference's enums) ------------------ */

/* src/physics/EquationTypes.H:8-16 */
/* KFVM_EQ_SRHYDRO: special-relativistic hydrodynamics (src/physics/srhydro):
 * conserved D = rho W, S = rho h W^2 v, E = rho h W^2 - p; the primitives are
 * recovered by Newton iteration on the pressure; HLL or LLF fluxes only */
enum kfvm_eq { KFVM_EQ_HYDRO = 0, KFVM_EQ_NAVIERSTOKES = 1, KFVM_EQ_MHD_GLM = 2, KFVM_EQ_SRHYDRO = 3 };
/* src/physics/RSTypes.H:6 */
enum kfvm_rs { KFVM_RS_LLF = 0, KFVM_RS_HLL = 1, KFVM_RS_HLLC = 2 };
/* src/numeric/RKTypes.H:6 (SSP4_3_2 is the only third-order SSP method there) */
enum kfvm_rk {
  KFVM_RK_THREESTARP = 0,
  KFVM_RK_FOURSTARP = 1,
  KFVM_RK_SSP4_3_2 = 2,
  KFVM_RK_SSP10_4_3 = 3
};
/* src/Types.H:37 */
/* BCType (src/Types.H:40) without "user": a reflecting wall mirrors the state
 * and negates the normal momentum (and the normal magnetic field for GLM-MHD); a
 * no-slip wall negates every momentum component (and the normal magnetic field),
 * with the coefficient tables of src/physics/<eq>/<Eq>_BCCoeffs.H. */
enum kfvm_bc {
  /* the values of the reference's BCType (src/Types.H:40), user included */
  KFVM_BC_PERIODIC = 0, KFVM_BC_OUTFLOW = 1, KFVM_BC_REFLECTING = 2, KFVM_BC_NOSLIP = 3,
  /* a face whose halo cells and outer face states a user function supplies
   * (BCType::user: the CellWest..CellTop and FaceWest..FaceTop functions of a
   * problem's UserBCs.H, src/BoundaryConditions_K.H:96-128, 569-615), through
   * the callback of kfvm_set_user_bc */
  KFVM_BC_USER = 4,
  /* a block face shared with another rank of a decomposed domain (the faces the
   * reference's LayoutMPI gives an MPI neighbour, src/LayoutMPI.H:44-97): its
   * halo cells and outer face states come from that rank through the exchange
   * callbacks of kfvm_set_exchange */
  KFVM_BC_EXCHANGE = 5
};
/* src/Types.H:40 */
enum kfvm_ts_status { KFVM_TS_ACCEPTED = 0, KFVM_TS_TOLERANCE = 1, KFVM_TS_UNPHYSICAL = 2 };
/* Troubled-cell indicator choice.  KXRCF is the reference's selector
 * (src/numeric/Numeric_K.H:292-398); ALL forces full WENO on every cell
 * (the reference's wenothresh < 0 path); NONE never flags (linear only). */
enum kfvm_indicator { KFVM_IND_KXRCF = 0, KFVM_IND_ALL = 1, KFVM_IND_NONE = 2, KFVM_IND_MLP = 3 };
/* arithmetic of the linear reconstruction contraction */
enum kfvm_precision { KFVM_PREC_FP64 = 0, KFVM_PREC_TF32X3 = 1 };
/* Initial conditions built into the library (cell averages by Q^d Gauss
 * quadrature, src/numeric/Numeric_K.H:31-107). */
enum kfvm_ic {
  KFVM_IC_ISENTROPIC_VORTEX = 0, /* 2D Euler, rho=u=v=p=1 + Shu vortex beta=5   */
  KFVM_IC_SPHERICAL_SOD = 1,     /* 3D Euler, rho,p = 1,1 in r<0.2 else .125,.1 */
  KFVM_IC_KELVIN_HELMHOLTZ = 2,  /* 2D Euler shear layer + seeded noise         */
  KFVM_IC_TAYLOR_GREEN = 3,      /* 3D Navier-Stokes Taylor-Green vortex        */
  KFVM_IC_ORSZAG_TANG = 4,       /* 2D GLM-MHD Orszag-Tang vortex               */
  KFVM_IC_SMOOTH_WAVE = 5,       /* any dim/eq: smooth density/velocity wave     */
  KFVM_IC_SR_SHOCK_TUBE = 6,     /* SR hydro: rho,p = 10,40/3 for |x|<1/2 else 1,1e-6
                                    (exec/SRHydro/SRShockTube)                    */
  KFVM_IC_SR_RIEMANN_2D = 7,     /* SR hydro 2D four-quadrant Riemann problem
                                    (exec/SRHydro/SRRiem2d)                       */
  KFVM_IC_STIR_TURB = 8          /* gas at rest, rho = 1, p = 1/gamma (GLM-MHD:
                                    plus bx = sqrt(2p/beta), user:beta 0.1), for
                                    random forcing (exec/{Hydro,NavierStokes,MHD}/StirTurb) */
};

/* ---- error codes -------------------------------------------------------- */
#define KFVM_OK 0
#define KFVM_ERR_ARG (-1)      /* bad argument / unsupported configuration   */
#define KFVM_ERR_CUDA (-2)     /* a CUDA runtime call failed                 */
#define KFVM_ERR_LAPACK (-3)   /* dgetrf/dgetrs reported a singular system   */
#define KFVM_ERR_NOMEM (-4)    /* device or host allocation failed           */
#define KFVM_ERR_STATE (-5)    /* call out of order (e.g. step before IC)    */
#define KFVM_ERR_IO (-6)       /* a plot / checkpoint file cannot be written or read */

/* ---- sizes -------------------------------------------------------------- */
#define KFVM_RAD 2          /* stencil radius (STENCIL_RADIUS)                 */
#define KFVM_MAX_CELLS 33   /* nCellsFull for r=2 in 3D (StencilInfo.H:69-84)  */
#define KFVM_MAX_SUB 8      /* nSub in 3D                                      */
#define KFVM_MAX_BIAS 6     /* nBias in 3D                                     */
#define KFVM_MAX_BCELLS 11  /* nCellsBias in 3D                                */
#define KFVM_MAX_INDIC 19   /* nIndic in 3D                                    */
#define KFVM_MAX_NQ 3       /* NUM_QUAD_PTS supported by the weight precompute */
#define KFVM_MAX_FACEQ 9    /* NQ^(d-1)                                        */
#define KFVM_MAX_CELLQ 27   /* NQ^d                                            */

/* Run configuration: the union of the reference's compile-time Definitions.H
 * choices and its run-time .init settings (src/ProblemSetup.H:26-82,
 * src/ParameterStructs.H:21-40).  Reals read from an .init file must already be
 * rounded through float, as std::stof does in the reference. */
typedef struct kfvm_config {
  int32_t dim;        /* SPACE_DIM: 2 or 3                                   */
  int32_t eq;         /* enum kfvm_eq                                        */
  int32_t rs;         /* enum kfvm_rs                                        */
  int32_t rk;         /* enum kfvm_rk                                        */
  int32_t nq;         /* NUM_QUAD_PTS: 2, or 3 (not for SRHydro in 3D)      */
  int32_t indicator;  /* enum kfvm_indicator                                 */
  int64_t nx, ny, nz; /* interior cells (nz = 1 in 2D)                       */
  double xlo, xup, ylo, yup, zlo, zup;
  int32_t bc[6];      /* enum kfvm_bc for west,east,south,north,bottom,top   */
  double gamma, reynolds, prandtl;
  double weno_thresh; /* eos:wenothresh; < 0 forces full WENO everywhere     */
  double lfac;        /* stencil:lfac (SE kernel length scale in cells)      */
  double cfl, atol, rtol, rejection_thresh, min_dt, final_time;
  int32_t rejection_limit;
  int32_t max_steps;  /* time:maxsteps (the stepping loop starts at nTS=1)   */
  int32_t have_sources; /* forced on for MHD_GLM (ProblemSetup.H:81)        */
  /* Domain decomposition (mesh:numblocks, src/ProblemSetup.H:224-233): nb[d]
   * blocks per axis, this rank's block at block[d].  nx, ny, nz are then the
   * cells of one block and xlo..zup the extents of the whole domain; as in the
   * reference's Geometry (src/Geometry.H:28-31) dx = (xup - xlo) / (nx nb[0])
   * and this block starts at xlo + dx (block[0] nx).  nb = {1, 1, 1}, block =
   * {0, 0, 0} for one domain. */
  int32_t nb[3];
  int32_t block[3];
  int32_t pad_;
} kfvm_config;

/* Precomputed stencil (the reference's Stencil object, src/stencil/Stencil.H:54-146).
 * Array shapes follow the reference's views with fixed maximum extents:
 *   off[3][C]                      lOff, tOff, ttOff
 *   sub_idx[nBias][nCellsBias]      subIdx
 *   face_w[nSub][2d][NQF][C]        faceWeights (zero-padded past each substencil)
 *   cell_w[nSub][NQ^d][C]           cellWeights, point index = ((qx*NQ)+qy)*NQz+qz
 *   deriv_w[nSub][nIndic][C]        derivWeights (already scaled by dx^px dy^py dz^pz) */
typedef struct kfvm_stencil {
  int32_t dim, nq;
  int32_t n_cells, n_cells_ctr, n_cells_bias, n_sub, n_bias, n_indic, nqf, nqc;
  int64_t off[3][KFVM_MAX_CELLS];
  int64_t sub_idx[KFVM_MAX_BIAS][KFVM_MAX_BCELLS];
  double face_w[KFVM_MAX_SUB][6][KFVM_MAX_FACEQ][KFVM_MAX_CELLS];
  double cell_w[KFVM_MAX_SUB][KFVM_MAX_CELLQ][KFVM_MAX_CELLS];
  double deriv_w[KFVM_MAX_SUB][KFVM_MAX_INDIC][KFVM_MAX_CELLS];
} kfvm_stencil;

/* Outcome of one TakeStep (src/Solver.cpp:188-343). */
typedef struct kfvm_step_info {
  double time;       /* simulation time after the step                     */
  double dt;         /* next time step size                                */
  double dt_taken;   /* size of the accepted step (0 if none was accepted) */
  double max_vel;    /* max wave speed seen in the accepted attempt        */
  double err_est;    /* errNew of the accepted attempt                     */
  int32_t status;    /* enum kfvm_ts_status of the last attempt            */
  int32_t attempts;  /* attempts made (<= rejection_limit)                 */
  int32_t accepted;  /* 1 if a step was accepted                           */
  int32_t last_step; /* 1 if the solver decided to stop                    */
  int64_t n_weno;    /* cells sent to WENO in the last RHS evaluation      */
  int64_t n_rhs;     /* total RHS evaluations so far                       */
  int32_t write_plot; /* 1 if the step ended on a plot time or the final time
                         (Solver.cpp:197-205); reported once               */
  int32_t reserved;
} kfvm_step_info;

typedef struct kfvm_solver kfvm_solver;

/* Fills a config with the reference's defaults (ProblemSetup.H:72-82,
 * ParameterStructs.H:37). */
void kfvm_default_config(kfvm_config *cfg);

/* Stencil geometry and reconstruction weights, host FP64, LU by LAPACK
 * dgetrf/dgetrs.  Replaces Stencil::Stencil(lfac, geom)
 * (src/stencil/Stencil.H:105-135) -> Core::findStencil (Stencil.cpp:47-156),
 * findSubStencils (Stencil.cpp:158-229), findWeights (Stencil.cpp:281-846). */
int kfvm_stencil_build(const kfvm_config *cfg, kfvm_stencil *out);

/* Allocates all device state for one solver.  Replaces the allocation part of
 * Solver::Solver (src/Solver.cpp:36-81).  Uses the current CUDA device. */
int kfvm_create(const kfvm_config *cfg, kfvm_solver **out);
void kfvm_destroy(kfvm_solver *s);

/* Fills U (and Uprev) with a built-in initial condition, evaluates the first
 * RHS to prime the FSAL stepper and picks dt = 0.01 cfl dmin / maxVel.
 * Replaces Solver::setIC (src/Solver.cpp:1948-1963) and the tail of
 * Solver::Solver (src/Solver.cpp:73-80).  seed feeds KFVM_IC_KELVIN_HELMHOLTZ. */
int kfvm_init_ic(kfvm_solver *s, int32_t ic_kind, uint64_t seed);

/* Sets U = Uprev = host state (SoA interior), then primes FSAL as above. */
int kfvm_set_state(kfvm_solver *s, const double *u_host);
/* Copies U (SoA interior) to the host. */
int kfvm_get_state(kfvm_solver *s, double *u_host);

/* One RHS evaluation on the current U at time t.  Replaces
 * Solver::evalRHS(U_halo, t) (src/Solver.cpp:410-530): cell BCs, linear
 * reconstruction, KXRCF selection, sparse/full WENO, positivity limiter, face
 * BCs, GLM speed and sources, Riemann fluxes with the max-speed reduction,
 * flux divergence and viscous terms.  rhs_host (nullable) receives the RHS in
 * SoA interior layout; max_vel (nullable) the max wave speed. */
int kfvm_eval_rhs(kfvm_solver *s, double t, double *rhs_host, double *max_vel);

/* Embedded error estimate of a state pair (RKFSAL_ErrEst_K,
 * src/numeric/Numeric_K.H:262-290): err = sum over cells and variables of
 * ((u-uhat)/(atol+rtol*max(|u|,|uhat|)))^2 with the solver's atol/rtol, and
 * posmin = min over cells of the positivity function (-1 where u holds a NaN).
 * u_dev and uhat_dev are device arrays in SoA interior layout of this solver's
 * grid; err and posmin are host pointers.  Uses the solver's scratch memory. */
int kfvm_err_est(kfvm_solver *s, const double *u_dev, const double *uhat_dev, double *err,
                 double *posmin);

/* Capacity of kfvm_err_est_noalloc's fixed scratch array (cells). */
#define KFVM_NOALLOC_MAX_CELLS (1 << 24)

/* The error estimate of kfvm_err_est without any allocation and without a
 * solver handle.  No counterpart in the reference: it serves callers that cannot
 * call cudaMalloc -- code whose device memory is owned by another allocator (a
 * host framework's memory pool with a fixed budget) or that runs in a setting
 * where device allocation after start-up is not permitted.  The caller passes the
 * inputs (u_dev, uhat_dev: n cells x NV variables, SoA, on the device) and the
 * output (out_dev: 2 doubles on the device, receiving err and posmin as in
 * kfvm_err_est); stream is a cudaStream_t (NULL for the legacy default stream).
 * Its scratch is a 1 MiB file-scope device array that every GPU loading the
 * library holds until exit; n above KFVM_NOALLOC_MAX_CELLS is rejected with
 * KFVM_ERR_ARG.  Every call looks up that array's device address on the current
 * device (cudaGetSymbolAddress, so a cudaDeviceReset in between is harmless); the
 * first call on a device also loads the library's device code there and should
 * come before any stream capture.  All calls
 * on one GPU share that GPU's copy of the array: calls that overlap on the same
 * GPU (for example on two streams) race and must be serialised by the caller.
 * Each call overwrites the scratch it reads, so no clearing is needed between
 * calls. */
int kfvm_err_est_noalloc(int32_t eq, const double *u_dev, const double *uhat_dev, int64_t n,
                         double atol, double rtol, double *out_dev, void *stream);

/* One adaptive FSAL time step.  Replaces Solver::TakeStep (src/Solver.cpp:188-343). */
int kfvm_take_step(kfvm_solver *s, kfvm_step_info *info);

/* Steps until max_steps / final_time / stagnation, like the loop of
 * Solver::Solve (src/Solver.cpp:84-140) without I/O.  n_steps_out (nullable)
 * receives the number of accepted steps. */
int kfvm_solve(kfvm_solver *s, int32_t max_steps, int64_t *n_steps_out,
               kfvm_step_info *last);

/* Current simulation time and dt (Solver::time, Solver::dt). */
int kfvm_get_time(kfvm_solver *s, double *time, double *dt);
/* Sets the simulation time and the size of the next step, as a restart from a
 * checkpoint does (Solver::Solver reading time and dt, src/Solver.cpp:57-66). */
int kfvm_set_time(kfvm_solver *s, double time, double dt);

/* Selects the troubled-cell indicator (enum kfvm_indicator). */
int kfvm_set_indicator(kfvm_solver *s, int32_t indicator);

/* Selects the arithmetic of the linear reconstruction contraction (enum
 * kfvm_precision).  KFVM_PREC_FP64 (default) is the reference's arithmetic and
 * summation order.  KFVM_PREC_TF32X3 computes the stencil sum of the light
 * (non-WENO) cells on the tcgen05 tensor cores: differences to the cell average
 * in FP32, split into two TF32 terms, three MMAs per K step, FP32 accumulation;
 * weights precompute, WENO cells, positivity, Riemann fluxes and the RK update
 * stay FP64.  No reference counterpart (the reference computes in FP64 only).
 * KFVM_ERR_ARG if the device is not compute capability 10.x. */
int kfvm_set_precision(kfvm_solver *s, int32_t precision);

/* Self-test of the bounded waits of the tensor-core kernels (no reference
 * counterpart): one thread waits on an mbarrier that nothing completes, with a
 * limit of limit_s seconds (0 < limit_s <= 1), and reports that it gave up and
 * how long it waited.  The tensor-core kernels use the same wait (1 s limit) and
 * turn a timeout into KFVM_ERR_CUDA on the host instead of a hang. */
int kfvm_selftest_wait(double limit_s, int32_t *gave_up, double *waited_s);

/* Self-test of the FP64 reciprocal used by the Riemann solvers (Newton-Raphson
 * refinement of the hardware approximation): over n pseudo-random doubles with
 * exponents in [-300, 300] and both signs, the largest distance in ulps between
 * it and the IEEE quotient 1/y, and the largest relative difference between
 * x * rcp(y) and x / y.  No reference counterpart (the reference divides). */
int kfvm_selftest_rcp(int64_t n, uint64_t seed, int64_t *max_ulp, double *max_rel_quot);

/* ---- Learned troubled-cell indicator (KFVM_IND_MLP) -----------------------
 * No reference counterpart: it replaces the KXRCF selector (WenoSelect_K,
 * src/numeric/Numeric_K.H:292-398) with a 2x32 MLP over the normalised 5^d
 * density / pressure patch of a cell: inputs x = (q_k - q_c) / (max|q_k - q_c| +
 * 1e-4 |q_c|), q = rho then p, 50 (2D) or 250 (3D); NI -> 32 -> 32 -> 1 with GELU
 * in its tanh approximation, x sigma(2 sqrt(2/pi) (x + 0.044715 x^3)), and a
 * sigmoid; BF16 weights, FP32 accumulation.  Weight layout (raw BF16):
 * W1[32][NI], b1[32], W2[32][32], b2[32], w3[32], b3.
 * Labels come from the method: a cell is troubled when the normalised WENO-JS
 * weights of its density or pressure (createOmegas, Stencil_K.H:556-580) depart
 * from the linear weights by more than tau somewhere.  In the stage, a hashed
 * fraction of the runs of 32 consecutive cells along x (the judge) always runs
 * full WENO; their labels are compared
 * with the predictions, and a step whose judged troubled cells were missed more
 * often than miss_limit sends the next two steps to KXRCF.  The kfvm_mlp_* calls
 * allocate the buffers they need; stepping still allocates nothing. */
/* number of weights for dim 2 or 3 (2721 / 9121), or KFVM_ERR_ARG */
int kfvm_mlp_num_weights(int32_t dim);
/* Glorot-uniform initial weights (zero biases) from seed; clears Adam state */
int kfvm_mlp_init_weights(kfvm_solver *s, uint64_t seed);
/* load / read the BF16 weights (n = kfvm_mlp_num_weights(dim)) */
int kfvm_mlp_set_weights(kfvm_solver *s, const uint16_t *bf16, int64_t n);
int kfvm_mlp_get_weights(kfvm_solver *s, uint16_t *bf16_out, int64_t n);
/* allocate (and empty) the training-sample buffer for up to capacity samples */
int kfvm_mlp_reserve(kfvm_solver *s, int64_t capacity);
/* append samples of the current state: every cell with departure > tau, other
 * cells with probability keep_frac (hashed with seed); totals of the buffer */
int kfvm_mlp_collect(kfvm_solver *s, double tau, double keep_frac, uint64_t seed, int64_t *n_samples,
                     int64_t *n_positive);
/* copy samples [first, first+count): BF16 features [count][NI], labels, cell index */
int kfvm_mlp_get_samples(kfvm_solver *s, int64_t first, int64_t count, uint16_t *feats_bf16, uint8_t *labels,
                         int64_t *cells);
/* Adam on the weighted binary cross entropy (positives weighted pos_weight):
 * steps minibatches of batch samples drawn from the buffer; mean loss of the
 * first and of the last 20 steps */
int kfvm_mlp_train(kfvm_solver *s, int32_t steps, int32_t batch, double lr, double pos_weight, uint64_t seed,
                   double *loss_first, double *loss_last);
/* decision threshold on the probability (default 0.5), judge fraction (1/256),
 * label threshold tau (0.3), allowed miss rate of the judge (0.25) */
int kfvm_mlp_config(kfvm_solver *s, double prob_threshold, double judge_frac, double tau, double miss_limit);
/* network probability of every cell for the current state ([nz][ny][nx]);
 * allocates a temporary device array */
int kfvm_mlp_probability(kfvm_solver *s, float *out_host);
/* cumulative judge counts: judged, of them troubled, troubled but missed,
 * predicted but not troubled; fallback events; fallback steps left */
int kfvm_mlp_stats(kfvm_solver *s, int64_t *out6);

/* Inspection of the last RHS evaluation, for parity tests:
 * face states after the positivity limiter and face BCs, before the Riemann
 * solve, in layout double[2 slots][NQF][NV][nfz][nfy][nfx] where (nfx,nfy,nfz)
 * is the face grid of direction dir (nx+1,ny,nz for x, ...).  Slot 0 is the
 * minus (left) state, slot 1 the plus (right) state, as in FaceDataView
 * (src/Types.H:73,87-88). */
int kfvm_get_faces(kfvm_solver *s, int32_t dir, double *out_host);
/* Per-cell WENO flags of the last RHS evaluation (1 = WENO reconstruction was
 * applied to the cell) and positivity theta (wenoFlag(.,1)); either pointer may
 * be null.  Layout [nz][ny][nx]. */
int kfvm_get_flags(kfvm_solver *s, uint8_t *weno_applied, double *theta);

/* ---- Plot and checkpoint files (src/io/WriterPDI.cpp, user/pdi_*_xdmf.yml) ----
 * XDMF 2 descriptions with raw little-endian FP64 datasets ([z][y][x], x fastest)
 * where the reference writes HDF5 through PDI; the dataset names, the 3DRectMesh
 * of nodal coordinates and the attribute list follow WriterPDI::writeXML.  A file
 * set is <dir>/<base>_<num:07d>.xmf, .<dataset>.bin per dataset and .meta (time,
 * time step, time step size, gamma, grid).  Conserved datasets always, the
 * auxiliary ones (vel*, eint, pres | prsg prsb) only for plots (ckpt = 0), and
 * weno / fomx (the two components of the WENO flag view: WENO applied, positivity
 * theta) in both.  u is the host-order state [v][z][y][x] of kfvm_get_state.
 * The directory is created if missing.  KFVM_ERR_IO if a file cannot be written. */
int kfvm_plotfile_write(const kfvm_config *cfg, const char *dir, const char *base, int32_t num, int32_t ckpt,
                        int32_t time_step, double time, double dt, const double *u, const uint8_t *weno,
                        const double *theta);
/* Reads a file set written by kfvm_plotfile_write (path of the .xmf).  The grid,
 * dimension and equations recorded in its .meta must match cfg (KFVM_ERR_ARG
 * otherwise); a missing or short dataset is KFVM_ERR_IO. */
int kfvm_plotfile_read(const kfvm_config *cfg, const char *xmf_path, double *u, uint8_t *weno, double *theta,
                       int32_t *time_step, double *time, double *dt);
/* The solver's current state, flags, time and step size written as above
 * (WriterPDI::writePlot / writeCkpt, Solver.cpp:113-122). */
int kfvm_write_plotfile(kfvm_solver *s, const char *dir, const char *base, int32_t num, int32_t ckpt,
                        int32_t time_step);
/* Restart from a checkpoint (Solver::Solver with ps.restart, Solver.cpp:60-80):
 * state, WENO flags and positivity theta from the file, the FSAL priming
 * evaluation with those flags, then time and step size from the file; returns
 * the file's time step (the caller continues at time_step + 1). */
int kfvm_restart(kfvm_solver *s, const char *xmf_path, int32_t *time_step);
/* Plot times for the step-size limit of kfvm_take_step: with plot_freq > 0 a step
 * that would pass plot_num * plot_freq is shortened to end on it and reports
 * write_plot (Solver.cpp:202-205).  The caller advances plot_num after writing. */
int kfvm_set_plot_freq(kfvm_solver *s, double plot_freq, int32_t plot_num);

/* Device time of the last kfvm_take_step call, for measurement (ms). */
int kfvm_last_stage_ms(kfvm_solver *s, double *ms);

/* Measurement support (no counterpart in the reference, which has no timers).
 * kfvm_get_stream: the cudaStream_t (as void*) all work of this solver runs on.
 * kfvm_set_timing: when on, CUDA events bracket every kernel class and the device
 *   time of each class accumulates; kfvm_get_timing copies the per-class totals
 *   (ms) and launch counts for the classes listed by KFVM_KCLASS_*.
 * kfvm_get_launch_count: kernels launched by this solver since creation. */
enum kfvm_kernel_class {
  KFVM_KCLASS_BC = 0, KFVM_KCLASS_SELECT = 1 /* WENO decision + heavy-list compaction */,
  KFVM_KCLASS_FLAG = 2, KFVM_KCLASS_RECON = 3, KFVM_KCLASS_HEAVY = 4, KFVM_KCLASS_RIEMANN = 5,
  KFVM_KCLASS_STAGE = 6, KFVM_KCLASS_OTHER = 7, KFVM_NUM_KCLASS = 8
};
int kfvm_get_stream(kfvm_solver *s, void **stream);
int kfvm_set_timing(kfvm_solver *s, int32_t on);
int kfvm_get_timing(kfvm_solver *s, double *ms_per_class, int64_t *launches_per_class);
int kfvm_get_launch_count(kfvm_solver *s, int64_t *launches);
/* Measured FP64 tensor-pipe throughput of the current device (no counterpart in
 * the reference): back-to-back independent m8n8k4 FP64 MMAs on every SM, timed
 * with CUDA events over about 10 ms; *tflops receives the rate in TFLOP/s (an
 * MMA = 512 flops).  The denominator of the FP64 reconstruction's roofline. */
int kfvm_measure_fp64_mma(double *tflops);
/* The equal-state Riemann variant (no counterpart in the reference): whether the
 * next Riemann launches use it (on: 0 or 1) and the cumulative number of face
 * points sampled for the choice and of those whose two states agree to 1e-14
 * (any pointer may be null). */
int kfvm_get_same_state(kfvm_solver *s, int32_t *on, int64_t *sampled, int64_t *equal);

/* ---- domain decomposition (multi-rank) ----
 * The reference's block decomposition and its boundary communication
 * (src/LayoutMPI.H:44-97, src/Solver.cpp:826-1460, src/BoundaryData.cpp), one
 * solver per rank.  kfvm_block_config turns the configuration of one block of a
 * decomposed domain (nb set, block ignored) into rank `rank`'s configuration:
 * its block coordinates (MPI Cartesian order, rank = (bx nb[1] + by) nb[2] + bz)
 * and KFVM_BC_EXCHANGE on every face with a neighbouring block (a periodic axis
 * of more than one block wraps); neighbors[6] (nullable) receives the ranks
 * across west, east, south, north, bottom, top, -1 where there is none.
 *
 * kfvm_set_exchange installs the transport.  Per RHS evaluation the solver
 *   - fills the halo axis by axis (x, then y over the x halo, then z over both,
 *     as setCellBCs does): per axis with exchange faces it packs the r = 2 cell
 *     layers along each exchange face, calls ex(user, axis, send_lo, recv_lo,
 *     send_hi, recv_hi, bytes_lo, bytes_hi), unpacks into the halo, then fills
 *     the axis's physical faces;
 *   - exchanges the boundary face states (and, for the KXRCF selector, the
 *     indicator values) after the linear reconstruction and again after the
 *     limiter, as the two setFaceBCs calls of evalRHS do (axis = 3 + face
 *     axis);
 *   - reduces the GLM cleaning-speed maxima (max) before the Riemann solve,
 *     and per step attempt the wave-speed maximum (max), the error sum (sum) and
 *     the positivity minimum (min) through ar(user, op, vals, n), in place on
 *     host doubles; kfvm_apply_forcing sums its two integrals the same way
 *     (forceStrComm), and the equal-state Riemann variant is chosen from the
 *     counts of all ranks (sum).
 * In ex, send_lo goes to the rank across the low face and send_hi to the rank
 * across the high face; recv_lo receives what the rank across the low face sent
 * from its high side and recv_hi what the high neighbour sent from its low side.
 * Buffers are device pointers (NULL and 0 bytes on a face without a
 * neighbour) and stay valid during the call only; the callback returns 0 on
 * success.  Every rank makes the same calls in the same order.  Flow
 * statistics and the learned indicator's sample collection and training work
 * on this rank's block only. */
enum kfvm_reduce_op { KFVM_REDUCE_SUM = 0, KFVM_REDUCE_MAX = 1, KFVM_REDUCE_MIN = 2 };
typedef int (*kfvm_exchange_fn)(void *user, int32_t axis, const void *send_lo, void *recv_lo,
                                const void *send_hi, void *recv_hi, int64_t bytes_lo, int64_t bytes_hi);
typedef int (*kfvm_allreduce_fn)(void *user, int32_t op, double *vals, int32_t n);
int kfvm_block_config(const kfvm_config *blocks, int32_t rank, kfvm_config *out, int32_t neighbors[6]);
int kfvm_set_exchange(kfvm_solver *s, kfvm_exchange_fn ex, kfvm_allreduce_fn ar, void *user);

/* ---- user-defined boundary conditions ----
 * For every face with KFVM_BC_USER the solver calls
 *   fn(user, kind, face, time, inner, outer, n_points, stream)
 * with device buffers that stay valid during the call only, after synchronising
 * its stream (the callback may launch work on `stream`, a cudaStream_t, or on
 * any other stream it synchronises before returning; it returns 0 on success).
 * face = 2 axis + side (west, east, south, north, bottom, top); time = the time
 * of the RHS evaluation (the stage time t + c dt).
 *   kind KFVM_USER_CELLS (setCellBCs, in its axis order: x faces, then y over the
 *   x halo, then z over both): inner holds the r = 2 interior cell layers along
 *   the face, outer receives the 2 halo layers, both as [v][layer][position]
 *   doubles.  Along the face's axis (extent n) layer h of inner is cell h (low
 *   side) or n - 2 + h (high side) and layer h of outer is cell h - 2 (low) or
 *   n + h (high); position t = p1 + e1 p2 runs over the other two axes, the lower
 *   one (p1) fastest, each over its padded range -2 .. n + 1 if that axis is
 *   filled before this one and over its interior 0 .. n - 1 otherwise (in 2D the
 *   z range is the single index 0).  Cell centres: x = x0 + dx (i + 1/2), x0 and
 *   dx as this block's geometry (kfvm_config).
 *   kind KFVM_USER_FACES (setFaceBCs): inner holds the face points' states from
 *   inside the domain, outer receives the states outside, both as [q][v][point]
 *   doubles; point runs over the face's cells in the other two axes (interior
 *   ranges, lower axis fastest) and q over its NQF quadrature points (in 3D
 *   q = q_a NQ + q_b, q_a along the lower of the two axes).  For the KXRCF
 *   selector the solver derives the outer indicator from the outer states.
 * n_points is the number of positions (cells) or face points times quadrature
 * points; the buffers hold NV such blocks. */
enum kfvm_user_kind { KFVM_USER_CELLS = 0, KFVM_USER_FACES = 1 };
typedef int (*kfvm_user_bc_fn)(void *user, int32_t kind, int32_t face, double time, const double *inner,
                               double *outer, int64_t n_points, void *stream);
int kfvm_set_user_bc(kfvm_solver *s, kfvm_user_bc_fn fn, void *user);

/* ---- random forcing (stirred turbulence) ----
 * The reference's ENABLE_RANDOM_FORCING path (src/ParameterStructs.H:20-74,
 * src/ParameterStructs.cpp:41-88, src/physics/Common_K.H:645-784,
 * src/Solver.cpp:99-103, 365-409).  Modes: the wavevectors k of the half space with
 * 0 < |k|^2 <= 9 (14 in 2D, 57 in 3D) in the reference's order; per mode and
 * direction a complex amplitude drawn as sigma N(0,1), sigma = sqrt(|k| (4 - |k|)).
 * The kick f (a Helmholtz mix of the modes, weight `ratio` on the compressive part)
 * is scaled so that it injects edot dt of kinetic energy into the domain, and is
 * added to the momenta (rho f) and the total energy; the stored FSAL stage is kept,
 * as in the reference.
 * A mode table is double[n_modes][dim][3]: (k_d, real amplitude, imaginary
 * amplitude) for each direction d. */
#define KFVM_FORCING_MAX_MODES 57
typedef struct kfvm_forcing {
  double edot;   /* eos:forceedot, energy injection rate */
  double ratio;  /* eos:forceratio, compressive-to-solenoidal weight */
  double t_off;  /* eos:forcetoff, no forcing from this time on */
  uint64_t seed; /* generator seed; the reference seeds each draw from std::random_device */
} kfvm_forcing;

/* number of forcing modes for dim (14 or 57), or KFVM_ERR_ARG */
int kfvm_forcing_num_modes(int32_t dim);
/* One draw of the mode table (EosParameters::updateForcing with its generator,
 * std::mt19937 + std::normal_distribution, seeded by seed32): host only. */
int kfvm_forcing_draw(int32_t dim, uint32_t seed32, double *modes);
/* Enables forcing on a solver (f NULL disables it).  kfvm_solve then forces before
 * every step while time < t_off (Solver::Solve, Solver.cpp:99-103).  Allocates the
 * solver's device mode table. */
int kfvm_set_forcing(kfvm_solver *s, const kfvm_forcing *f);
/* Solver::applyForcing: forces the current state once with the table modes_in, or
 * (modes_in NULL) with the next draw of the solver's generator, at the current step
 * size.  modes_out (optional) receives the table used, force_str (optional) the
 * strength.  Synchronises the solver's stream (the strength needs the domain
 * integrals). */
int kfvm_apply_forcing(kfvm_solver *s, const double *modes_in, double *modes_out, double *force_str);

/* Solver::evalFlowStats (src/Solver.cpp:153-185; FlowStats<Eq>, src/physics/hydro/
 * Hydro_K.H:103-178, navierstokes/NavierStokes_K.H:102-175, mhd_glm/MHD_GLM_K.H:108-211):
 * volume averages of the current state's kinetic energy and enstrophy (velocity
 * gradients by central differences over the boundary-filled halo), and for
 * GLM-MHD the current helicity B . curl B.  stats receives n_stats values (2; GLM-MHD
 * 3; SRHydro 1, always 0 as in the reference), n_stats may be NULL.  Synchronises
 * the solver's stream. */
int kfvm_flow_stats(kfvm_solver *s, double *stats, int32_t *n_stats);

/* Human-readable text for the last error on this thread. */
const char *kfvm_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* KFVM_B200_H_ */
