"""TEST INFRASTRUCTURE ONLY: build the reference solver itself, on the CPU.

The reference (slug-cfd/kfvm-kokkos) is one C++17 executable per problem: its
src/ is compiled together with a problem directory of user headers
(Definitions.H, InitialCondition.H, SourceTerms.H, UserBCs.H, UserParameters.H,
ProblemSetup.cpp; src/CMakeLists.txt:10-12).  Kokkos, KokkosKernels, MPI and PDI
are not installed here, so the reference's sources are compiled UNCHANGED
against the host-only stand-ins in oracle/refshim/ (OpenMP loops, a one-rank
MPI, a PDI that writes checkpoints as raw files), with LAPACK from the OpenBLAS
bundled with scipy.  No reference file is copied: g++ reads them where they lie.

For every benchmark problem this script writes the problem directory (the
user-side code a reference user writes for a problem: the problem's initial
condition as this repository states it, its boundary types and compile-time
choices) into oracle/_ref/<problem>/ and compiles oracle/_ref/<problem>/kfvm_ref.
Run it with the reference's path:

    python oracle/build_ref.py /path/to/kfvm-kokkos [problem ...]

oracle/_ref/ is build output (git-ignored).  The binaries are used by
tests/golden/make_ref_fixtures.py (golden states from the reference's own run),
by tests that compare the oracle and the CUDA path with those states, and by
bench.py's reference arm (the reference's CPU code timed on the host cores).
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
SHIM = os.path.join(HERE, "refshim")
OUT = os.path.join(HERE, "_ref")

# Reference sources of the kfvm.ex target (src/CMakeLists.txt:10 and the
# numeric / stencil / io libraries), relative to the reference's src/.
REF_SOURCES = ["main.cpp", "Solver.cpp", "BoundaryData.cpp", "ParameterStructs.cpp",
               "numeric/Numeric.cpp", "stencil/Stencil.cpp", "stencil/ReconVectors.cpp",
               "stencil/StencilSymmetry.cpp", "stencil/Monomials.cpp", "io/WriterPDI.cpp"]

# ---------------------------------------------------------------- problems
# Each problem: compile-time choices (Definitions.H), boundary types
# (ProblemSetup.cpp), whether the GLM source terms are on, and the initial
# condition at a point (InitialCondition.H).  The initial conditions are the
# ones this repository states for its workloads (csrc/ic.cu, the oracle's
# ic_point); the Kelvin-Helmholtz noise needs the cell index, which the user
# function recovers from the point's coordinates (Gauss points lie strictly
# inside their cell).
IC_VORTEX = r"""
  (void)z; (void)userParams;
  const Real g = eosParams.gamma, gm = g - 1.0;
  const Real beta = 5.0, r2 = x * x + y * y;
  const Real f = beta / (2.0 * M_PI) * std::exp(0.5 * (1.0 - r2));
  const Real u = 1.0 - y * f, v = 1.0 + x * f;
  const Real T = 1.0 - gm * beta * beta / (8.0 * g * M_PI * M_PI) * std::exp(1.0 - r2);
  const Real rho = std::pow(T, 1.0 / gm), p = rho * T;
  state[0] = rho;
  state[1] = rho * u;
  state[2] = rho * v;
  state[3] = 0.0;
  state[4] = p / gm + 0.5 * rho * (u * u + v * v);
"""

IC_SOD = r"""
  (void)userParams;
  const Real gm = eosParams.gamma - 1.0;
  const Real dx = x - 0.5, dy = y - 0.5, dz = z - 0.5;
  const bool in = std::sqrt(dx * dx + dy * dy + dz * dz) < 0.2;
  const Real rho = in ? 1.0 : 0.125, p = in ? 1.0 : 0.1;
  state[0] = rho;
  state[1] = 0.0;
  state[2] = 0.0;
  state[3] = 0.0;
  state[4] = p / gm;
"""

IC_KH = r"""
  (void)z;
  const Real gm = eosParams.gamma - 1.0;
  // cell index of the point, then the cell's seeded noise (splitmix64 of the
  // seed xor the cell index, uniform in [-1e-3, 1e-3])
  const int64_t i = (int64_t)std::floor((x - userParams.khXlo) / userParams.khDx);
  const int64_t j = (int64_t)std::floor((y - userParams.khYlo) / userParams.khDy);
  uint64_t s = userParams.khSeed ^ (uint64_t)(j * userParams.khNx + i);
  s += 0x9E3779B97F4A7C15ull;
  s = (s ^ (s >> 30)) * 0xBF58476D1CE4E5B9ull;
  s = (s ^ (s >> 27)) * 0x94D049BB133111EBull;
  s = s ^ (s >> 31);
  const Real u01 = (Real)(s >> 11) * (1.0 / 9007199254740992.0);
  const Real noise = 1.0e-3 * (2.0 * u01 - 1.0);
  const bool in = std::fabs(y - 0.5) < 0.25;
  const Real rho = in ? 2.0 : 1.0, u = in ? 0.5 : -0.5, p = 2.5;
  const Real v = 0.01 * std::sin(4.0 * M_PI * x) + noise;
  state[0] = rho;
  state[1] = rho * u;
  state[2] = rho * v;
  state[3] = 0.0;
  state[4] = p / gm + 0.5 * rho * (u * u + v * v);
"""

IC_TGV = r"""
  const Real g = eosParams.gamma, gm = g - 1.0;
  const Real mach = userParams.mach;
  const Real gMasq = g * mach * mach;
  const Real u = std::sin(x) * std::cos(y) * std::cos(z);
  const Real v = -std::cos(x) * std::sin(y) * std::cos(z);
  const Real w = 0.0;
  const Real q = (std::cos(2.0 * x) + std::cos(2.0 * y)) * (std::cos(2.0 * z) + 2.0);
  const Real rho = 1.0 + gMasq * q / 16.0;
  const Real p = 1.0 / gMasq + q / 16.0;
  state[0] = rho;
  state[1] = rho * u;
  state[2] = rho * v;
  state[3] = rho * w;
  state[4] = p / gm + 0.5 * rho * (u * u + v * v + w * w);
"""

IC_OT = r"""
  (void)z; (void)userParams;
  const Real g = eosParams.gamma, gm = g - 1.0;
  const Real rho = g * g, p = g;
  const Real u = -std::sin(2.0 * M_PI * y), v = std::sin(2.0 * M_PI * x), w = 0.0;
  const Real bx = -std::sin(2.0 * M_PI * y), by = std::sin(4.0 * M_PI * x), bz = 0.0;
  state[0] = rho;
  state[1] = rho * u;
  state[2] = rho * v;
  state[3] = rho * w;
  state[4] = p / gm + rho * (u * u + v * v + w * w) / 2.0 + (bx * bx + by * by + bz * bz) / 2.0;
  state[5] = bx;
  state[6] = by;
  state[7] = bz;
  state[8] = 0.0;
"""

IC_SR_RIEM2D = r"""
  (void)z; (void)userParams;
  // four-quadrant special-relativistic Riemann problem (the states of the
  // repository's sr_riemann_2d workload), as D, S and E from the primitives
  const Real gR = eosParams.gamma / (eosParams.gamma - 1.0), v0 = 0.99;
  Real rho, vx, vy, p;
  if (x > 0.0) {
    if (y > 0.0) { rho = 0.1; vx = 0.0; vy = 0.0; p = 0.01; }
    else { rho = 0.1; vx = 0.0; vy = v0; p = 1.0; }
  } else {
    if (y > 0.0) { rho = 0.1; vx = v0; vy = 0.0; p = 1.0; }
    else { rho = 0.5; vx = 0.0; vy = 0.0; p = 1.0; }
  }
  const Real W = 1.0 / std::sqrt(1.0 - vx * vx - vy * vy), h = 1.0 + p * gR / rho;
  state[0] = rho * W;
  state[1] = rho * W * W * h * vx;
  state[2] = rho * W * W * h * vy;
  state[3] = 0.0;
  state[4] = rho * W * W * h - p;
"""

# a supersonic inflow through the western face (the kind of boundary the
# DoubleMach problem writes in its UserBCs.H): rho 1.5, u 1.2, p 1.5 in every
# halo cell and every outer face point
INFLOW_STATE = r"""
  state[0] = 1.5;
  state[1] = 1.5 * 1.2;
  state[2] = 0.0;
  state[3] = 0.0;
  state[4] = 1.5 / (eosParams.gamma - 1.0) + 0.5 * 1.5 * 1.2 * 1.2;
"""


IC_SR_SHOCK_TUBE = r"""
  (void)y; (void)z; (void)userParams;
  // the repository's relativistic shock tube: a dense hot slab for x < 0.5 at rest
  const Real gR = eosParams.gamma / (eosParams.gamma - 1.0), ax = std::fabs(x), W = 1.0;
  const Real rho = ax < 0.5 ? 10.0 : 1.0, p = ax < 0.5 ? 40.0 / 3.0 : 1.e-6;
  const Real h = 1.0 + p * gR / rho;
  state[0] = rho * W;
  state[1] = 0.0;
  state[2] = 0.0;
  state[3] = 0.0;
  state[4] = rho * h * W * W - p;
"""

PROBLEMS = {
    # name: (dim, eq, rs, rk, nq, bc, sources, ic body)
    "isentropic_vortex": (2, "Hydro", "HLLC", "SSP4_3_2", 2, "periodic", False, IC_VORTEX),
    "sod3d": (3, "Hydro", "HLLC", "SSP4_3_2", 2, "outflow", False, IC_SOD),
    "kelvin_helmholtz": (2, "Hydro", "HLLC", "SSP4_3_2", 2, "periodic", False, IC_KH),
    "taylor_green": (3, "NavierStokes", "HLLC", "SSP4_3_2", 2, "periodic", False, IC_TGV),
    "orszag_tang": (2, "MHD_GLM", "HLL", "SSP4_3_2", 2, "periodic", True, IC_OT),
    "orszag_tang_3d": (3, "MHD_GLM", "HLL", "SSP4_3_2", 2, "periodic", True, IC_OT),
    # three Gauss points (NUM_QUAD_PTS 3, as MHD/MagVort3d): 27 interior source points
    "orszag_tang_3d_q3": (3, "MHD_GLM", "HLL", "SSP4_3_2", 3, "periodic", True, IC_OT),
    # special-relativistic hydro (the Newton pressure recovery and its limiter)
    "sr_riemann_2d": (2, "SRHydro", "LLF", "SSP4_3_2", 2, "outflow", False, IC_SR_RIEM2D),
    # walls: reflecting on every face of the blast; no-slip y faces of the
    # otherwise periodic Taylor-Green box (west east south north bottom top)
    "sod3d_reflecting": (3, "Hydro", "HLLC", "SSP4_3_2", 2, ("reflecting",) * 6, False, IC_SOD),
    "taylor_green_noslip": (3, "NavierStokes", "HLLC", "SSP4_3_2", 2,
                            ("periodic", "periodic", "noslip", "noslip", "periodic", "periodic"), False, IC_TGV),
    # the other Runge-Kutta schemes, Riemann solvers and the three-point rule in 2D
    "sod3d_ssp10": (3, "Hydro", "HLLC", "SSP10_4_3", 2, "outflow", False, IC_SOD),
    "vortex_threestar": (2, "Hydro", "HLLC", "ThreeStarP", 2, "periodic", False, IC_VORTEX),
    "sod3d_fourstar": (3, "Hydro", "HLLC", "FourStarP", 2, "outflow", False, IC_SOD),
    "kelvin_helmholtz_hll": (2, "Hydro", "HLL", "SSP4_3_2", 2, "periodic", False, IC_KH),
    "kelvin_helmholtz_q3": (2, "Hydro", "HLLC", "SSP4_3_2", 3, "periodic", False, IC_KH),
    "sod3d_llf": (3, "Hydro", "LLF", "SSP4_3_2", 2, "outflow", False, IC_SOD),
    "orszag_tang_llf": (2, "MHD_GLM", "LLF", "SSP4_3_2", 2, "periodic", True, IC_OT),
    # three Gauss points in 3D for Euler and Navier-Stokes (54 reconstruction rows)
    "sod3d_q3": (3, "Hydro", "HLLC", "SSP4_3_2", 3, "outflow", False, IC_SOD),
    "taylor_green_q3": (3, "NavierStokes", "HLLC", "SSP4_3_2", 3, "periodic", False, IC_TGV),
    # a user boundary: the supersonic inflow through the western face of the blast
    "sod3d_inflow": (3, "Hydro", "HLLC", "SSP4_3_2", 2, ("user",) + ("outflow",) * 5, False, IC_SOD),
    # 2D walls (reflecting y faces) for Euler and GLM-MHD, and SR in 3D with HLL
    "kelvin_helmholtz_reflect": (2, "Hydro", "HLLC", "SSP4_3_2", 2,
                                 ("periodic", "periodic", "reflecting", "reflecting", "periodic", "periodic"),
                                 False, IC_KH),
    "orszag_tang_reflect": (2, "MHD_GLM", "HLL", "SSP4_3_2", 2,
                            ("periodic", "periodic", "reflecting", "reflecting", "periodic", "periodic"),
                            True, IC_OT),
    "sr_shock_tube": (3, "SRHydro", "HLL", "SSP4_3_2", 2, ("outflow", "outflow") + ("periodic",) * 4, False,
                      IC_SR_SHOCK_TUBE),
    # Navier-Stokes in 2D (the two-dimensional viscous terms) on the shear layers
    "kelvin_helmholtz_ns": (2, "NavierStokes", "HLLC", "SSP4_3_2", 2, "periodic", False, IC_KH),
    # the remaining wall combinations: no-slip for Euler, reflecting for Navier-Stokes,
    # reflecting z walls for 3D GLM-MHD
    "sod3d_noslip": (3, "Hydro", "HLLC", "SSP4_3_2", 2, ("noslip",) * 6, False, IC_SOD),
    "taylor_green_reflect": (3, "NavierStokes", "HLLC", "SSP4_3_2", 2,
                             ("reflecting",) * 2 + ("periodic",) * 4, False, IC_TGV),
    "orszag_tang_3d_reflect": (3, "MHD_GLM", "HLL", "SSP4_3_2", 2, ("periodic",) * 4 + ("reflecting",) * 2,
                               True, IC_OT),
}
# user boundary hooks of the problems that have BCType::user faces
USER_BCS = {"sod3d_inflow": {"CellWest": INFLOW_STATE, "FaceWest": INFLOW_STATE}}


def definitions_h(dim, eq, rs, rk, nq):
    return f"""#ifndef DEFINITIONS_H_
#define DEFINITIONS_H_
// Compile-time choices of this problem (generated by oracle/build_ref.py)
#include "numeric/RKTypes.H"
#include "physics/EquationTypes.H"
#include "physics/RSTypes.H"
#include "stencil/KernelTypes.H"
#define SPACE_DIM {dim}
#define STENCIL_RADIUS 2
#define NUM_QUAD_PTS {nq}
#define KFVM_EXEC_HOST
constexpr KFVM::KernelType kernelType = KFVM::KernelType::SE;
constexpr KFVM::EquationType eqType = KFVM::EquationType::{eq};
constexpr KFVM::RSType rsType = KFVM::RSType::{rs};
constexpr KFVM::RKType rkType = KFVM::RKType::{rk};
#endif
"""


def initial_condition_h(body):
    return f"""// Initial condition of this problem at a point (generated by oracle/build_ref.py)
#include <cmath>
#include <cstdint>
#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
KOKKOS_INLINE_FUNCTION
void InitialCondition(Real x, Real y, Real z, EosParameters eosParams,
                      UserParameters userParams, Real state[NUM_VARS]) {{
{body}
}}
"""


SOURCE_TERMS_H = """// No user source terms (generated by oracle/build_ref.py)
KOKKOS_INLINE_FUNCTION
void SourceTerm(Real t, Real x, Real y, Real z, EosParameters eosParams,
                UserParameters userParams, const Real state[NUM_VARS],
                Real force[NUM_VARS]) {
  (void)t; (void)x; (void)y; (void)z; (void)eosParams; (void)userParams;
  (void)state; (void)force;
}
"""

USER_PARAMETERS_H = """// User parameters of the problems (generated by oracle/build_ref.py): the
// Taylor-Green Mach number (read through std::stof, as the reference's
// TaylorGreen problem does) and the Kelvin-Helmholtz noise grid and seed
// (read exactly).
struct UserParameters : ParameterStructs {
  Real mach, khXlo, khYlo, khDx, khDy;
  int64_t khNx;
  uint64_t khSeed;
  UserParameters() : mach(0.1), khXlo(0), khYlo(0), khDx(1), khDy(1), khNx(1), khSeed(0) {}
  bool set(const std::string &fld, const std::string &val) {
    std::size_t pos;
    if (fld == "mach") {
      mach = std::stof(val, &pos);
    } else if (fld == "khxlo") {
      khXlo = std::stod(val, &pos);
    } else if (fld == "khylo") {
      khYlo = std::stod(val, &pos);
    } else if (fld == "khdx") {
      khDx = std::stod(val, &pos);
    } else if (fld == "khdy") {
      khDy = std::stod(val, &pos);
    } else if (fld == "khnx") {
      khNx = std::stoll(val, &pos);
    } else if (fld == "khseed") {
      khSeed = std::stoull(val, &pos);
    } else {
      return false;
    }
    return true;
  }
};
"""


def user_bcs_h(bodies=None):
    """The twelve user boundary hooks every problem must define; bodies maps a hook
    name (CellWest, FaceWest, ...) to its code, the others are empty."""
    bodies = bodies or {}
    out = ["#ifndef USERBCS_H_", "#define USERBCS_H_",
           "// User boundary hooks (generated by oracle/build_ref.py)"]
    for side, (a, b) in (("West", ("j", "k")), ("East", ("j", "k")), ("South", ("i", "k")),
                         ("North", ("i", "k")), ("Bottom", ("i", "j")), ("Top", ("i", "j"))):
        n = {"West": "nX", "East": "nX", "South": "nY", "North": "nY", "Bottom": "nZ", "Top": "nZ"}[side]
        cell = bodies.get("Cell" + side, f"(void){n}; (void){a}; (void){b}; (void)eosParams; (void)state;")
        face = bodies.get("Face" + side, f"(void){a}; (void){b}; (void)eosParams; (void)state;")
        out.append(f"""template <class DataViewType>
KOKKOS_INLINE_FUNCTION void Cell{side}(const DataViewType &, int, int {n}, int {a}, int {b},
    int, Real, Real, Real, Real, EosParameters eosParams, UserParameters, Real state[NUM_VARS]) {{ {cell} }}
template <class DataViewType>
KOKKOS_INLINE_FUNCTION void Face{side}(const DataViewType &, int {a}, int {b}, int, Real, Real,
    Real, Real, EosParameters eosParams, UserParameters, Real state[NUM_VARS]) {{ {face} }}""")
    out.append("#endif")
    return "\n".join(out) + "\n"


def problem_setup_cpp(bc, sources):
    """bc: one boundary type for every face, or six (west east south north bottom top)."""
    names = (bc,) * 6 if isinstance(bc, str) else tuple(bc)
    b = ", ".join(f"KFVM::BCType::{n}" for n in names)
    return f"""// Boundary types and source-term switch of this problem (generated by oracle/build_ref.py)
#include <array>
#include "BoundaryConditions_K.H"
#include "ProblemSetup.H"
std::array<KFVM::BCType, 6> KFVM::ProblemSetup::bcType = {{{b}}};
bool KFVM::ProblemSetup::haveSourceTerms = {"true" if sources else "false"};
"""


def init_file(cfg, steps, datadir, base="ref", seed=12345):
    """An .init file with the configuration's settings, checkpoints every step."""
    dx = (cfg.xup - cfg.xlo) / cfg.nx
    dy = (cfg.yup - cfg.ylo) / cfg.ny
    ext = f"{cfg.xlo!r} {cfg.xup!r} {cfg.ylo!r} {cfg.yup!r}"
    res = f"{cfg.nx} {cfg.ny}"
    if cfg.dim == 3:
        ext += f" {cfg.zlo!r} {cfg.zup!r}"
        res += f" {cfg.nz}"
    return "\n".join([
        f"mesh:resolution {res}", "mesh:numblocks 1 1 1" if cfg.dim == 3 else "mesh:numblocks 1 1",
        f"mesh:extent {ext}",
        f"time:final {cfg.final_time!r}", f"time:mindt {cfg.min_dt!r}", f"time:cfl {cfg.cfl!r}",
        f"time:maxsteps {steps + 1}", f"time:atol {cfg.atol!r}", f"time:rtol {cfg.rtol!r}",
        f"time:rejectionthresh {cfg.rejection_thresh!r}", f"time:rejectionlimit {cfg.rejection_limit}",
        f"stencil:lfac {cfg.lfac!r}",
        f"eos:gamma {cfg.gamma!r}", f"eos:wenothresh {cfg.weno_thresh!r}",
        f"eos:reynolds {cfg.reynolds!r}", f"eos:prandtl {cfg.prandtl!r}",
        "io:pdiconf none", f"io:datadir {datadir}", f"io:basename {base}",
        "io:plotfreq -1.0", "io:ckptfreq 1", "io:statsfreq -1", "io:verbose 1",
        "user:mach 0.1", f"user:khxlo {cfg.xlo!r}", f"user:khylo {cfg.ylo!r}",
        f"user:khdx {dx!r}", f"user:khdy {dy!r}", f"user:khnx {cfg.nx}", f"user:khseed {seed}", ""])


def _openblas():
    import scipy
    d = os.path.dirname(scipy.__file__) + ".libs"
    for f in sorted(os.listdir(d)):
        if f.startswith("libscipy_openblas") and f.endswith(".so"):
            return d, os.path.join(d, f)
    raise RuntimeError("scipy's bundled OpenBLAS not found")


def _fmt_include():
    import torch
    return os.path.join(os.path.dirname(torch.__file__), "include")


def write_problem(name):
    dim, eq, rs, rk, nq, bc, sources, ic = PROBLEMS[name]
    d = os.path.join(OUT, name)
    os.makedirs(d, exist_ok=True)
    files = {
        "Definitions.H": definitions_h(dim, eq, rs, rk, nq),
        "InitialCondition.H": initial_condition_h(ic),
        "SourceTerms.H": SOURCE_TERMS_H,
        "UserBCs.H": user_bcs_h(USER_BCS.get(name)),
        "UserParameters.H": USER_PARAMETERS_H,
        "ProblemSetup.cpp": problem_setup_cpp(bc, sources),
    }
    for fn, txt in files.items():
        p = os.path.join(d, fn)
        if not os.path.exists(p) or open(p).read() != txt:
            with open(p, "w") as f:
                f.write(txt)
    return d


def compile_problem(ref, name, exe_name="kfvm_ref"):
    """Compile the reference's sources with this problem's headers; returns the binary."""
    d = write_problem(name)
    src = os.path.join(ref, "src")
    bdir, blas = _openblas()
    exe = os.path.join(d, exe_name)
    inc = [f"-I{d}", f"-I{SHIM}", f"-I{src}", f"-I{src}/stencil", f"-I{src}/numeric",
           f"-I{src}/io", f"-I{_fmt_include()}"]
    sources = [os.path.join(src, s) for s in REF_SOURCES]
    sources += [os.path.join(d, "ProblemSetup.cpp"), os.path.join(SHIM, "pdi_shim.cpp")]
    deps = sources + [os.path.join(d, f) for f in os.listdir(d) if f.endswith((".H", ".cpp"))]
    deps += [os.path.join(SHIM, f) for f in os.listdir(SHIM)] + [os.path.abspath(__file__)]
    if os.path.exists(exe) and all(os.path.getmtime(x) <= os.path.getmtime(exe) for x in deps):
        return exe
    cmd = ["g++", "-O2", "-std=c++17", "-fopenmp", "-ffp-contract=off", "-w",
           "-DFMT_HEADER_ONLY", "-Ddgetrf_=scipy_dgetrf_", "-Ddgetrs_=scipy_dgetrs_",
           *inc, *sources, "-o", exe, blas, f"-Wl,-rpath,{bdir}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stderr[-20000:])
        raise RuntimeError(f"reference build failed for {name}")
    return exe


def build_all(ref, names=None):
    names = names or list(PROBLEMS)
    os.makedirs(OUT, exist_ok=True)
    with ThreadPoolExecutor(max_workers=min(len(names), os.cpu_count() or 1)) as ex:
        futs = {n: ex.submit(compile_problem, ref, n) for n in names}
        out = {n: f.result() for n, f in futs.items()}
    return out


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: build_ref.py <path of the reference checkout> [problem ...]")
    print(build_all(sys.argv[1], sys.argv[2:] or None))
