"""ctypes mirror of include/kfvm_b200.h (the C ABI of the per-stage hot path).

Also holds the run configurations of the benchmark problems, built the way the
reference builds them from an .init file: every real parsed by std::stof in the
reference (src/ProblemSetup.H:229-296, src/ParameterStructs.cpp:14-39) is rounded
through float32 here.
"""
import ctypes as C
import struct

KFVM_EQ_HYDRO, KFVM_EQ_NAVIERSTOKES, KFVM_EQ_MHD_GLM, KFVM_EQ_SRHYDRO = 0, 1, 2, 3
KFVM_RS_LLF, KFVM_RS_HLL, KFVM_RS_HLLC = 0, 1, 2
KFVM_RK_THREESTARP, KFVM_RK_FOURSTARP, KFVM_RK_SSP4_3_2, KFVM_RK_SSP10_4_3 = 0, 1, 2, 3
KFVM_BC_PERIODIC, KFVM_BC_OUTFLOW, KFVM_BC_REFLECTING, KFVM_BC_NOSLIP, KFVM_BC_USER, KFVM_BC_EXCHANGE = 0, 1, 2, 3, 4, 5
KFVM_USER_CELLS, KFVM_USER_FACES = 0, 1
KFVM_REDUCE_SUM, KFVM_REDUCE_MAX, KFVM_REDUCE_MIN = 0, 1, 2
KFVM_TS_ACCEPTED, KFVM_TS_TOLERANCE, KFVM_TS_UNPHYSICAL = 0, 1, 2
KFVM_IND_KXRCF, KFVM_IND_ALL, KFVM_IND_NONE, KFVM_IND_MLP = 0, 1, 2, 3
KFVM_PREC_FP64, KFVM_PREC_TF32X3 = 0, 1
(KFVM_IC_ISENTROPIC_VORTEX, KFVM_IC_SPHERICAL_SOD, KFVM_IC_KELVIN_HELMHOLTZ,
 KFVM_IC_TAYLOR_GREEN, KFVM_IC_ORSZAG_TANG, KFVM_IC_SMOOTH_WAVE,
 KFVM_IC_SR_SHOCK_TUBE, KFVM_IC_SR_RIEMANN_2D, KFVM_IC_STIR_TURB) = range(9)
KFVM_FORCING_MAX_MODES = 57

KFVM_MAX_CELLS, KFVM_MAX_SUB, KFVM_MAX_BIAS, KFVM_MAX_BCELLS = 33, 8, 6, 11
KFVM_MAX_INDIC, KFVM_MAX_FACEQ, KFVM_MAX_CELLQ = 19, 9, 27


# the exchange and allreduce callbacks of kfvm_set_exchange (kfvm_exchange_fn,
# kfvm_allreduce_fn)
EXCHANGE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                          C.c_int64, C.c_int64)
ALLREDUCE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.c_int32)
# the user boundary callback of kfvm_set_user_bc (kfvm_user_bc_fn)
USER_BC_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int32, C.c_int32, C.c_double, C.c_void_p, C.c_void_p,
                         C.c_int64, C.c_void_p)


class KfvmConfig(C.Structure):
    _fields_ = [
        ("dim", C.c_int32), ("eq", C.c_int32), ("rs", C.c_int32), ("rk", C.c_int32),
        ("nq", C.c_int32), ("indicator", C.c_int32),
        ("nx", C.c_int64), ("ny", C.c_int64), ("nz", C.c_int64),
        ("xlo", C.c_double), ("xup", C.c_double), ("ylo", C.c_double),
        ("yup", C.c_double), ("zlo", C.c_double), ("zup", C.c_double),
        ("bc", C.c_int32 * 6),
        ("gamma", C.c_double), ("reynolds", C.c_double), ("prandtl", C.c_double),
        ("weno_thresh", C.c_double), ("lfac", C.c_double),
        ("cfl", C.c_double), ("atol", C.c_double), ("rtol", C.c_double),
        ("rejection_thresh", C.c_double), ("min_dt", C.c_double),
        ("final_time", C.c_double),
        ("rejection_limit", C.c_int32), ("max_steps", C.c_int32),
        ("have_sources", C.c_int32), ("nb", C.c_int32 * 3), ("block", C.c_int32 * 3), ("pad_", C.c_int32),
    ]


class KfvmStencil(C.Structure):
    _fields_ = [
        ("dim", C.c_int32), ("nq", C.c_int32),
        ("n_cells", C.c_int32), ("n_cells_ctr", C.c_int32), ("n_cells_bias", C.c_int32),
        ("n_sub", C.c_int32), ("n_bias", C.c_int32), ("n_indic", C.c_int32),
        ("nqf", C.c_int32), ("nqc", C.c_int32),
        ("off", (C.c_int64 * KFVM_MAX_CELLS) * 3),
        ("sub_idx", (C.c_int64 * KFVM_MAX_BCELLS) * KFVM_MAX_BIAS),
        ("face_w", ((C.c_double * KFVM_MAX_CELLS) * KFVM_MAX_FACEQ * 6) * KFVM_MAX_SUB),
        ("cell_w", ((C.c_double * KFVM_MAX_CELLS) * KFVM_MAX_CELLQ) * KFVM_MAX_SUB),
        ("deriv_w", ((C.c_double * KFVM_MAX_CELLS) * KFVM_MAX_INDIC) * KFVM_MAX_SUB),
    ]


class KfvmForcing(C.Structure):
    _fields_ = [("edot", C.c_double), ("ratio", C.c_double), ("t_off", C.c_double), ("seed", C.c_uint64)]


class KfvmStepInfo(C.Structure):
    _fields_ = [
        ("time", C.c_double), ("dt", C.c_double), ("dt_taken", C.c_double),
        ("max_vel", C.c_double), ("err_est", C.c_double),
        ("status", C.c_int32), ("attempts", C.c_int32), ("accepted", C.c_int32),
        ("last_step", C.c_int32), ("n_weno", C.c_int64), ("n_rhs", C.c_int64),
        ("write_plot", C.c_int32), ("reserved", C.c_int32),
    ]


def stof(x):
    """Round a real through float32, as std::stof does when the reference parses .init."""
    return struct.unpack("f", struct.pack("f", float(x)))[0]


def default_config():
    """The reference's defaults (ProblemSetup.H:72-82, ParameterStructs.H:37)."""
    c = KfvmConfig()
    c.dim, c.eq, c.rs, c.rk, c.nq, c.indicator = 2, KFVM_EQ_HYDRO, KFVM_RS_HLLC, KFVM_RK_SSP4_3_2, 2, KFVM_IND_KXRCF
    c.nx, c.ny, c.nz = 1, 1, 1
    c.xlo, c.xup, c.ylo, c.yup, c.zlo, c.zup = 0.0, 1.0, 0.0, 1.0, 0.0, 1.0
    for f in range(6):
        c.bc[f] = KFVM_BC_PERIODIC
    c.gamma, c.reynolds, c.prandtl, c.weno_thresh = stof(1.4), 1.0, stof(0.71), 10.0
    c.lfac = 20.0
    c.cfl, c.atol, c.rtol = 0.75, stof(1e-4), stof(1e-4)
    c.rejection_thresh, c.min_dt, c.final_time = stof(0.8), stof(1e-10), 1.0
    c.rejection_limit, c.max_steps, c.have_sources = 4, 1000, 0
    for d in range(3):
        c.nb[d], c.block[d] = 1, 0
    return c


def make_config(dim, eq, nx, ny, nz=1, extent=(0, 1, 0, 1, 0, 1), bc="periodic",
                rs=KFVM_RS_HLLC, rk=KFVM_RK_SSP4_3_2, gamma=1.4, cfl=0.8,
                weno_thresh=1.0, lfac=5.0, steps=20, reynolds=1.0, prandtl=0.71,
                indicator=KFVM_IND_KXRCF, final_time=1.0e6, atol=1e-4, rtol=1e-4):
    """Build a config as the reference would read it from an .init file
    (stof-rounded reals; time:maxsteps = steps + 1 since the loop starts at nTS=1)."""
    c = default_config()
    c.dim, c.eq, c.rs, c.rk, c.indicator = dim, eq, rs, rk, indicator
    c.nx, c.ny, c.nz = nx, ny, (nz if dim == 3 else 1)
    e = [stof(v) for v in extent]
    c.xlo, c.xup, c.ylo, c.yup = e[0], e[1], e[2], e[3]
    if dim == 3:
        c.zlo, c.zup = e[4], e[5]
    codes = {"periodic": KFVM_BC_PERIODIC, "outflow": KFVM_BC_OUTFLOW, "reflecting": KFVM_BC_REFLECTING,
             "noslip": KFVM_BC_NOSLIP}
    # one name for all faces, or one per face (west east south north bottom top)
    names = [bc] * 6 if isinstance(bc, str) else list(bc) + [bc[-1]] * (6 - len(bc))
    for f in range(6):
        c.bc[f] = codes[names[f]]
    c.gamma, c.cfl, c.weno_thresh, c.lfac = stof(gamma), stof(cfl), stof(weno_thresh), stof(lfac)
    c.reynolds, c.prandtl = stof(reynolds), stof(prandtl)
    c.atol, c.rtol, c.final_time = stof(atol), stof(rtol), stof(final_time)
    c.max_steps = steps + 1
    c.have_sources = 1 if eq == KFVM_EQ_MHD_GLM else 0
    return c


def workload(name, scale=None, steps=None):
    """The benchmark workloads (Sod 3D, Kelvin-Helmholtz, Taylor-Green, Orszag-Tang,
    isentropic vortex) and the SR-hydro and stirred-turbulence problems.

    scale, if given, replaces the grid resolution per axis (for small parity runs).
    Returns (config, ic_kind)."""
    import math
    two_pi = 2.0 * math.pi
    if name == "isentropic_vortex":
        n = scale or 128
        c = make_config(2, KFVM_EQ_HYDRO, n, n, extent=(-5, 5, -5, 5), cfl=0.8,
                        steps=steps or 20)
        return c, KFVM_IC_ISENTROPIC_VORTEX
    if name == "sod3d":
        n = scale or 256
        c = make_config(3, KFVM_EQ_HYDRO, n, n, n, extent=(0, 1, 0, 1, 0, 1),
                        bc="outflow", cfl=0.8, steps=steps or 50)
        return c, KFVM_IC_SPHERICAL_SOD
    if name == "kelvin_helmholtz":
        n = scale or 1024
        c = make_config(2, KFVM_EQ_HYDRO, n, n, extent=(0, 1, 0, 1), cfl=0.8,
                        steps=steps or 500)
        return c, KFVM_IC_KELVIN_HELMHOLTZ
    if name == "taylor_green":
        n = scale or 256
        c = make_config(3, KFVM_EQ_NAVIERSTOKES, n, n, n,
                        extent=(0, two_pi, 0, two_pi, 0, two_pi), cfl=0.8,
                        reynolds=1600.0, prandtl=0.71, steps=steps or 200)
        return c, KFVM_IC_TAYLOR_GREEN
    if name == "orszag_tang":
        n = scale or 1024
        c = make_config(2, KFVM_EQ_MHD_GLM, n, n, extent=(0, 1, 0, 1),
                        gamma=5.0 / 3.0, rs=KFVM_RS_HLL, cfl=0.4, steps=steps or 1000)
        return c, KFVM_IC_ORSZAG_TANG
    # 3D GLM-MHD: the Orszag-Tang vortex extruded in z (exec/MHD/OrszagTang/orsztang3d.init)
    if name == "orszag_tang_3d":
        n = scale or 128
        c = make_config(3, KFVM_EQ_MHD_GLM, n, n, n, extent=(0, 1, 0, 1, 0, 1),
                        gamma=5.0 / 3.0, rs=KFVM_RS_HLL, cfl=0.4, steps=steps or 100)
        return c, KFVM_IC_ORSZAG_TANG
    # special-relativistic hydro (exec/SRHydro/SRShockTube, exec/SRHydro/SRRiem2d)
    if name == "sr_shock_tube":
        n = scale or 2000
        c = make_config(3, KFVM_EQ_SRHYDRO, n, 4, 4, extent=(0, 1, 0, 0.002, 0, 0.002),
                        bc=["outflow", "outflow", "periodic", "periodic", "periodic", "periodic"],
                        gamma=1.66666666666666, rs=KFVM_RS_HLL, cfl=1.25, steps=steps or 100,
                        atol=1e-3, rtol=1e-3)
        return c, KFVM_IC_SR_SHOCK_TUBE
    if name == "sr_riemann_2d":
        n = scale or 512
        c = make_config(2, KFVM_EQ_SRHYDRO, n, n, extent=(-1, 1, -1, 1), bc="outflow",
                        gamma=1.66666666666666, rs=KFVM_RS_LLF, cfl=1.0, steps=steps or 200,
                        atol=1e-3, rtol=1e-3)
        return c, KFVM_IC_SR_RIEMANN_2D
    # randomly forced turbulence (exec/Hydro/StirTurb/stirturb3d.init; forcing
    # parameters: eos:forceedot 60, forceratio 1, forcetoff 1.5)
    if name == "stir_turb":
        n = scale or 128
        c = make_config(3, KFVM_EQ_HYDRO, n, n, n, extent=(0, 1, 0, 1, 0, 1), gamma=1.001, rs=KFVM_RS_HLL,
                        cfl=1.25, weno_thresh=-1.0, steps=steps or 100, atol=1e-3, rtol=1e-3)
        return c, KFVM_IC_STIR_TURB
    raise ValueError(name)


def stir_turb_forcing(seed=1):
    """eos:forceedot 60, eos:forceratio 1, eos:forcetoff 1.5 of stirturb3d.init (stof-rounded)."""
    return KfvmForcing(stof(60.0), stof(1.0), stof(1.5), seed)


def nvars(cfg):
    return 9 if cfg.eq == KFVM_EQ_MHD_GLM else 5


def ncells(cfg):
    return cfg.nx * cfg.ny * (cfg.nz if cfg.dim == 3 else 1)
