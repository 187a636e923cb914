"""Regenerate tests/golden/ref/*.npz: states from the reference's own run.

Builds the reference solver from its sources (oracle/build_ref.py: the
reference's src/ compiled unchanged against the host stand-ins of
oracle/refshim/), runs each case below with a checkpoint after every step, and
stores per case: the configuration (workload, grid, steps, indicator), the time
and proposed step size after every step, the WENO cell count of every step, the
per-variable sums of the state after every step, and the final state and WENO
flags in full.  The tests replay the same steps in the oracle and in the CUDA
path with the reference's step sizes imposed and compare with these states.

Usage: python tests/golden/make_ref_fixtures.py <path of the reference checkout>
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (os.path.join(ROOT, "oracle"), os.path.join(ROOT, "kfvm-kokkos_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

import build_ref  # noqa: E402
import kfvm_abi as abi  # noqa: E402
import refrun  # noqa: E402

# (case, workload, grid per axis, accepted steps, wenothresh override or None,
#  Gauss points, reference problem build[, wall codes[, configuration overrides]])
CASES = [
    ("vortex_128_c1", "isentropic_vortex", 128, 20, None, 2, None),   # the problem list's C1, as stated
    ("sod3d_24", "sod3d", 24, 5, None, 2, None),
    ("sod3d_16_fullweno", "sod3d", 16, 3, -1.0, 2, None),             # wenothresh < 0: WENO everywhere
    ("kelvin_helmholtz_64", "kelvin_helmholtz", 64, 10, None, 2, None),
    ("taylor_green_16", "taylor_green", 16, 4, None, 2, None),
    ("orszag_tang_64", "orszag_tang", 64, 10, None, 2, None),
    ("orszag_tang_3d_16", "orszag_tang_3d", 16, 3, None, 2, None),   # 3D GLM-MHD sources at Q^3 points
    ("orszag_tang_3d_q3_12", "orszag_tang_3d", 12, 2, None, 3, "orszag_tang_3d_q3"),  # three points
    ("sr_riemann_2d_32", "sr_riemann_2d", 32, 4, None, 2, None),      # special-relativistic hydro
    # walls (codes west east south north bottom top: r reflecting, n no-slip, p periodic)
    ("sod3d_reflecting_16", "sod3d", 16, 3, None, 2, "sod3d_reflecting", "rrrrrr"),
    ("taylor_green_noslip_12", "taylor_green", 12, 3, None, 2, "taylor_green_noslip", "ppnnpp"),
    # the other schemes and solvers (Runge-Kutta and Riemann overrides), three points in 2D
    ("sod3d_ssp10_16", "sod3d", 16, 3, None, 2, "sod3d_ssp10", "", {"rk": abi.KFVM_RK_SSP10_4_3}),
    ("vortex_threestar_32", "isentropic_vortex", 32, 4, None, 2, "vortex_threestar", "",
     {"rk": abi.KFVM_RK_THREESTARP}),
    # (on the vortex at 32^2 the embedded error of SSP(10,4) and FourStarP sits near
    # the rounding floor, so their step-size proposals are noise; the blast's are not)
    ("sod3d_fourstar_16", "sod3d", 16, 3, None, 2, "sod3d_fourstar", "", {"rk": abi.KFVM_RK_FOURSTARP}),
    ("kelvin_helmholtz_hll_32", "kelvin_helmholtz", 32, 5, None, 2, "kelvin_helmholtz_hll", "",
     {"rs": abi.KFVM_RS_HLL}),
    ("kelvin_helmholtz_q3_32", "kelvin_helmholtz", 32, 5, None, 3, "kelvin_helmholtz_q3"),
    ("sod3d_llf_16", "sod3d", 16, 3, None, 2, "sod3d_llf", "", {"rs": abi.KFVM_RS_LLF}),
    ("orszag_tang_llf_32", "orszag_tang", 32, 5, None, 2, "orszag_tang_llf", "", {"rs": abi.KFVM_RS_LLF}),
    # three points in 3D (54 rows): the blast puts the WENO and limiter paths under test
    ("sod3d_q3_12", "sod3d", 12, 2, None, 3, "sod3d_q3"),
    ("taylor_green_q3_10", "taylor_green", 10, 2, None, 3, "taylor_green_q3"),
    # a user boundary (u): the western inflow of oracle/build_ref.py's sod3d_inflow
    ("sod3d_inflow_16", "sod3d", 16, 3, None, 2, "sod3d_inflow", "uooooo"),
    ("kelvin_helmholtz_reflect_32", "kelvin_helmholtz", 32, 4, None, 2, "kelvin_helmholtz_reflect", "pprrpp"),
    ("orszag_tang_reflect_32", "orszag_tang", 32, 4, None, 2, "orszag_tang_reflect", "pprrpp"),
    ("sr_shock_tube_64", "sr_shock_tube", 64, 3, None, 2, None),       # 64 x 4 x 4, HLL
    ("kelvin_helmholtz_ns_32", "kelvin_helmholtz", 32, 4, None, 2, "kelvin_helmholtz_ns", "",
     {"eq": abi.KFVM_EQ_NAVIERSTOKES, "reynolds": abi.stof(1000.0), "prandtl": abi.stof(0.71)}),
    ("sod3d_noslip_16", "sod3d", 16, 3, None, 2, "sod3d_noslip", "nnnnnn"),
    ("taylor_green_reflect_12", "taylor_green", 12, 3, None, 2, "taylor_green_reflect", "rrpppp"),
    ("orszag_tang_3d_reflect_16", "orszag_tang_3d", 16, 2, None, 2, "orszag_tang_3d_reflect", "pppprr"),
]
WALLS = {"r": abi.KFVM_BC_REFLECTING, "n": abi.KFVM_BC_NOSLIP, "p": abi.KFVM_BC_PERIODIC,
         "o": abi.KFVM_BC_OUTFLOW, "u": abi.KFVM_BC_USER}
# the state the user boundary of the sod3d_inflow build sets (rho 1.5, u 1.2, p 1.5)
INFLOW = {"sod3d_inflow": (1.5, 1.2, 1.5)}


def case_config(workload, scale, steps, thresh, nq=2, walls="", over=None):
    cfg, ic = abi.workload(workload, scale=scale, steps=steps)
    for key, val in (over or {}).items():   # Runge-Kutta scheme, Riemann solver
        setattr(cfg, key, val)
    if thresh is not None:
        cfg.weno_thresh = abi.stof(thresh)
        cfg.indicator = abi.KFVM_IND_ALL if thresh < 0 else abi.KFVM_IND_KXRCF
    cfg.nq = nq
    for f, w in enumerate(walls):
        cfg.bc[f] = WALLS[w]
    return cfg, ic


def main():
    if len(sys.argv) < 2:
        sys.exit("usage: make_ref_fixtures.py <path of the reference checkout> [case ...]")
    cases = [c for c in CASES if len(sys.argv) == 2 or c[0] in sys.argv[2:]]
    build_ref.build_all(sys.argv[1], sorted({c[6] or c[1] for c in cases}))
    out = os.path.join(HERE, "ref")
    os.makedirs(out, exist_ok=True)
    for case, workload, scale, steps, thresh, nq, problem, *extra in cases:
        walls = extra[0] if extra else ""
        over = extra[1] if len(extra) > 1 else {}
        cfg, ic = case_config(workload, scale, steps, thresh, nq, walls, over)
        cks, _ = refrun.run(problem or workload, cfg, steps)
        inflow = INFLOW.get(problem, ())
        assert len(cks) == steps + 1, (case, len(cks))
        np.savez_compressed(
            os.path.join(out, case + ".npz"),
            workload=workload, scale=scale, steps=steps, nq=nq, walls=walls, rk=cfg.rk, rs=cfg.rs,
            eq=cfg.eq, reynolds=cfg.reynolds, prandtl=cfg.prandtl,
            inflow=np.array(inflow, dtype=np.float64),
            weno_thresh=np.nan if thresh is None else thresh,
            times=np.array([c[1] for c in cks]), dts=np.array([c[2] for c in cks]),
            weno_counts=np.array([int((c[4][0] > 0).sum()) for c in cks]),
            sums=np.array([c[3].sum(axis=1) for c in cks]),
            abs_sums=np.array([np.abs(c[3]).sum(axis=1) for c in cks]),
            state=cks[-1][3], flags=cks[-1][4])
        print(case, "steps", steps, "weno cells last", int((cks[-1][4][0] > 0).sum()))


if __name__ == "__main__":
    main()
