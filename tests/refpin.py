"""Shared helpers of the tests that compare with the reference's own run
(tests/golden/ref/*.npz, made by tests/golden/make_ref_fixtures.py from the
reference's sources compiled against oracle/refshim/)."""
import glob
import os

import numpy as np

import kfvm_abi as abi

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref")


def fixtures():
    return sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))


def load(path):
    z = np.load(path)
    return {k: z[k] for k in z.files}


def config(fx):
    """The configuration a fixture was made with (workload, grid, steps, indicator)."""
    cfg, ic = abi.workload(str(fx["workload"]), scale=int(fx["scale"]), steps=int(fx["steps"]))
    if "nq" in fx:
        cfg.nq = int(fx["nq"])
    for key in ("rk", "rs", "eq"):   # the Runge-Kutta scheme, Riemann solver, equations of the run
        if key in fx:
            setattr(cfg, key, int(fx[key]))
    for key in ("reynolds", "prandtl"):
        if key in fx:
            setattr(cfg, key, float(fx[key]))
    for f, w in enumerate(str(fx["walls"]) if "walls" in fx else ""):
        cfg.bc[f] = {"r": abi.KFVM_BC_REFLECTING, "n": abi.KFVM_BC_NOSLIP, "p": abi.KFVM_BC_PERIODIC,
                     "o": abi.KFVM_BC_OUTFLOW, "u": abi.KFVM_BC_USER}[w]
    th = float(fx["weno_thresh"])
    if not np.isnan(th):
        cfg.weno_thresh = abi.stof(th)
        cfg.indicator = abi.KFVM_IND_ALL if th < 0 else abi.KFVM_IND_KXRCF
    return cfg, ic


def install_user_bc(solver, fx, cfg):
    """The user boundary a fixture's reference build had (its hooks set a fixed
    inflow state rho, u, p on the faces marked u), as the same callback."""
    if "inflow" not in fx or len(fx["inflow"]) == 0:
        return
    import userbc
    rho, u, p = (float(x) for x in fx["inflow"])
    state = [rho, rho * u, 0.0, 0.0, p / (cfg.gamma - 1.0) + 0.5 * rho * u * u]
    nqf = cfg.nq * cfg.nq if cfg.dim == 3 else cfg.nq
    solver.set_user_bc(userbc.inflow(state, nqf, 5))


def replay(solver, fx):
    """Advance a solver (CUDA path or oracle) through the fixture's steps with the
    reference's step sizes imposed: step n starts at the reference's time and
    proposed step size after step n-1 (step 1 at t=0 with the size the reference
    took, t_1 - 0).  Returns per step (time, proposed dt) of the solver."""
    times, dts = fx["times"], fx["dts"]
    out = []
    for n in range(1, int(fx["steps"]) + 1):
        if n == 1:
            solver.set_time(0.0, float(times[1]))
        else:
            solver.set_time(float(times[n - 1]), float(dts[n - 1]))
        info = solver.take_step()
        assert info.accepted == 1, (n, info.status, info.attempts)
        out.append(solver.time_dt())
    return out


def rel_l1(a, b):
    """Relative L1 difference per variable.  A variable whose reference norm is
    below 1e-6 of the mean norm is measured against the mean norm: such a variable
    is analytically zero and made of rounding alone (the GLM scalar psi of a
    divergence-free field, z-momentum in 2D)."""
    den = np.abs(b).sum(axis=-1)
    mean = max(den.mean(), 1e-300)
    den = np.where(den < 1e-6 * mean, mean, den)
    return np.abs(a - b).sum(axis=-1) / den
