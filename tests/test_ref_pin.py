"""The oracle against the reference's own code.

The fixtures in tests/golden/ref/ hold states from the reference solver itself
(its src/ compiled unchanged against the host stand-ins of oracle/refshim/,
run with a checkpoint after every step).  The oracle replays every case with
the reference's step sizes and must reproduce the reference bit for bit: the
state after every step (checked through per-variable sums, and in full after
the last step), the WENO flags and positivity theta, and the proposed next
step size.  Where the reference build itself is present (oracle/_ref, built
from the reference's sources by oracle/build_ref.py), small cases are also run
through it directly.
"""
import numpy as np
import pytest

import refpin

FIXTURES = refpin.fixtures()


def test_fixtures_present():
    names = {f.rsplit("/", 1)[-1] for f in FIXTURES}
    assert "vortex_128_c1.npz" in names and len(names) >= 6, names


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: p.rsplit("/", 1)[-1][:-4])
def test_oracle_matches_reference_bitwise(path, oracle_lib):
    fx = refpin.load(path)
    cfg, ic = refpin.config(fx)
    o = oracle_lib.OracleSolver(cfg)
    refpin.install_user_bc(o, fx, cfg)
    o.init_ic(ic)
    # the initial condition: the reference's first checkpoint
    u0 = o.get_state()
    np.testing.assert_array_equal(u0.sum(axis=1), fx["sums"][0])
    times, dts = fx["times"], fx["dts"]
    for n in range(1, int(fx["steps"]) + 1):
        o.set_time(0.0 if n == 1 else float(times[n - 1]), float(times[1]) if n == 1 else float(dts[n - 1]))
        info = o.take_step()
        assert info.accepted == 1
        u = o.get_state()
        np.testing.assert_array_equal(u.sum(axis=1), fx["sums"][n], err_msg=f"step {n}")
        np.testing.assert_array_equal(np.abs(u).sum(axis=1), fx["abs_sums"][n], err_msg=f"step {n}")
        t, dt = o.time_dt()
        assert t == times[n], (n, t, times[n])
        # the next step size comes from a sum over cells whose order follows
        # the thread partition of each side, so it is compared to rounding
        assert abs(dt - dts[n]) <= 1e-12 * abs(dts[n]), (n, dt, dts[n])
    np.testing.assert_array_equal(o.get_state(), fx["state"])
    a, th = o.flags()
    if not float(fx["weno_thresh"]) < 0:  # the full-WENO path leaves the flag view untouched
        np.testing.assert_array_equal(a.astype(bool), fx["flags"][0] > 0)
    np.testing.assert_array_equal(th, fx["flags"][1])


# direct runs of the reference build when it is present
DIRECT = [("kelvin_helmholtz", 24, 3), ("sod3d", 12, 2), ("orszag_tang", 24, 2), ("sr_riemann_2d", 24, 2)]


@pytest.mark.parametrize("name,scale,steps", DIRECT)
def test_oracle_matches_reference_build(name, scale, steps, oracle_lib):
    import refrun
    if refrun.binary(name) is None:
        pytest.skip("reference build absent (oracle/build_ref.py needs the reference sources)")
    import kfvm_abi as abi
    cfg, ic = abi.workload(name, scale=scale, steps=steps)
    cks, _ = refrun.run(name, cfg, steps, threads=4)
    o = oracle_lib.OracleSolver(cfg)
    o.init_ic(ic)
    np.testing.assert_array_equal(o.get_state(), cks[0][3])
    for n in range(1, steps + 1):
        o.set_time(cks[n - 1][1], cks[1][1] if n == 1 else cks[n - 1][2])
        o.take_step()
        np.testing.assert_array_equal(o.get_state(), cks[n][3])


def test_fixtures_cover_the_path():
    """Between them the reference's own runs cover every equation system, Riemann
    solver, Runge-Kutta scheme, Gauss-point count and boundary type of the path."""
    import kfvm_abi as abi
    eqs, rss, rks, nqs, bcs, dims = set(), set(), set(), set(), set(), set()
    for path in FIXTURES:
        cfg, _ = refpin.config(refpin.load(path))
        eqs.add(cfg.eq)
        rss.add(cfg.rs)
        rks.add(cfg.rk)
        nqs.add(cfg.nq)
        dims.add(cfg.dim)
        bcs.update(cfg.bc[f] for f in range(2 * cfg.dim))
    assert eqs == {abi.KFVM_EQ_HYDRO, abi.KFVM_EQ_NAVIERSTOKES, abi.KFVM_EQ_MHD_GLM, abi.KFVM_EQ_SRHYDRO}
    assert rss == {abi.KFVM_RS_LLF, abi.KFVM_RS_HLL, abi.KFVM_RS_HLLC}
    assert rks == {abi.KFVM_RK_THREESTARP, abi.KFVM_RK_FOURSTARP, abi.KFVM_RK_SSP4_3_2, abi.KFVM_RK_SSP10_4_3}
    assert nqs == {2, 3} and dims == {2, 3}
    assert bcs == {abi.KFVM_BC_PERIODIC, abi.KFVM_BC_OUTFLOW, abi.KFVM_BC_REFLECTING, abi.KFVM_BC_NOSLIP,
                   abi.KFVM_BC_USER}
