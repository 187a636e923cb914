"""The CUDA path (through the C ABI) against the reference's own run.

Each fixture in tests/golden/ref/ holds the state after N accepted steps of the
reference solver itself (its src/ compiled unchanged for the CPU against the
stand-ins of oracle/refshim/).  The CUDA path replays the case with the
reference's step sizes imposed and must agree to 1e-12 relative L1 per
conserved variable (the FP64 parity bar); its WENO flags must equal the
reference's and its positivity theta agree to 1e-12.  The first case is the
problem list's C1 exactly as stated: the 128^2 isentropic vortex, 20 steps.
"""
import numpy as np
import pytest

import refpin

pytestmark = pytest.mark.gpu

STEP_TOL = 1e-12


@pytest.mark.parametrize("path", refpin.fixtures(), ids=lambda p: p.rsplit("/", 1)[-1][:-4])
def test_cuda_path_matches_reference(path, gpu, product_lib):
    fx = refpin.load(path)
    cfg, ic = refpin.config(fx)
    g = product_lib.Solver(cfg)
    g.init_ic(ic)
    err0 = refpin.rel_l1(g.get_state().sum(axis=1, keepdims=True), fx["sums"][0][:, None])
    assert np.all(err0 <= 1e-14), err0
    props = refpin.replay(g, fx)
    err = refpin.rel_l1(g.get_state(), fx["state"])
    assert np.all(err <= STEP_TOL), err
    for n, (t, dt) in enumerate(props, start=1):
        assert abs(t - fx["times"][n]) <= 1e-14 * abs(fx["times"][n])
        assert abs(dt - fx["dts"][n]) <= 1e-7 * abs(fx["dts"][n]), (n, dt, fx["dts"][n])
    a, th = g.flags()
    if not float(fx["weno_thresh"]) < 0:  # the full-WENO path leaves the flag view untouched
        np.testing.assert_array_equal(a.astype(bool), fx["flags"][0] > 0)
    assert np.abs(th - fx["flags"][1]).max() <= 1e-12
    g.close()
