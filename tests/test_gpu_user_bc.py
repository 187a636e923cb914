"""User boundary conditions on the CUDA path (kfvm_set_user_bc, BCType::user of
src/BoundaryConditions_K.H:96-128, 569-615).

1. A user function that mirrors the built-in outflow / reflecting / no-slip faces
   reproduces the built-in CUDA run bit for bit (on the device, through CUDA
   tensors over the solver's packed buffers).
2. A supersonic inflow written by the user (a fixed state on the western face,
   the DoubleMach problem's inflow) against the oracle with the same function on
   host buffers: 1e-12 relative L1 after N steps with the oracle's step sizes,
   identical WENO cell counts.
"""
import numpy as np
import pytest

import kfvm_abi as abi
import userbc
from test_user_bc import CASES, built_in_and_user, nqf_of

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,scale,steps,faces", CASES)
def test_user_mirror_equals_built_in_gpu(name, scale, steps, faces, gpu, product_lib):
    cfg, ic = abi.workload(name, scale=scale, steps=steps)
    b, u = built_in_and_user(cfg, faces)
    gb = product_lib.Solver(b)
    gu = product_lib.Solver(u)
    gu.set_user_bc(userbc.mirror_wall(list(b.bc), abi.nvars(cfg), nqf_of(cfg)))
    gb.init_ic(ic)
    gu.init_ic(ic)
    for _ in range(steps):
        ib, iu = gb.take_step(), gu.take_step()
        assert (ib.accepted, ib.n_weno) == (iu.accepted, iu.n_weno)
        assert ib.dt == iu.dt
    assert np.array_equal(gb.get_state(), gu.get_state())
    gb.close()
    gu.close()


def test_user_inflow_against_oracle(gpu, product_lib, oracle_lib):
    cfg, ic = abi.workload("sod3d", scale=24, steps=4)
    cfg.bc[0] = abi.KFVM_BC_USER
    g, o = product_lib.Solver(cfg), oracle_lib.OracleSolver(cfg)
    gamma = cfg.gamma
    rho, u, p = 1.5, 1.2, 1.5
    state = [rho, rho * u, 0.0, 0.0, p / (gamma - 1.0) + 0.5 * rho * u * u]
    g.set_user_bc(userbc.inflow(state, nqf_of(cfg), 5))
    o.set_user_bc(userbc.inflow(state, nqf_of(cfg), 5))
    g.init_ic(ic)
    o.init_ic(ic)
    for n in range(4):
        t, dt = o.time_dt()
        g.set_time(t, dt)
        ig, io = g.take_step(), o.take_step()
        assert ig.accepted == io.accepted == 1
        assert ig.n_weno == io.n_weno, (n, ig.n_weno, io.n_weno)
    ug, uo = g.get_state(), o.get_state()
    err = np.abs(ug - uo).sum(axis=1) / np.maximum(np.abs(uo).sum(axis=1), 1e-300)
    assert np.all(err <= 1e-12), err
    # mass entered through the western face
    assert ug[0].sum() > oracle_lib.ic_cells(cfg, ic)[0].sum()
    g.close()
