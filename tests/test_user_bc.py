"""User boundary conditions (BCType::user: a problem's UserBCs.H,
src/BoundaryConditions_K.H:96-128, 569-615) on the oracle, CPU.

1. A user function that mirrors the built-in outflow / reflecting / no-slip
   faces reproduces the built-in run bit for bit: the packed layouts, the layer
   order and the call order are the ones kfvm_set_user_bc states.
2. The callback sees the stage times of the RK scheme (t + c dt) and is called per
   user face for cells and face states, in setCellBCs' axis order.
3. A failing callback fails the step.
"""
import numpy as np
import pytest

import kfvm_abi as abi
import userbc

CASES = [
    ("sod3d", 16, 3, {0: abi.KFVM_BC_OUTFLOW, 3: abi.KFVM_BC_OUTFLOW, 5: abi.KFVM_BC_OUTFLOW}),
    ("kelvin_helmholtz", 32, 3, {2: abi.KFVM_BC_REFLECTING, 3: abi.KFVM_BC_REFLECTING}),
    ("orszag_tang", 32, 3, {0: abi.KFVM_BC_REFLECTING, 1: abi.KFVM_BC_REFLECTING}),
    ("taylor_green", 12, 2, {2: abi.KFVM_BC_NOSLIP, 3: abi.KFVM_BC_NOSLIP}),
]


def nqf_of(cfg):
    return cfg.nq if cfg.dim == 2 else cfg.nq * cfg.nq


def built_in_and_user(cfg, faces):
    """(configuration with the built-in walls, configuration with user faces)."""
    b = abi.KfvmConfig.from_buffer_copy(cfg)
    u = abi.KfvmConfig.from_buffer_copy(cfg)
    for f, t in faces.items():
        b.bc[f] = t
        u.bc[f] = abi.KFVM_BC_USER
    return b, u


@pytest.mark.parametrize("name,scale,steps,faces", CASES)
def test_user_mirror_equals_built_in(name, scale, steps, faces, oracle_lib):
    cfg, ic = abi.workload(name, scale=scale, steps=steps)
    b, u = built_in_and_user(cfg, faces)
    ob = oracle_lib.OracleSolver(b)
    ou = oracle_lib.OracleSolver(u)
    ou.set_user_bc(userbc.mirror_wall(list(b.bc), abi.nvars(cfg), nqf_of(cfg)))
    ob.init_ic(ic)
    ou.init_ic(ic)
    for _ in range(steps):
        # the same step size on both (the oracle's error sum is an OpenMP reduction,
        # whose combining order, and so the last bit of the next step size, can vary)
        t, dt = ob.time_dt()
        ou.set_time(t, dt)
        ib, iu = ob.take_step(), ou.take_step()
        assert (ib.accepted, ib.n_weno) == (iu.accepted, iu.n_weno)
        assert abs(ib.dt - iu.dt) <= 1e-14 * ib.dt
    assert np.array_equal(ob.get_state(), ou.get_state())


def test_user_callback_times_and_order(oracle_lib):
    cfg, ic = abi.workload("sod3d", scale=12, steps=1)
    b, u = built_in_and_user(cfg, {1: abi.KFVM_BC_OUTFLOW, 4: abi.KFVM_BC_OUTFLOW})
    log = []
    o = oracle_lib.OracleSolver(u)
    o.set_user_bc(userbc.mirror_wall(list(b.bc), 5, 4, log))
    o.init_ic(ic)
    # the priming evaluation at t = 0: cells of face 1 (x) before face 4 (z), then
    # the face states after the linear reconstruction and after the limiter
    assert log == [(0, 1, 0.0), (0, 4, 0.0), (1, 1, 0.0), (1, 4, 0.0), (1, 1, 0.0), (1, 4, 0.0)]
    t0, dt = o.time_dt()
    del log[:]
    o.take_step()
    _, _, rk = oracle_lib.tables(cfg.nq, cfg.rk)
    want = [t0 + c * dt for c in rk["c"][1:]] + [t0 + dt]
    seen = sorted({t for k, f, t in log})
    assert np.allclose(seen, sorted(set(want)), rtol=0, atol=1e-15), (seen, want)


def test_user_callback_failure_fails_the_step(oracle_lib):
    cfg, ic = abi.workload("sod3d", scale=12, steps=1)
    _, u = built_in_and_user(cfg, {0: abi.KFVM_BC_OUTFLOW})
    o = oracle_lib.OracleSolver(u)

    def bad(kind, face, time, inner, outer):
        raise RuntimeError("no inflow data")

    o.set_user_bc(bad)
    o.init_ic(ic)
    info = abi.KfvmStepInfo()
    assert oracle_lib.lib().orc_take_step(o.h, info) != 0
    assert isinstance(o.user_bc_error, RuntimeError)
