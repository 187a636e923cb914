"""The FP32 form (KFVM_PREC_TF32X3): the linear reconstruction's stencil sums on
the tcgen05 tensor cores (3xTF32 products, FP32 accumulation in tensor memory).

It is checked against the FP64 path of the same library on the same state:
face states to FP32-split accuracy for every dimension x equation set (each
instantiation has its own tensor-memory width), and, as the accuracy bar that
matters, the L1 error against the exact solution of the isentropic vortex after
one period: the FP32 form's error must stay within 1.05x of the plain FP64 run.
"""
import math

import numpy as np
import pytest

import kfvm_abi as abi

pytestmark = pytest.mark.gpu

# max |F_tf32 - F_fp64| per variable over max |F_fp64| of that variable (floored at
# 1e-3 of the largest variable): the stencil sum carries ~21 bits per product
FACE_TOL = 4e-6
L1_RATIO = 1.05   # FP32-form L1 error vs the plain FP64 form's, same grid and steps


def _solver(cfg, ic, prec):
    import kfvm
    s = kfvm.Solver(cfg)
    s.set_precision(prec)
    s.init_ic(ic)
    return s


def _cfg3_glm(n):
    return abi.make_config(3, abi.KFVM_EQ_MHD_GLM, n, n, n, extent=(0, 1, 0, 1, 0, 1),
                           gamma=5.0 / 3.0, rs=abi.KFVM_RS_HLL, cfl=0.4, steps=4)


def _cfg2_ns(n):
    return abi.make_config(2, abi.KFVM_EQ_NAVIERSTOKES, n, n, extent=(-5, 5, -5, 5),
                           reynolds=100.0, steps=4)


CASES = [
    ("vortex 2D Euler", lambda: abi.workload("isentropic_vortex", scale=64, steps=4)),
    ("KH 2D Euler", lambda: abi.workload("kelvin_helmholtz", scale=64, steps=4)),
    ("vortex 2D NS", lambda: (_cfg2_ns(48), abi.KFVM_IC_ISENTROPIC_VORTEX)),
    ("OT 2D GLM", lambda: abi.workload("orszag_tang", scale=64, steps=4)),
    ("Sod 3D Euler", lambda: abi.workload("sod3d", scale=24, steps=4)),
    ("TGV 3D NS", lambda: abi.workload("taylor_green", scale=20, steps=4)),
    ("OT 3D GLM", lambda: (_cfg3_glm(16), abi.KFVM_IC_ORSZAG_TANG)),
]


@pytest.mark.parametrize("name,mk", CASES, ids=[c[0] for c in CASES])
def test_tc_faces_match_fp64(name, mk, product_lib, gpu):
    cfg, ic = mk()
    ref = _solver(cfg, ic, abi.KFVM_PREC_FP64)
    tc = _solver(cfg, ic, abi.KFVM_PREC_TF32X3)
    ref.set_indicator(abi.KFVM_IND_NONE)   # every cell linear: the whole grid goes through the MMA
    tc.set_indicator(abi.KFVM_IND_NONE)
    r_ref, mv_ref = ref.eval_rhs()
    r_tc, mv_tc = tc.eval_rhs()
    for d in range(cfg.dim):
        fr, ft = ref.faces(d), tc.faces(d)
        assert np.isfinite(ft).all(), (name, d)
        scale = np.abs(fr).max(axis=(0, 1, 3))
        scale = np.maximum(scale, 1e-3 * scale.max())
        err = np.abs(ft - fr).max(axis=(0, 1, 3)) / scale
        assert err.max() <= FACE_TOL, (name, d, err)
        # not bit-identical: the tensor-core path really ran
        assert np.abs(ft - fr).max() > 0.0, (name, d)
    assert abs(mv_tc - mv_ref) <= 1e-5 * mv_ref, (name, mv_tc, mv_ref)
    num = np.abs(r_tc - r_ref).sum(axis=1)
    tot = np.abs(r_ref).sum(axis=1)
    den = np.maximum(tot, 1e-8 * tot.mean() + 1e-300)
    assert (num / den).max() <= 1e-3, (name, num / den)
    ref.close()
    tc.close()


def test_tc_kxrcf_steps_close(product_lib, gpu):
    """With the KXRCF selector on (Sod blast: flagged cells go to the FP64 WENO), a
    few steps of the FP32 form stay close to the FP64 run."""
    cfg, ic = abi.workload("sod3d", scale=32, steps=3)
    a = _solver(cfg, ic, abi.KFVM_PREC_FP64)
    b = _solver(cfg, ic, abi.KFVM_PREC_TF32X3)
    for _ in range(3):
        ia, ib = a.take_step(), b.take_step()
        assert ia.accepted == ib.accepted == 1
        assert abs(ia.n_weno - ib.n_weno) <= max(2, 0.01 * ia.n_weno), (ia.n_weno, ib.n_weno)
    ua, ub = a.get_state(), b.get_state()
    rel = np.abs(ub - ua).sum(axis=1) / np.maximum(np.abs(ua).sum(axis=1), 1e-300)
    assert rel[[0, 4]].max() <= 1e-5, rel
    a.close()
    b.close()


def _vortex_period_error(n, prec):
    cfg, ic = abi.workload("isentropic_vortex", scale=n, steps=100000)
    cfg.final_time = abi.stof(10.0)       # velocity (1,1) on a 10 x 10 periodic box
    s = _solver(cfg, ic, prec)
    exact = s.get_state().copy()          # cell averages of the initial condition
    nsteps, info = s.solve(cfg.max_steps)
    t, _ = s.time_dt()
    assert abs(t - 10.0) < 1e-9, t
    u = s.get_state()
    s.close()
    return np.abs(u - exact).sum(axis=1) * (10.0 / n) ** 2, nsteps


@pytest.mark.parametrize("n", [64, 128])
def test_tc_vortex_l1_vs_exact(n, product_lib, gpu):
    e64, n64 = _vortex_period_error(n, abi.KFVM_PREC_FP64)
    e32, n32 = _vortex_period_error(n, abi.KFVM_PREC_TF32X3)
    assert n64 > 50 and abs(n32 - n64) <= 2, (n64, n32)
    for v in (0, 1, 2, 4):
        assert e32[v] <= L1_RATIO * e64[v], (n, v, e32, e64)
    assert math.isfinite(e32.sum())


def test_tc_precision_argument(product_lib, gpu):
    import kfvm
    cfg, ic = abi.workload("isentropic_vortex", scale=16, steps=1)
    s = kfvm.Solver(cfg)
    with pytest.raises(kfvm.KfvmError):
        s.set_precision(7)
    s.set_precision(abi.KFVM_PREC_TF32X3)
    s.set_precision(abi.KFVM_PREC_FP64)
    s.close()
