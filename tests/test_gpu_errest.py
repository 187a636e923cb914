"""kfvm_err_est (RKFSAL_ErrEst_K, src/numeric/Numeric_K.H:262-290) against a numpy
evaluation of the same formula on the same device arrays."""
import numpy as np
import pytest

import kfvm_abi as abi

pytestmark = pytest.mark.gpu


def reference(u, uh, atol, rtol, glm):
    e = (u - uh) / (atol + rtol * np.maximum(np.abs(u), np.abs(uh)))
    err = float((e * e).sum())
    ek = 0.5 * (u[1] ** 2 + u[2] ** 2 + u[3] ** 2) / u[0]
    eint = u[4] - ek
    if glm:
        eint = u[4] - 0.5 * (u[5] ** 2 + u[6] ** 2 + u[7] ** 2) - ek - 0.5 * u[8] ** 2
    pos = np.minimum(u[0], eint)
    pos = np.where(np.isnan(u).any(axis=0), -1.0, pos)
    return err, float(min(1.0, pos.min()))


@pytest.mark.parametrize("name,scale", [("kelvin_helmholtz", 48), ("orszag_tang", 40), ("sod3d", 20)])
def test_err_est_matches_formula(name, scale, gpu, product_lib):
    import torch
    cfg, ic = abi.workload(name, scale=scale)
    s = product_lib.Solver(cfg)
    s.init_ic(ic)
    u = s.get_state()
    rng = np.random.default_rng(7)
    uh = u * (1.0 + 1e-5 * rng.standard_normal(u.shape))
    du, duh = torch.from_numpy(u).cuda(), torch.from_numpy(uh).cuda()
    torch.cuda.synchronize()
    err, pos = s.err_est(du.data_ptr(), duh.data_ptr())
    rerr, rpos = reference(u, uh, cfg.atol, cfg.rtol, cfg.eq == abi.KFVM_EQ_MHD_GLM)
    assert abs(err - rerr) <= 1e-12 * rerr
    assert abs(pos - rpos) <= 1e-14 * abs(rpos)
    # a NaN anywhere makes the positivity flag negative
    u2 = u.copy()
    u2[2, 5] = np.nan
    du2 = torch.from_numpy(u2).cuda()
    torch.cuda.synchronize()
    _, pos2 = s.err_est(du2.data_ptr(), duh.data_ptr())
    assert pos2 == -1.0
    s.close()
