"""kfvm_err_est_noalloc: the error estimate for callers that cannot call
cudaMalloc (their device memory belongs to another allocator, or their setting
forbids device allocation after start-up).  Its scratch is a fixed file-scope
device array; this test checks it against kfvm_err_est (which uses a solver's
allocated scratch) through the C ABI on two calls in a row, and the size limit.
The file sorts last so that a run stopping at the first failure has already run
every other test; it also passes alone in a fresh process."""
import numpy as np
import pytest

import kfvm_abi as abi

pytestmark = pytest.mark.gpu


def test_noalloc_matches_err_est(gpu, product_lib):
    import torch
    cfg, ic = abi.workload("sod3d", scale=32)
    s = product_lib.Solver(cfg)
    s.init_ic(ic)
    u = s.get_state()
    n = abi.ncells(cfg)
    rng = np.random.default_rng(11)
    du = torch.from_numpy(u).cuda()
    out = torch.full((2,), -7.0, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):  # two calls in a row, different inputs each time
        uh = u * (1.0 + (call + 1) * 1e-5 * rng.standard_normal(u.shape))
        duh = torch.from_numpy(uh).cuda()
        torch.cuda.synchronize()
        want_err, want_pos = s.err_est(du.data_ptr(), duh.data_ptr())
        product_lib.err_est_noalloc(cfg.eq, du.data_ptr(), duh.data_ptr(), n, cfg.atol, cfg.rtol,
                                    out.data_ptr(), stream)
        torch.cuda.synchronize()
        got_err, got_pos = out.cpu().tolist()
        assert abs(got_err - want_err) <= 1e-13 * abs(want_err), (call, got_err, want_err)
        assert abs(got_pos - want_pos) <= 1e-13 * abs(want_pos), (call, got_pos, want_pos)
    s.close()


def test_noalloc_rejects_oversize(gpu, product_lib):
    import torch
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    x = torch.ones(8, dtype=torch.float64, device="cuda")
    with pytest.raises(product_lib.KfvmError, match="capacity"):
        product_lib.err_est_noalloc(abi.KFVM_EQ_HYDRO, x.data_ptr(), x.data_ptr(),
                                    (1 << 24) + 1, 1e-4, 1e-4, out.data_ptr(), 0)
