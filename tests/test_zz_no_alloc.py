"""kfvm_err_est_noalloc: the error estimate for callers that cannot call
cudaMalloc (their device memory belongs to another allocator, or their setting
forbids device allocation after start-up).  Its scratch is a fixed file-scope
device array; this test checks it through the C ABI against kfvm_err_est (which
uses a solver's allocated scratch) on two calls in a row, for every equation
family, on grids whose cell count is and is not a multiple of the 256-cell
reduction block, and against the numpy formula at exactly the array's capacity;
and it checks the size limit.  The file sorts last so that a run stopping at the
first failure has already run every other test; it also passes alone in a fresh
process."""
import numpy as np
import pytest

import kfvm_abi as abi

pytestmark = pytest.mark.gpu

CASES = [
    # (workload or config, grid): 32^3 = 32768 cells (whole blocks), 33 x 31 = 1023 (a partial block)
    ("sod3d", 32, None),
    ("orszag_tang", (33, 31), abi.KFVM_EQ_MHD_GLM),
    ("sr_riemann_2d", (33, 31), abi.KFVM_EQ_SRHYDRO),
    ("kelvin_helmholtz", (33, 31), abi.KFVM_EQ_HYDRO),
]


def _config(name, grid):
    if isinstance(grid, tuple):
        cfg, ic = abi.workload(name, scale=grid[0])
        cfg.nx, cfg.ny = grid
        return cfg, ic
    return abi.workload(name, scale=grid)


@pytest.mark.parametrize("name,grid,eq", CASES, ids=[c[0] for c in CASES])
def test_noalloc_matches_err_est(name, grid, eq, gpu, product_lib):
    import torch
    cfg, ic = _config(name, grid)
    s = product_lib.Solver(cfg)
    s.init_ic(ic)
    u = s.get_state()
    n = abi.ncells(cfg)
    assert (n % 256 == 0) == (not isinstance(grid, tuple))
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


def test_noalloc_at_capacity(gpu, product_lib):
    """n = KFVM_NOALLOC_MAX_CELLS (2^24 cells, every slot of the fixed array used)
    against the numpy formula of the error estimate."""
    import torch
    n, atol, rtol = 1 << 24, 1e-4, 1e-4
    g = torch.Generator(device="cuda").manual_seed(3)
    u = torch.empty((5, n), dtype=torch.float64, device="cuda")
    u[0].uniform_(0.5, 2.0, generator=g)
    u[1:4].uniform_(-0.5, 0.5, generator=g)
    u[4] = 3.0 + 0.5 * (u[1] ** 2 + u[2] ** 2 + u[3] ** 2) / u[0]
    uh = u * (1.0 + 1e-5 * torch.randn(u.shape, dtype=torch.float64, device="cuda", generator=g))
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    product_lib.err_est_noalloc(abi.KFVM_EQ_HYDRO, u.data_ptr(), uh.data_ptr(), n, atol, rtol, out.data_ptr(),
                                torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    e = (u - uh) / (atol + rtol * torch.maximum(u.abs(), uh.abs()))
    want_err = float((e * e).sum())
    ek = 0.5 * (u[1] ** 2 + u[2] ** 2 + u[3] ** 2) / u[0]
    want_pos = float(min(1.0, float(torch.minimum(u[0], u[4] - ek).min())))
    got_err, got_pos = out.cpu().tolist()
    assert abs(got_err - want_err) <= 1e-12 * want_err, (got_err, want_err)
    assert abs(got_pos - want_pos) <= 1e-14 * abs(want_pos), (got_pos, want_pos)


def test_noalloc_rejects_oversize(gpu, product_lib):
    import torch
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    x = torch.ones(8, dtype=torch.float64, device="cuda")
    with pytest.raises(product_lib.KfvmError, match="capacity"):
        product_lib.err_est_noalloc(abi.KFVM_EQ_HYDRO, x.data_ptr(), x.data_ptr(),
                                    (1 << 24) + 1, 1e-4, 1e-4, out.data_ptr(), 0)
