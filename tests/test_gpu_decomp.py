"""Domain decomposition on the GPU: the blocks of a decomposed domain, each its own
solver on the device, against the one-domain solver.

Each block runs in its own host thread with its own stream; the exchange
callbacks (decomp.LocalExchange on device buffers) pack, copy and unpack the
halo cells and boundary face states between the blocks' device buffers, and
the step scalars are reduced across the blocks -- the path of
src/Solver.cpp:744-1460 with the transport of one process.  Kernels never wait
on another block's kernels; only the host threads meet at the exchange calls.

Bar: bit for bit.  Started from the matching part of the one-domain initial
state, with the one-domain step sizes imposed, every block's state after N
steps equals the one-domain state's cells, for the FP64 form and for the FP32
(3xTF32) form; the WENO cell counts summed over the blocks equal the one-domain
count.  (The learned indicator's judge samples cells by their block-local index,
so that form is not compared bit for bit.)
"""
import numpy as np
import pytest

import kfvm_abi as abi
from test_decomp import block_slice, blocks_of, workload

pytestmark = pytest.mark.gpu

CASES = [
    ("kelvin_helmholtz", 64, 4, (2, 2, 1), abi.KFVM_PREC_FP64),
    ("orszag_tang", 64, 4, (1, 2, 1), abi.KFVM_PREC_FP64),
    ("sod3d", 32, 3, (2, 1, 2), abi.KFVM_PREC_FP64),
    ("sod3d", 32, 3, (2, 1, 2), abi.KFVM_PREC_TF32X3),
    ("taylor_green", 32, 3, (2, 2, 2), abi.KFVM_PREC_FP64),
    ("orszag_tang_3d", 16, 2, (1, 2, 1), abi.KFVM_PREC_FP64),
    ("orszag_tang_3d_q3", 12, 2, (1, 2, 1), abi.KFVM_PREC_FP64),  # 81 rows: the row-pass reconstruction
]


@pytest.mark.parametrize("name,scale,steps,nb,prec", CASES)
def test_blocks_match_one_domain(name, scale, steps, nb, prec, gpu, product_lib):
    import torch

    import decomp
    kfvm = product_lib
    cfg, ic = workload(name, scale, steps)
    one = kfvm.Solver(cfg)
    one.set_precision(prec)
    one.init_ic(ic)
    u0 = one.get_state()
    dts, nweno = [], []
    for _ in range(steps):
        dts.append(one.time_dt())
        info = one.take_step()
        assert info.accepted == 1
        nweno.append(info.n_weno)
    ref = one.get_state()
    one.close()

    b = blocks_of(cfg, nb)
    nr = nb[0] * nb[1] * nb[2]
    hub = decomp.LocalExchange(nr, device=torch.device("cuda", 0), timeout=120)
    out = [None] * nr

    def block(r):
        def run():
            torch.cuda.set_device(0)
            c, nbr = kfvm.block_config(b, r)
            s = kfvm.Solver(c)
            try:
                s.set_precision(prec)
                s.set_exchange(hub.endpoint(r, nbr))
                s.set_state(block_slice(u0, cfg, c))
                nw = []
                for t, dt in dts:
                    s.set_time(t, dt)
                    info = s.take_step()
                    assert info.accepted == 1
                    nw.append(info.n_weno)
                out[r] = (c, s.get_state(), nw)
            finally:
                s.close()
        return run

    decomp.run_blocks([block(r) for r in range(nr)])
    for c, u, _ in out:
        want = block_slice(ref, cfg, c)
        assert np.array_equal(u, want), (list(c.block), np.abs(u - want).max())
    assert [sum(o[2][n] for o in out) for n in range(steps)] == nweno


def test_block_faces_hold_neighbour_states(gpu, product_lib):
    """After an evaluation the outer slot of an exchange face holds the neighbouring
    block's state at that face, as the one-domain face array does there."""
    import torch

    import decomp
    kfvm = product_lib
    cfg, ic = abi.workload("kelvin_helmholtz", scale=32, steps=1)
    one = kfvm.Solver(cfg)
    one.init_ic(ic)
    u0 = one.get_state()
    one.eval_rhs(0.0)
    fx = one.faces(0)                      # [2, nqf, nv, faces] of the x faces
    one.close()
    b = blocks_of(cfg, (2, 1, 1))
    hub = decomp.LocalExchange(2, device=torch.device("cuda", 0), timeout=120)
    got = [None, None]

    def block(r):
        def run():
            torch.cuda.set_device(0)
            c, nbr = kfvm.block_config(b, r)
            s = kfvm.Solver(c)
            try:
                s.set_exchange(hub.endpoint(r, nbr))
                s.set_state(block_slice(u0, cfg, c))
                s.eval_rhs(0.0)
                got[r] = (c, s.faces(0))
            finally:
                s.close()
        return run

    decomp.run_blocks([block(0), block(1)])
    nx = cfg.nx
    full = fx.reshape(fx.shape[0], fx.shape[1], fx.shape[2], cfg.ny, nx + 1)
    for c, f in got:
        f = f.reshape(f.shape[0], f.shape[1], f.shape[2], c.ny, c.nx + 1)
        x0 = c.block[0] * c.nx
        assert np.array_equal(f, full[..., x0:x0 + c.nx + 1])


def test_blocks_with_user_inflow(gpu, product_lib):
    """Exchange faces beside a user-supplied inflow face on the device: Sod 24^3
    in 2 x 1 x 2 blocks, the western face a fixed supersonic inflow, against the
    one-domain run with the same function, bit for bit."""
    import torch

    import decomp
    import userbc
    kfvm = product_lib
    cfg, ic = abi.workload("sod3d", scale=24, steps=3)
    cfg.bc[0] = abi.KFVM_BC_USER
    state = [1.5, 1.8, 0.0, 0.0, 1.5 / (cfg.gamma - 1.0) + 0.5 * 1.5 * 1.2 * 1.2]
    fn = userbc.inflow(state, 4, 5)
    one = kfvm.Solver(cfg)
    one.set_user_bc(fn)
    one.init_ic(ic)
    u0 = one.get_state()
    dts = []
    for _ in range(3):
        dts.append(one.time_dt())
        assert one.take_step().accepted == 1
    ref = one.get_state()
    one.close()
    b = blocks_of(cfg, (2, 1, 2))
    hub = decomp.LocalExchange(4, device=torch.device("cuda", 0), timeout=120)
    out = [None] * 4

    def block(r):
        def run():
            torch.cuda.set_device(0)
            c, nbr = kfvm.block_config(b, r)
            s = kfvm.Solver(c)
            try:
                s.set_exchange(hub.endpoint(r, nbr))
                if c.bc[0] == abi.KFVM_BC_USER:
                    s.set_user_bc(fn)
                s.set_state(block_slice(u0, cfg, c))
                for t, dt in dts:
                    s.set_time(t, dt)
                    assert s.take_step().accepted == 1
                out[r] = (c, s.get_state())
            finally:
                s.close()
        return run

    decomp.run_blocks([block(r) for r in range(4)])
    for c, u in out:
        want = block_slice(ref, cfg, c)
        assert np.array_equal(u, want), (list(c.block), np.abs(u - want).max())
