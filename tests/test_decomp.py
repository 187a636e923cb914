"""Domain decomposition on the CPU: the block layout of kfvm_block_config, and
the oracle's decomposed run against the one-domain run.

The reference splits the domain into one block per MPI rank
(src/LayoutMPI.H:44-97) and exchanges halo cells and boundary face states
between neighbouring blocks on every RHS evaluation (src/Solver.cpp:744-1460).
Decomposition must not change the answer: started from the matching part of the
one-domain initial state and with the step sizes of the one-domain run imposed
(the error sum is added in another order across ranks, so the controller's next
step size may differ in the last bit), every block's state after N steps equals
the matching part of the one-domain state bit for bit.  The initial condition of
a block is evaluated at the block's own cell centres, dx (i + 1/2) + xLo with
xLo = xLo_g + dx bxLo (src/Geometry.H:28-31, 50-57), which can round differently
from the one-domain centre dx (bxLo + i + 1/2) + xLo_g; it agrees to rounding,
and exactly where dx is a power of two.

The blocks run as threads of this process (decomp.LocalExchange) and, for the
transport of the multi-rank path, as gloo ranks in separate processes
(decomp.DistExchange).
"""
import datetime
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

import kfvm_abi as abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def blocks_of(cfg, nb):
    """The per-block configuration of a domain split into nb blocks."""
    b = abi.KfvmConfig.from_buffer_copy(cfg)
    for d in range(3):
        b.nb[d] = nb[d]
    b.nx //= nb[0]
    b.ny //= nb[1]
    if cfg.dim == 3:
        b.nz //= nb[2]
    return b


def block_slice(full, cfg, c):
    """The cells of block c in a one-domain state [nv, cells]."""
    nv = full.shape[0]
    gz = cfg.nz if cfg.dim == 3 else 1
    bz = c.nz if c.dim == 3 else 1
    u = full.reshape(nv, gz, cfg.ny, cfg.nx)
    z0, y0, x0 = c.block[2] * bz, c.block[1] * c.ny, c.block[0] * c.nx
    return u[:, z0:z0 + bz, y0:y0 + c.ny, x0:x0 + c.nx].reshape(nv, -1)


def workload(name, scale, steps):
    """abi.workload, plus the three-point variant of the 3D Orszag-Tang problem."""
    if name == "orszag_tang_3d_q3":
        cfg, ic = abi.workload("orszag_tang_3d", scale=scale, steps=steps)
        cfg.nq = 3
        return cfg, ic
    return abi.workload(name, scale=scale, steps=steps)


def one_domain(oracle, name, scale, steps, user=None):
    cfg, ic = workload(name, scale, steps)
    if user is not None:
        for f in user[0]:
            cfg.bc[f] = abi.KFVM_BC_USER
    s = oracle.OracleSolver(cfg)
    if user is not None:
        s.set_user_bc(user[1])
    s.init_ic(ic)
    u0 = s.get_state()
    dts = []
    for _ in range(steps):
        dts.append(s.time_dt())
        assert s.take_step().accepted == 1
    return cfg, ic, u0, dts, s.get_state()


# ------------------------------------------------------------------- block layout
def test_block_config_layout(product_lib):
    kfvm = product_lib
    cfg, _ = abi.workload("taylor_green", scale=16, steps=1)     # periodic on every face
    b = blocks_of(cfg, (2, 3, 2))
    seen = set()
    for r in range(12):
        c, nbr = kfvm.block_config(b, r)
        bx, by, bz = c.block[0], c.block[1], c.block[2]
        # MPI_Cart_coords' row-major order: z fastest
        assert r == (bx * 3 + by) * 2 + bz
        seen.add((bx, by, bz))
        assert list(c.nb) == [2, 3, 2]
        assert all(c.bc[f] == abi.KFVM_BC_EXCHANGE for f in range(6))
        # periodic wrap: MPI_Cart_shift with periods set
        assert nbr[0] == ((((bx - 1) % 2) * 3 + by) * 2 + bz)
        assert nbr[1] == ((((bx + 1) % 2) * 3 + by) * 2 + bz)
        assert nbr[2] == ((bx * 3 + (by - 1) % 3) * 2 + bz)
        assert nbr[3] == ((bx * 3 + (by + 1) % 3) * 2 + bz)
        assert nbr[4] == ((bx * 3 + by) * 2 + (bz - 1) % 2)
        assert nbr[5] == ((bx * 3 + by) * 2 + (bz + 1) % 2)
        assert (c.nx, c.ny, c.nz) == (b.nx, b.ny, b.nz)
    assert len(seen) == 12


def test_block_config_walls_and_errors(product_lib):
    kfvm = product_lib
    cfg, _ = abi.workload("sod3d", scale=16, steps=1)            # outflow on every face
    b = blocks_of(cfg, (2, 1, 1))
    c0, n0 = kfvm.block_config(b, 0)
    c1, n1 = kfvm.block_config(b, 1)
    assert n0 == [-1, 1, -1, -1, -1, -1] and n1 == [0, -1, -1, -1, -1, -1]
    assert c0.bc[0] == cfg.bc[0] and c0.bc[1] == abi.KFVM_BC_EXCHANGE
    assert c1.bc[0] == abi.KFVM_BC_EXCHANGE and c1.bc[1] == cfg.bc[1]
    assert all(c0.bc[f] == cfg.bc[f] for f in range(2, 6))
    with pytest.raises(kfvm.KfvmError):
        kfvm.block_config(b, 2)                                  # only two blocks
    k2, _ = abi.workload("kelvin_helmholtz", scale=16, steps=1)
    bad = blocks_of(k2, (1, 1, 1))
    bad.nb[2] = 2                                                # z blocks in 2D
    with pytest.raises(kfvm.KfvmError):
        kfvm.block_config(bad, 0)
    one, nbr = kfvm.block_config(blocks_of(k2, (1, 1, 1)), 0)    # one block: unchanged
    assert nbr == [-1] * 6 and list(one.bc) == list(k2.bc)


# --------------------------------------------------------- oracle, blocks as threads
THREAD_CASES = [
    ("kelvin_helmholtz", 32, 3, (2, 1, 1)),
    ("orszag_tang_3d_q3", 12, 2, (1, 2, 1)),    # 3D GLM-MHD with three Gauss points (81 rows)
    ("kelvin_helmholtz", 32, 3, (2, 2, 1)),      # corners: y halo over the exchanged x halo
    ("orszag_tang", 32, 3, (1, 2, 1)),           # GLM: cleaning speed and sources across blocks
    ("sod3d", 16, 2, (2, 1, 2)),                 # exchange faces beside outflow faces
    ("taylor_green", 16, 2, (2, 2, 2)),          # Navier-Stokes, periodic, eight blocks
    ("orszag_tang_3d", 12, 2, (1, 2, 1)),
]


@pytest.mark.parametrize("name,scale,steps,nb", THREAD_CASES)
def test_oracle_blocks_match_one_domain(name, scale, steps, nb, oracle_lib, product_lib):
    import decomp
    oracle_lib.set_threads(2)
    cfg, ic, u0, dts, ref = one_domain(oracle_lib, name, scale, steps)
    b = blocks_of(cfg, nb)
    nr = nb[0] * nb[1] * nb[2]
    hub = decomp.LocalExchange(nr, timeout=60)
    out = [None] * nr

    def block(r):
        def run():
            c, nbr = product_lib.block_config(b, r)
            s = oracle_lib.OracleSolver(c)
            s.set_exchange(hub.endpoint(r, nbr))
            s.set_state(block_slice(u0, cfg, c))
            for t, dt in dts:
                s.set_time(t, dt)
                assert s.take_step().accepted == 1
            out[r] = (c, s.get_state())
        return run

    decomp.run_blocks([block(r) for r in range(nr)])
    for c, u in out:
        assert np.array_equal(u, block_slice(ref, cfg, c)), (list(c.block), np.abs(u - block_slice(ref, cfg, c)).max())


@pytest.mark.parametrize("name,scale,nb,exact", [("kelvin_helmholtz", 32, (2, 2, 1), True),
                                                  ("kelvin_helmholtz", 24, (2, 1, 1), False),
                                                  ("taylor_green", 12, (1, 2, 2), False)])
def test_oracle_block_initial_condition(name, scale, nb, exact, oracle_lib, product_lib):
    """A block's initial condition at its own cell centres (and, for Kelvin-Helmholtz,
    with the noise of its cells' indices in the whole domain)."""
    cfg, ic = abi.workload(name, scale=scale, steps=1)
    full = oracle_lib.ic_cells(cfg, ic)
    b = blocks_of(cfg, nb)
    for r in range(nb[0] * nb[1] * nb[2]):
        c, _ = product_lib.block_config(b, r)
        u = oracle_lib.ic_cells(c, ic)
        ref = block_slice(full, cfg, c)
        if exact:
            assert np.array_equal(u, ref)
        else:
            scale_v = np.abs(full).max(axis=1, keepdims=True)
            assert np.all(np.abs(u - ref) <= 1e-14 * scale_v)


def test_oracle_blocks_with_user_inflow(oracle_lib, product_lib):
    """Exchange faces beside a user-supplied inflow face: Sod 16^3 in 2 x 1 x 2
    blocks, the western face a fixed supersonic inflow (a user function), against
    the one-domain run with the same function, bit for bit."""
    import decomp
    import userbc
    state = [1.5, 1.8, 0.0, 0.0, 1.5 / (1.4 - 1.0) + 0.5 * 1.5 * 1.2 * 1.2]
    fn = userbc.inflow(state, 4, 5)
    cfg, ic, u0, dts, ref = one_domain(oracle_lib, "sod3d", 16, 2, user=([0], fn))
    b = blocks_of(cfg, (2, 1, 2))
    hub = decomp.LocalExchange(4, timeout=60)
    out = [None] * 4

    def block(r):
        def run():
            c, nbr = product_lib.block_config(b, r)
            s = oracle_lib.OracleSolver(c)
            s.set_exchange(hub.endpoint(r, nbr))
            if c.bc[0] == abi.KFVM_BC_USER:
                s.set_user_bc(fn)
            s.set_state(block_slice(u0, cfg, c))
            for t, dt in dts:
                s.set_time(t, dt)
                assert s.take_step().accepted == 1
            out[r] = (c, s.get_state())
        return run

    decomp.run_blocks([block(r) for r in range(4)])
    for c, u in out:
        assert np.array_equal(u, block_slice(ref, cfg, c)), list(c.block)
    assert sum(1 for c, _ in out if c.bc[0] == abi.KFVM_BC_USER) == 2


def test_missing_transport_fails(oracle_lib, product_lib):
    """A block with exchange faces and no transport stops with an error instead of
    reading stale halo cells."""
    cfg, _ = abi.workload("kelvin_helmholtz", scale=16, steps=1)
    c, _ = product_lib.block_config(blocks_of(cfg, (2, 1, 1)), 0)
    s = oracle_lib.OracleSolver(c)
    # no set_exchange: the priming evaluation records the failure, the step reports it
    s.init_ic(abi.KFVM_IC_KELVIN_HELMHOLTZ)
    info = abi.KfvmStepInfo()
    assert oracle_lib.lib().orc_take_step(s.h, info) != 0


def test_broken_peer_fails_the_step(oracle_lib, product_lib):
    """A block whose peer never arrives (its thread exits before the first exchange)
    ends its step with an error once the barrier's time limit passes."""
    import decomp
    cfg, ic = abi.workload("kelvin_helmholtz", scale=16, steps=1)
    b = blocks_of(cfg, (2, 1, 1))
    hub = decomp.LocalExchange(2, timeout=2)
    c, nbr = product_lib.block_config(b, 0)
    s = oracle_lib.OracleSolver(c)
    ep = hub.endpoint(0, nbr)
    s.set_exchange(ep)
    s.init_ic(ic)                                # rank 1 never joins
    info = abi.KfvmStepInfo()
    assert oracle_lib.lib().orc_take_step(s.h, info) != 0
    assert ep.error is not None


# ------------------------------------------------------ oracle, gloo ranks over P2P
def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_rank(rank, world, port, name, scale, steps, nb, q):
    try:
        import torch.distributed as dist
        sys.path[:0] = [os.path.join(ROOT, "kfvm-kokkos_b200"), os.path.join(ROOT, "oracle")]
        import decomp
        import kfvm
        import oracle
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
        oracle.set_threads(1)
        cfg, ic, u0, dts, ref = one_domain(oracle, name, scale, steps)
        c, nbr = kfvm.block_config(blocks_of(cfg, nb), rank)
        s = oracle.OracleSolver(c)
        s.set_exchange(decomp.DistExchange(nbr))
        s.set_state(block_slice(u0, cfg, c))
        for t, dt in dts:
            s.set_time(t, dt)
            s.take_step()
        u = s.get_state()
        ok = bool(np.array_equal(u, block_slice(ref, cfg, c)))
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, ok, float(np.abs(u - block_slice(ref, cfg, c)).max())))
    except BaseException as e:  # noqa: BLE001
        q.put((rank, False, repr(e)))


@pytest.mark.parametrize("name,scale,steps,nb", [("kelvin_helmholtz", 24, 2, (2, 1, 1)),
                                                 ("orszag_tang", 16, 2, (2, 2, 1))])
def test_oracle_gloo_ranks_match_one_domain(name, scale, steps, nb, oracle_lib, product_lib):
    world = nb[0] * nb[1] * nb[2]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gloo_rank, args=(r, world, port, name, scale, steps, nb, q))
             for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ok, info in sorted(out):
        assert ok, (rank, info)
