"""Random forcing of the stirred-turbulence problems (ENABLE_RANDOM_FORCING:
src/ParameterStructs.H:45-73, src/ParameterStructs.cpp:41-88,
src/physics/Common_K.H:645-784, src/Solver.cpp:99-103, 365-409).

CPU: the mode table (band, order, amplitude law), the oracle's kick (it injects
exactly edot dt of energy and no net momentum) and the driver keys.  GPU: the
device integrals, strength and kick against the oracle with the same mode table,
and forced steps."""
import json
import os
import subprocess

import numpy as np
import pytest

import kfvm_abi as abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RUN = os.path.join(ROOT, "kfvm-kokkos_b200", "kfvm_run")


def band(dim):
    """The reference's wavevector loop (ParameterStructs.H:50-71), written out."""
    out = []
    kz = range(-3, 4) if dim == 3 else [0]
    for i in range(0, 4):
        for j in range(-3, 4):
            for k in kz:
                ksq = i * i + j * j + k * k
                if ksq == 0 or ksq > 9 or (i == 0 and (j < 0 or k < 0)):
                    continue
                out.append((i, j, k)[:dim])
    return out


@pytest.mark.parametrize("dim,n", [(2, 14), (3, 57)])
def test_mode_table(dim, n, product_lib):
    kfvm = product_lib
    assert kfvm.forcing_num_modes(dim) == n       # NUM_FORCING_MODES (src/Types.H:107-109)
    m = kfvm.forcing_draw(dim, 7)
    assert m.shape == (n, dim, 3)
    assert [tuple(int(x) for x in row) for row in m[:, :, 0]] == band(dim)
    # the same seed gives the same draw, another seed another
    assert np.array_equal(m, kfvm.forcing_draw(dim, 7))
    assert not np.array_equal(m[:, :, 1:], kfvm.forcing_draw(dim, 8)[:, :, 1:])


def test_amplitude_law(product_lib):
    """amplitude = sigma N(0,1) with sigma = sqrt(|k| (4 - |k|)), real and imaginary
    parts independent (ParameterStructs.cpp:58-72)."""
    kfvm = product_lib
    draws = np.stack([kfvm.forcing_draw(3, s) for s in range(200)])
    k = draws[0, :, :, 0]
    kmag = np.sqrt((k * k).sum(axis=1))
    sig = np.sqrt(kmag * (4.0 - kmag))
    z = (draws[:, :, :, 1:] / sig[None, :, None, None]).ravel()
    assert abs(z.mean()) < 0.02 and abs(z.var() - 1.0) < 0.03, (z.mean(), z.var())


@pytest.mark.parametrize("dim,n", [(2, 24), (3, 10)])
def test_oracle_kick_injects_edot_dt(dim, n, product_lib, oracle_lib):
    """From rest the kick adds edot dt of kinetic (and total) energy to the domain
    (the strength solves A s^2 + B s + C = 0, Solver.cpp:395-409) and, the modes being
    periodic on the box, no net momentum; a second kick on the moving gas again
    adds edot dt of total energy."""
    cfg, ic = abi.workload("stir_turb", scale=n, steps=4)
    if dim == 2:
        cfg = abi.make_config(2, abi.KFVM_EQ_HYDRO, n, n, gamma=1.001, rs=abi.KFVM_RS_HLL, cfl=1.25,
                              weno_thresh=-1.0, steps=4)
    o = oracle_lib.OracleSolver(cfg)
    o.init_ic(ic)
    f = abi.stir_turb_forcing()
    t, dt = o.time_dt()
    dvol = (1.0 / n) ** dim
    u0 = o.get_state()
    o.apply_forcing(product_lib.forcing_draw(dim, 3), f.edot, f.ratio)
    u1 = o.get_state()
    ke = 0.5 * ((u1[1:4] ** 2).sum(axis=0) / u1[0]).sum() * dvol
    assert abs(ke - f.edot * dt) <= 1e-12 * f.edot * dt
    assert abs((u1[4] - u0[4]).sum() * dvol - f.edot * dt) <= 1e-12 * f.edot * dt
    assert np.all(np.abs(u1[1:4].sum(axis=1)) <= 1e-10 * np.abs(u1[1:4]).sum(axis=1))
    assert np.array_equal(u1[0], u0[0])
    o.apply_forcing(product_lib.forcing_draw(dim, 4), f.edot, f.ratio)
    u2 = o.get_state()
    assert abs((u2[4] - u1[4]).sum() * dvol - f.edot * dt) <= 1e-11 * f.edot * dt


def test_driver_forcing_keys(tmp_path, product_lib):
    p = tmp_path / "st.init"
    src = open(os.path.join(ROOT, "kfvm-kokkos_b200", "problems", "stirturb3d.init")).read()
    p.write_text(src)
    got = json.loads(subprocess.run([RUN, "--parse-only", str(p)], capture_output=True, text=True,
                                    check=True).stdout)
    assert got["forcing"] == 1 and got["ic"] == abi.KFVM_IC_STIR_TURB
    assert got["force_edot"] == 60.0 and got["force_ratio"] == 1.0 and got["force_t_off"] == 1.5
    assert got["warnings"] == 0


@pytest.mark.gpu
@pytest.mark.parametrize("dim,n,eq", [(3, 12, abi.KFVM_EQ_HYDRO), (2, 32, abi.KFVM_EQ_HYDRO),
                                      (2, 32, abi.KFVM_EQ_MHD_GLM), (3, 12, abi.KFVM_EQ_NAVIERSTOKES)])
def test_forcing_against_oracle(dim, n, eq, gpu, product_lib, oracle_lib):
    """Forced steps, GPU against the oracle: each step the GPU draws a mode table,
    both sides kick with it at the same dt (strength to 1e-13, state to 1e-14) and
    take the step (1e-12 after the last)."""
    kfvm = product_lib
    rs = abi.KFVM_RS_LLF if eq == abi.KFVM_EQ_MHD_GLM else abi.KFVM_RS_HLL
    cfg = abi.make_config(dim, eq, n, n, n, gamma=1.001, rs=rs, cfl=1.0 if dim == 2 else 1.25,
                          weno_thresh=1.0, steps=6, reynolds=400.0, atol=1e-3, rtol=1e-3)
    g = kfvm.Solver(cfg)
    o = oracle_lib.OracleSolver(cfg)
    g.init_ic(abi.KFVM_IC_STIR_TURB)
    o.init_ic(abi.KFVM_IC_STIR_TURB)
    f = abi.stir_turb_forcing(seed=11)
    g.set_forcing(f)
    for step in range(4):
        t, dt = o.time_dt()
        g.set_time(t, dt)
        modes, sg = g.apply_forcing()
        so = o.apply_forcing(modes, f.edot, f.ratio)
        assert abs(sg - so) <= 1e-13 * abs(so), (step, sg, so)
        ug, uo = g.get_state(), o.get_state()
        # per variable against its own scale; a variable near rounding level (z momentum
        # in 2D, psi of a divergence-free field: |psi| ~ 1e-12, differences ~ 1e-17)
        # against 1e-4 of the mean scale
        num, den = np.abs(ug - uo).max(axis=1), np.abs(uo).max(axis=1)
        den = np.maximum(den, 1e-4 * den.mean())
        assert np.all(num / den <= 1e-13), (step, num / den)
        ig, io = g.take_step(), o.take_step()
        assert ig.accepted == io.accepted == 1
    ug, uo = g.get_state(), o.get_state()
    den = np.abs(uo).sum(axis=1)
    den = np.maximum(den, 1e-4 * den.mean())    # psi stays at rounding level, as above
    assert np.all(np.abs(ug - uo).sum(axis=1) / den <= 1e-12)
    g.close()


@pytest.mark.gpu
def test_solve_forces_until_t_off(gpu, product_lib):
    """kfvm_solve forces before each step while time < t_off (Solver.cpp:99-103):
    the kinetic energy grows while forced and the draws differ step to step."""
    kfvm = product_lib
    cfg, ic = abi.workload("stir_turb", scale=16, steps=6)
    g = kfvm.Solver(cfg)
    g.init_ic(ic)
    f = abi.stir_turb_forcing(seed=5)
    f.t_off = 1e9
    g.set_forcing(f)
    n, info = g.solve(cfg.max_steps)
    u = g.get_state()
    ke = 0.5 * ((u[1:4] ** 2).sum(axis=0) / u[0]).mean()
    assert n == 6 and ke > 0.0
    m1, _ = g.apply_forcing()
    m2, _ = g.apply_forcing()
    assert not np.array_equal(m1, m2)
    g.close()
