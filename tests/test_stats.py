"""Flow statistics (Solver::evalFlowStats, src/Solver.cpp:153-185; FlowStats<Eq> in
src/physics/hydro/Hydro_K.H:103-178, navierstokes/NavierStokes_K.H:102-175,
mhd_glm/MHD_GLM_K.H:108-211): volume-averaged kinetic energy and enstrophy (and the
current helicity for GLM-MHD).  CPU: the oracle against the Taylor-Green vortex's
analytic averages and the driver key; GPU: the device reduction against the oracle
and the driver's stats file."""
import json
import os
import subprocess

import numpy as np
import pytest

import kfvm_abi as abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RUN = os.path.join(ROOT, "kfvm-kokkos_b200", "kfvm_run")


def test_oracle_taylor_green_averages(oracle_lib):
    """u = sin x cos y cos z, v = -cos x sin y cos z: <|u|^2>/2 = 1/8 and
    <|curl u|^2>/2 = 3/8, up to the density's Mach-0.1 variation and the central
    differences' factor (sin dx / dx)^2 at 32^3."""
    cfg, ic = abi.workload("taylor_green", scale=32, steps=2)
    o = oracle_lib.OracleSolver(cfg)
    o.init_ic(ic)
    ek, en = o.flow_stats()
    dx = 2.0 * np.pi / 32
    assert abs(ek - 0.125) < 2e-3, ek
    assert abs(en - 0.375 * (np.sin(dx) / dx) ** 2) < 5e-3, en


def test_oracle_stats_counts(oracle_lib):
    cfg, ic = abi.workload("orszag_tang", scale=16, steps=2)
    o = oracle_lib.OracleSolver(cfg)
    o.init_ic(ic)
    st = o.flow_stats()
    assert st.shape == (3,) and np.all(np.isfinite(st)) and st[0] > 0.0
    cfg, ic = abi.workload("sr_riemann_2d", scale=16, steps=2)
    o = oracle_lib.OracleSolver(cfg)
    o.init_ic(ic)
    assert np.array_equal(o.flow_stats(), [0.0])    # no statistics for SRHydro


def test_driver_statsfreq_key(tmp_path, product_lib):
    p = tmp_path / "s.init"
    p.write_text("setup:dim 3\nio:statsfreq 5\n")
    got = json.loads(subprocess.run([RUN, "--parse-only", str(p)], capture_output=True, text=True,
                                    check=True).stdout)
    assert got["stats_freq"] == 5 and got["warnings"] == 0


@pytest.mark.gpu
@pytest.mark.parametrize("name,scale,steps", [("taylor_green", 12, 2), ("kelvin_helmholtz", 32, 3),
                                              ("orszag_tang", 32, 3), ("sod3d", 12, 2),
                                              ("sr_riemann_2d", 16, 2)])
def test_stats_against_oracle(name, scale, steps, gpu, product_lib, oracle_lib):
    cfg, ic = abi.workload(name, scale=scale, steps=steps)
    g = product_lib.Solver(cfg)
    o = oracle_lib.OracleSolver(cfg)
    g.init_ic(ic)
    o.init_ic(ic)
    for _ in range(steps):
        t, dt = o.time_dt()
        g.set_time(t, dt)
        g.take_step()
        o.take_step()
    sg, so = g.flow_stats(), o.flow_stats()
    assert sg.shape == so.shape
    assert np.all(np.abs(sg - so) <= 1e-11 * np.maximum(np.abs(so), 1e-300)), (sg, so)
    g.close()


@pytest.mark.gpu
def test_driver_writes_stats_rows(tmp_path, gpu, product_lib):
    """Rows before stepping, every statsfreq steps and after the last step
    (Solver.cpp:87-91, 108-111, 124-126)."""
    src = open(os.path.join(ROOT, "kfvm-kokkos_b200", "problems", "taygreen.init")).read()
    src = src.replace("mesh:resolution 256 256 256", "mesh:resolution 16 16 16")
    p = tmp_path / "tg.init"
    p.write_text(src + "time:maxsteps 8\nio:statsfreq 3\nio:basename tg\nio:datadir out\n")
    r = subprocess.run([RUN, str(p)], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    rows = np.loadtxt(tmp_path / "out" / "R2_NX16_NY16_NZ16" / "tg_stats.dat", ndmin=2)
    # steps 1..7 end at maxsteps, not at the final time: before stepping and after
    # steps 3 and 6 (the row after the last step needs lastTimeStep)
    assert rows.shape == (3, 3), rows.shape
    assert np.all(np.diff(rows[:, 0]) > 0.0)
    assert np.all(np.diff(rows[:, 1]) < 0.0)        # the vortex decays


# halo signs of the wall types (Hydro_BCCoeffs.H: reflect negates the normal
# momentum, no-slip every momentum)
def _halo_signs(bc, axis):
    s = np.ones(5)
    if bc == abi.KFVM_BC_REFLECTING:
        s[1 + axis] = -1.0
    elif bc == abi.KFVM_BC_NOSLIP:
        s[1:4] = -1.0
    return s


def _flow_stats_np(u, cfg):
    """FlowStats<Hydro / NavierStokes> (Hydro_K.H:103-178, NavierStokes_K.H:102-175)
    in numpy on an interior state (5, nz, ny, nx).  The one halo layer it reads is
    filled here from the boundary types alone, independently of the solver:
    periodic wrap, outflow copy, and the mirrored boundary cell with the sign table
    of the wall type."""
    a = u.copy()
    for ax, arr_ax in ((0, 3), (1, 2), (2, 1)):      # x, y, z: array axes 3, 2, 1
        lo, hi = cfg.bc[2 * ax], cfg.bc[2 * ax + 1]
        if lo == abi.KFVM_BC_PERIODIC:
            a = np.concatenate([np.take(a, [-1], axis=arr_ax), a, np.take(a, [0], axis=arr_ax)], axis=arr_ax)
            continue
        sl = _halo_signs(lo, ax).reshape(5, 1, 1, 1)
        sh = _halo_signs(hi, ax).reshape(5, 1, 1, 1)
        a = np.concatenate([sl * np.take(a, [0], axis=arr_ax), a, sh * np.take(a, [-1], axis=arr_ax)],
                           axis=arr_ax)
    dx = (cfg.xup - cfg.xlo) / cfg.nx
    dy = (cfg.yup - cfg.ylo) / cfg.ny
    dz = (cfg.zup - cfg.zlo) / cfg.nz
    v = a[1:4] / a[0]
    c = (slice(1, -1),) * 3

    def d(comp, ax, h):
        p = [slice(1, -1)] * 3
        m = [slice(1, -1)] * 3
        p[ax] = slice(2, None)
        m[ax] = slice(0, -2)
        return 0.5 * (v[comp][tuple(p)] - v[comp][tuple(m)]) / h
    # array axes of v[comp]: 0 = z, 1 = y, 2 = x
    dyu, dxv = d(0, 1, dy), d(1, 2, dx)
    dzu, dzv, dxw, dyw = d(0, 0, dz), d(1, 0, dz), d(2, 2, dx), d(2, 1, dy)
    om2 = (dyw - dzv) ** 2 + (dzu - dxw) ** 2 + (dxv - dyu) ** 2
    rho = a[0][c]
    ek = 0.5 * (a[1][c] ** 2 + a[2][c] ** 2 + a[3][c] ** 2) / rho
    ifac = (dx * dy * dz) / ((cfg.xup - cfg.xlo) * (cfg.yup - cfg.ylo) * (cfg.zup - cfg.zlo))
    return np.array([ifac * ek.sum(), ifac * (0.5 * rho * om2).sum()])


@pytest.mark.gpu
@pytest.mark.parametrize("walls", ["ppnnrr", "rrppnn"])
def test_stats_after_restart_with_walls(walls, tmp_path, gpu, product_lib):
    """Right after a restart the solver has evaluated nothing, so the halo the
    statistics read comes from the statistics call itself.  Checked against the
    reference's formula in numpy with a halo filled independently from the wall
    types, on a Taylor-Green box with no-slip and reflecting walls."""
    codes = {"p": abi.KFVM_BC_PERIODIC, "r": abi.KFVM_BC_REFLECTING, "n": abi.KFVM_BC_NOSLIP}
    cfg, ic = abi.workload("taylor_green", scale=12, steps=2)
    for f, w in enumerate(walls):
        cfg.bc[f] = codes[w]
    a = product_lib.Solver(cfg)
    a.init_ic(ic)
    for _ in range(2):
        assert a.take_step().accepted
    a.write_plotfile(tmp_path / "ck", "tg", 2, ckpt=True, time_step=2)
    b = product_lib.Solver(cfg)
    assert b.restart(tmp_path / "ck" / "tg_0000002.xmf") == 2
    u = b.get_state().reshape(5, cfg.nz, cfg.ny, cfg.nx)
    ref = _flow_stats_np(u, cfg)
    got = b.flow_stats()
    assert np.all(np.abs(got - ref) <= 1e-12 * np.abs(ref)), (got, ref)
    # the solver that stepped there reports the same statistics
    assert np.all(np.abs(a.flow_stats() - ref) <= 1e-12 * np.abs(ref))
    a.close()
    b.close()
