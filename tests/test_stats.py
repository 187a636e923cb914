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
