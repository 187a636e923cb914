"""Plot and checkpoint files (the XDMF + raw binary counterpart of the reference's
WriterPDI, src/io/WriterPDI.cpp): layout, datasets, auxiliary variables as
AuxVars computes them, the checkpoint round trip, and the restart through the
solver and the kfvm_run driver (GPU)."""
import os
import subprocess
import xml.etree.ElementTree as ET

import numpy as np
import pytest

import kfvm_abi as abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "kfvm-kokkos_b200")
RUN = os.path.join(PKG, "kfvm_run")


def small_cfg(dim, eq, nx=6, ny=5, nz=4):
    c = abi.default_config()
    c.dim, c.eq = dim, eq
    c.nx, c.ny, c.nz = nx, ny, (nz if dim == 3 else 1)
    c.xlo, c.xup, c.ylo, c.yup, c.zlo, c.zup = -1.0, 2.0, 0.0, 1.0, 0.5, 2.5
    c.gamma = abi.stof(5.0 / 3.0) if eq == abi.KFVM_EQ_MHD_GLM else abi.stof(1.4)
    return c


def random_state(cfg, seed=3):
    rng = np.random.default_rng(seed)
    nv, n = abi.nvars(cfg), abi.ncells(cfg)
    u = rng.normal(size=(nv, n))
    u[0] = 0.5 + rng.random(n)        # density
    u[4] = 10.0 + rng.random(n)       # total energy
    weno = (rng.random(n) < 0.3).astype(np.uint8)
    theta = np.where(rng.random(n) < 0.2, rng.random(n), 1.0)
    return u, weno, theta


def items(xmf):
    """{attribute name: [binary file names]} and the geometry's coordinate files."""
    root = ET.parse(xmf).getroot()
    grid = root.find("Domain").find("Grid")
    attrs = {}
    for a in grid.findall("Attribute"):
        attrs[a.get("Name")] = [d.text.strip() for d in a.iter("DataItem") if d.get("Format") == "Binary"]
    geo = [d.text.strip() for d in grid.find("Geometry").findall("DataItem")]
    return grid, attrs, geo


def test_plot_layout_and_aux_hydro_3d(tmp_path, product_lib):
    kfvm = product_lib
    cfg = small_cfg(3, abi.KFVM_EQ_HYDRO)
    u, weno, theta = random_state(cfg)
    xmf = kfvm.plotfile_write(cfg, tmp_path / "plot", "sod", 3, u, weno, theta, time=0.25, time_step=3)
    assert os.path.basename(xmf) == "sod_0000003.xmf" and os.path.exists(xmf)
    grid, attrs, geo = items(xmf)
    assert grid.find("Topology").get("TopologyType") == "3DRectMesh"
    assert grid.find("Topology").get("NumberOfElements") == "5 6 7"   # nz+1 ny+1 nx+1
    assert float(grid.find("Time").get("Value")) == 0.25
    # WriterPDI::writeAttrHydro then weno, fomx
    assert list(attrs) == ["dens", "mom", "etot", "vel", "eint", "pres", "weno", "fomx"]
    d = tmp_path / "plot"
    n = abi.ncells(cfg)
    for names in list(attrs.values()) + [geo]:
        for f in names:
            assert os.path.exists(d / f), f
    rd = lambda name: np.fromfile(d / f"sod_0000003.{name}.bin", dtype="<f8")
    for v, name in enumerate(["dens", "momx", "momy", "momz", "etot"]):
        assert np.array_equal(rd(name), u[v])
    # AuxVars<Hydro>: velocities, internal energy, pressure (Hydro_K.H:66-97)
    assert np.array_equal(rd("velx"), u[1] / u[0])
    assert np.array_equal(rd("velz"), u[3] / u[0])
    ei = u[4] - 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / u[0]
    assert np.array_equal(rd("eint"), ei)
    assert np.array_equal(rd("pres"), (cfg.gamma - 1.0) * ei)
    assert np.array_equal(rd("weno"), weno.astype(np.float64))
    assert np.array_equal(rd("fomx"), theta)
    # nodal coordinates (WriterPDI.cpp:38-52)
    assert np.allclose(rd("xcoord"), -1.0 + 0.5 * np.arange(7), rtol=0, atol=1e-15)
    assert np.allclose(rd("zcoord"), 0.5 + 0.5 * np.arange(5), rtol=0, atol=1e-15)
    assert all(rd(x).size == n for x in ("dens", "eint", "weno"))


def test_plot_glm_2d_names(tmp_path, product_lib):
    kfvm = product_lib
    cfg = small_cfg(2, abi.KFVM_EQ_MHD_GLM)
    u, weno, theta = random_state(cfg, seed=5)
    xmf = kfvm.plotfile_write(cfg, tmp_path, "ot", 0, u, weno, theta)
    grid, attrs, _ = items(xmf)
    assert grid.find("Topology").get("NumberOfElements") == "2 6 7"
    assert list(attrs) == ["dens", "mom", "B", "etot", "psi", "vel", "eint", "prsg", "prsb", "weno", "fomx"]
    rd = lambda name: np.fromfile(tmp_path / f"ot_0000000.{name}.bin", dtype="<f8")
    pb = 0.5 * (u[5] * u[5] + u[6] * u[6] + u[7] * u[7])
    ke = 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / u[0]
    ei = u[4] - pb - ke - 0.5 * u[8] * u[8]
    assert np.array_equal(rd("prsb"), pb)
    assert np.array_equal(rd("eint"), ei)
    assert np.array_equal(rd("prsg"), (cfg.gamma - 1.0) * ei)
    # 2D: one cell layer, z spacing dmin (WriterPDI.cpp:45)
    assert np.allclose(rd("zcoord"), [0.0, 0.2], rtol=0, atol=1e-15)


def test_checkpoint_round_trip(tmp_path, product_lib):
    kfvm = product_lib
    cfg = small_cfg(3, abi.KFVM_EQ_NAVIERSTOKES)
    u, weno, theta = random_state(cfg, seed=7)
    xmf = kfvm.plotfile_write(cfg, tmp_path / "ckpt", "tg", 40, u, weno, theta, time=0.1234567890123,
                              time_step=40, dt=3.3e-3, ckpt=True)
    _, attrs, _ = items(xmf)
    assert list(attrs) == ["dens", "mom", "etot", "weno", "fomx"]   # no auxiliary variables
    r = kfvm.plotfile_read(cfg, xmf)
    assert np.array_equal(r["u"], u) and np.array_equal(r["weno"], weno) and np.array_equal(r["theta"], theta)
    assert r["time"] == 0.1234567890123 and r["dt"] == 3.3e-3 and r["time_step"] == 40


def test_read_rejects_other_grid_and_short_files(tmp_path, product_lib):
    kfvm = product_lib
    cfg = small_cfg(2, abi.KFVM_EQ_HYDRO)
    u, weno, theta = random_state(cfg)
    xmf = kfvm.plotfile_write(cfg, tmp_path, "a", 1, u, weno, theta, ckpt=True, dt=1e-3)
    other = small_cfg(2, abi.KFVM_EQ_HYDRO, nx=7)
    with pytest.raises(kfvm.KfvmError):
        kfvm.plotfile_read(other, xmf)
    with open(tmp_path / "a_0000001.etot.bin", "r+b") as f:
        f.truncate(8 * 3)
    with pytest.raises(kfvm.KfvmError):
        kfvm.plotfile_read(cfg, xmf)


def test_io_keys_parsed(tmp_path, product_lib):
    p = tmp_path / "x.init"
    p.write_text("setup:dim 2\nio:plotfreq 0.1\nio:ckptfreq 5\nio:restartfile d/ckpt/a_0000005.xmf\n")
    out = subprocess.run([RUN, "--parse-only", str(p)], capture_output=True, text=True, check=True)
    import json
    got = json.loads(out.stdout)
    assert got["plot_freq"] == float(np.float32(0.1)) and got["ckpt_freq"] == 5 and got["restart"] == 1


@pytest.mark.gpu
def test_driver_plots_on_plot_times_and_restarts(tmp_path, gpu, product_lib):
    kfvm = product_lib
    src = open(os.path.join(PKG, "problems", "isenvort.init")).read()
    src = src.replace("mesh:resolution 128 128", "mesh:resolution 32 32").replace("time:maxsteps 21", "time:maxsteps 12")
    # final time short enough that plot times fall inside the run
    p = tmp_path / "iv.init"
    p.write_text(src + "io:plotfreq 0.005\nio:ckptfreq 4\nio:basename iv\nio:datadir out\ntime:final 0.05\n")
    r = subprocess.run([RUN, str(p)], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    plot = tmp_path / "out" / "R2_NX32_NY32" / "plot"
    ckpt = tmp_path / "out" / "R2_NX32_NY32" / "ckpt"
    metas = sorted(plot.glob("iv_*.meta"))
    assert len(metas) >= 3
    times = [float([l for l in open(m) if l.startswith("time ")][0].split()[1]) for m in metas]
    assert times[0] == 0.0
    # a plot on every multiple of plotfreq that the run passed (Solver.cpp:202-205)
    for k, t in enumerate(times[1:-1], start=1):
        assert abs(t - k * float(np.float32(0.005))) < 1e-12, (k, t)
    assert (ckpt / "iv_0000000.xmf").exists() and (ckpt / "iv_0000004.xmf").exists()

    # restart from the step-4 checkpoint and compare with an uninterrupted run
    cfg, ic = abi.workload("isentropic_vortex", scale=32, steps=12)
    a = kfvm.Solver(cfg)
    a.init_ic(ic)
    for _ in range(4):
        a.take_step()
    a.write_plotfile(tmp_path / "ck", "iv", 4, ckpt=True, time_step=4)
    u4 = a.get_state().copy()
    t4, dt4 = a.time_dt()
    b = kfvm.Solver(cfg)
    assert b.restart(tmp_path / "ck" / "iv_0000004.xmf") == 4
    assert np.array_equal(b.get_state(), u4)
    assert b.time_dt() == (t4, dt4)
    ia, ib = a.take_step(), b.take_step()
    assert ia.accepted and ib.accepted
    # same state, step size and FSAL stage: the step after the restart is the same
    # (the error-controller history is not in the checkpoint, as in the reference,
    # so later step sizes may differ)
    assert np.array_equal(a.get_state(), b.get_state())
    a.close()
    b.close()


def test_plot_srhydro_aux_recovers_primitives(tmp_path, product_lib):
    """AuxVars<SRHydro> (SRHydro_K.H:59-88, WriterPDI.cpp:268-278): rho, vel, lorz and
    pres from the Newton pressure recovery of SRHydro_EOS.H, checked against the
    primitives the conserved state was built from, over both branches of the
    recovery (D^2 / (E^2 - S^2) above and below 1e-4) and Lorentz factors up to 22."""
    kfvm = product_lib
    cfg = small_cfg(2, abi.KFVM_EQ_SRHYDRO)
    cfg.gamma = abi.stof(5.0 / 3.0)
    g = cfg.gamma
    rng = np.random.default_rng(11)
    n = abi.ncells(cfg)
    rho = 10.0 ** rng.uniform(-3, 1, n)
    p = 10.0 ** rng.uniform(-3, 2, n)
    speed = np.concatenate([rng.uniform(0, 0.999, n - 4), [0.0, 0.5, 0.99, 0.999]])
    ang = rng.uniform(0, 2 * np.pi, n)
    vx, vy, vz = speed * np.cos(ang), speed * np.sin(ang) * 0.8, speed * np.sin(ang) * 0.6
    W = 1.0 / np.sqrt(1.0 - (vx * vx + vy * vy + vz * vz))
    h = 1.0 + g * p / ((g - 1.0) * rho)
    u = np.stack([rho * W, rho * W * W * h * vx, rho * W * W * h * vy, rho * W * W * h * vz,
                  rho * W * W * h - p])
    weno = np.zeros(n, np.uint8)
    theta = np.ones(n)
    xmf = kfvm.plotfile_write(cfg, tmp_path, "sr", 2, u, weno, theta)
    _, attrs, _ = items(xmf)
    assert list(attrs) == ["dens", "mom", "etot", "rho", "vel", "lorz", "pres", "weno", "fomx"]
    rd = lambda name: np.fromfile(tmp_path / f"sr_0000002.{name}.bin", dtype="<f8")
    assert np.allclose(rd("pres"), p, rtol=1e-8, atol=0)
    assert np.allclose(rd("rho"), rho, rtol=1e-8, atol=0)
    assert np.allclose(rd("lorz"), W, rtol=1e-8, atol=0)
    for name, v in (("velx", vx), ("vely", vy), ("velz", vz)):
        assert np.allclose(rd(name), v, rtol=1e-8, atol=1e-12)
