"""The C++ host layer (kfvm-kokkos_b200/host): .init parsing with the reference's
std::stof semantics, and the kfvm_run driver (the counterpart of kfvm.ex)."""
import json
import os
import subprocess

import numpy as np
import pytest

import kfvm_abi as abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "kfvm-kokkos_b200")
RUN = os.path.join(PKG, "kfvm_run")
PROBLEMS = {"sod3d.init": "sod3d", "isenvort.init": "isentropic_vortex",
            "kelvhelm.init": "kelvin_helmholtz", "taygreen.init": "taylor_green",
            "orszagtang.init": "orszag_tang"}


def parse(path):
    out = subprocess.run([RUN, "--parse-only", path], capture_output=True, text=True, check=True)
    return json.loads(out.stdout)


@pytest.mark.parametrize("fname,name", sorted(PROBLEMS.items()))
def test_problem_files_match_workloads(fname, name, product_lib):
    got = parse(os.path.join(PKG, "problems", fname))
    cfg, ic = abi.workload(name)
    assert got["warnings"] == 0
    assert got["ic"] == ic
    for k in ("dim", "eq", "rs", "rk", "nq", "nx", "ny", "max_steps", "have_sources"):
        assert got[k] == getattr(cfg, k), k
    for k in ("gamma", "cfl", "weno_thresh", "lfac", "atol", "rtol"):
        assert got[k] == getattr(cfg, k), k
    ext = [cfg.xlo, cfg.xup, cfg.ylo, cfg.yup, cfg.zlo, cfg.zup]
    n = 6 if cfg.dim == 3 else 4
    assert got["extent"][:n] == ext[:n]


def test_stof_semantics(tmp_path, product_lib):
    p = tmp_path / "x.init"
    p.write_text("setup:dim 2\neos:gamma 1.4\ntime:cfl 0.8\nmesh:extent -5.0 5.0 -5.0 5.0\n"
                 "time:maxsteps 21\nbogus:line 1\n")
    got = parse(str(p))
    assert got["gamma"] == float(np.float32(1.4))
    assert got["cfl"] == float(np.float32(0.8))
    assert got["max_steps"] == 21
    assert got["warnings"] == 1


@pytest.mark.gpu
def test_kfvm_run_matches_python_driver(tmp_path, gpu, product_lib):
    p = tmp_path / "iv.init"
    src = open(os.path.join(PKG, "problems", "isenvort.init")).read()
    src = src.replace("mesh:resolution 128 128", "mesh:resolution 32 32").replace("time:maxsteps 21", "time:maxsteps 6")
    p.write_text(src + "io:dumpstate 1\nio:basename " + str(tmp_path / "iv") + "\n")
    r = subprocess.run([RUN, str(p)], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    assert "Time stepping completed" in r.stdout
    u_cpp = np.fromfile(str(tmp_path / "iv_state.bin"), dtype=np.float64).reshape(5, -1)
    cfg, ic = abi.workload("isentropic_vortex", scale=32, steps=5)
    s = product_lib.Solver(cfg)
    s.init_ic(ic)
    s.solve(cfg.max_steps)
    assert np.array_equal(u_cpp, s.get_state())
