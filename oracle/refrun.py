"""TEST INFRASTRUCTURE ONLY: run the reference build (oracle/_ref/<problem>/kfvm_ref,
made by oracle/build_ref.py) and read its checkpoints.

The reference writes a checkpoint after the initial condition and after every
accepted step when io:ckptfreq is 1 (src/Solver.cpp:54-56, 113-122); the PDI
stand-in (oracle/refshim/pdi_shim.cpp) stores each as a raw file with the
step number, time, proposed next step size, the state with its halo and the
two WENO flag components.  Only tests/, the fixture script under tests/golden/
and bench.py's reference arm use this module.
"""
import glob
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(HERE, "_ref")
if HERE not in sys.path:
    sys.path.insert(0, HERE)


def binary(name):
    """Path of the reference build for a problem, or None if it was not built."""
    p = os.path.join(REF, name, "kfvm_ref")
    return p if os.path.exists(p) else None


def read_checkpoint(path):
    """(step, time, dt, state [nv, cells] interior in x-fastest order,
    weno flags [2, cells]) of one raw checkpoint."""
    b = open(path, "rb").read()
    if b[:8] != b"KFVMREF1":
        raise ValueError(f"{path}: not a reference checkpoint")
    h = np.frombuffer(b[8:44], dtype=np.int32)
    step, nv = int(h[0]), int(h[1])
    n, g = h[3:6], h[6:9]
    t, dt = np.frombuffer(b[44:60], dtype=np.float64)
    hs = [int(n[d] + 2 * g[d]) for d in range(3)]
    tot = hs[0] * hs[1] * hs[2] * nv
    u = np.frombuffer(b[60:60 + 8 * tot], dtype=np.float64).reshape(nv, hs[2], hs[1], hs[0])
    u = u[:, g[2]:g[2] + n[2], g[1]:g[1] + n[1], g[0]:g[0] + n[0]].reshape(nv, -1).copy()
    w = np.frombuffer(b[60 + 8 * tot:], dtype=np.float64).reshape(2, -1).copy()
    return step, float(t), float(dt), u, w


def run(name, cfg, steps, threads=None, ckpt=True, workdir=None, seed=12345):
    """Run the reference for `steps` accepted steps of a configuration.

    Returns (list of checkpoints in step order if ckpt else [], wall seconds)."""
    import build_ref
    exe = binary(name)
    if exe is None:
        raise FileNotFoundError(f"no reference build for {name} (run oracle/build_ref.py)")
    own = workdir is None
    tmp = tempfile.TemporaryDirectory() if own else None
    d = tmp.name if own else workdir
    try:
        init = build_ref.init_file(cfg, steps, os.path.join(d, "data"), seed=seed)
        if not ckpt:
            init = init.replace("io:ckptfreq 1", "io:ckptfreq 0")
        with open(os.path.join(d, "p.init"), "w") as f:
            f.write(init)
        env = dict(os.environ)
        env["OMP_NUM_THREADS"] = str(threads or os.cpu_count() or 1)
        env.setdefault("OMP_PROC_BIND", "close")
        t0 = time.perf_counter()
        r = subprocess.run([exe, "p.init"], cwd=d, env=env, capture_output=True, text=True)
        wall = time.perf_counter() - t0
        if r.returncode != 0:
            raise RuntimeError(f"reference run failed ({r.returncode}): {r.stdout[-2000:]}{r.stderr[-2000:]}")
        cks = []
        if ckpt:
            files = sorted(glob.glob(os.path.join(d, "data", "*", "ckpt", "*.raw")))
            cks = [read_checkpoint(f) for f in files]
        return cks, wall
    finally:
        if tmp is not None:
            tmp.cleanup()


def time_steps(name, cfg, steps, threads=None):
    """Seconds per accepted step of the reference's own stepping loop: the wall time of a
    run of `steps` steps minus that of a run of 0 steps (both pay the same setup:
    weights, initial condition and the FSAL priming evaluation; no files written)."""
    _, w0 = run(name, cfg, 0, threads=threads, ckpt=False)
    _, w1 = run(name, cfg, steps, threads=threads, ckpt=False)
    _, w0b = run(name, cfg, 0, threads=threads, ckpt=False)
    return max(w1 - min(w0, w0b), 1e-9) / steps
