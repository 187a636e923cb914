"""TEST INFRASTRUCTURE ONLY: ctypes front end of the CPU oracle (liboracle.so).

The oracle is a plain CPU restatement of the reference's per-stage hot path
(see oracle_solver.cpp for the reference file:line map).  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg may use it, and only as
the checker / the timed CPU baseline -- never as the product path.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_PKG = os.path.join(os.path.dirname(_HERE), "kfvm-kokkos_b200")
if _PKG not in sys.path:
    sys.path.insert(0, _PKG)

import kfvm_abi as abi  # noqa: E402

_LIB = None


def build():
    """Compile liboracle.so with the committed Makefile (g++, OpenMP, scipy's OpenBLAS)."""
    subprocess.run(["make", "-s", "-C", _HERE, f"PY={sys.executable}"], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        P, I32, I64, D = C.c_void_p, C.c_int32, C.c_int64, C.c_double
        L.orc_stencil_build.argtypes = [C.POINTER(abi.KfvmConfig), C.POINTER(abi.KfvmStencil)]
        L.orc_create.argtypes = [C.POINTER(abi.KfvmConfig)]
        L.orc_create.restype = P
        L.orc_destroy.argtypes = [P]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_init_ic.argtypes = [P, I32, C.c_uint64]
        L.orc_set_state.argtypes = [P, P]
        L.orc_get_state.argtypes = [P, P]
        L.orc_eval_rhs.argtypes = [P, D, P, P]
        L.orc_take_step.argtypes = [P, C.POINTER(abi.KfvmStepInfo)]
        L.orc_solve.argtypes = [P, I32, C.POINTER(I64), C.POINTER(abi.KfvmStepInfo)]
        L.orc_get_time.argtypes = [P, P, P]
        L.orc_set_time.argtypes = [P, D, D]
        L.orc_apply_forcing.argtypes = [P, P, I32, D, D, P]
        L.orc_flow_stats.argtypes = [P, P, P]
        L.orc_get_faces.argtypes = [P, I32, P]
        L.orc_keep_faces.argtypes = [P, I32]
        L.orc_get_flags.argtypes = [P, P, P]
        L.orc_set_indicator.argtypes = [P, I32]
        L.orc_weno_departure.argtypes = [P, P]
        L.orc_ic_cells.argtypes = [C.POINTER(abi.KfvmConfig), I32, C.c_uint64, P]
        L.orc_tables.argtypes = [I32, I32, P, P]
        L.orc_set_exchange.argtypes = [P, abi.EXCHANGE_FN, abi.ALLREDUCE_FN, P]
        L.orc_set_user_bc.argtypes = [P, abi.USER_BC_FN, P]
        _LIB = L
    return _LIB


def set_threads(n):
    return lib().orc_set_threads(int(n))


def stencil(cfg):
    st = abi.KfvmStencil()
    rc = lib().orc_stencil_build(C.byref(cfg), C.byref(st))
    if rc != 0:
        raise RuntimeError(f"orc_stencil_build failed: {rc}")
    return st


def tables(nq, rk):
    """(quadrature abscissae, weights, RK coefficient dict) as used by the oracle."""
    q = np.zeros(2 * nq)
    r = np.zeros(128)
    if lib().orc_tables(int(nq), int(rk), q.ctypes.data, r.ctypes.data) != 0:
        raise ValueError(rk)
    ns = int(r[0])
    cols = ["gam1", "gam2", "gam3", "delta", "beta", "bhat", "c"]
    d = {"nStages": ns}
    for k, name in enumerate(cols):
        d[name] = list(r[1 + k * ns: 1 + (k + 1) * ns])
    m = 1 + 7 * ns
    d["bhatfsal"], d["ep1"], d["ep2"] = r[m], r[m + 1], r[m + 2]
    return list(q[:nq]), list(q[nq:]), d


def ic_cells(cfg, ic_kind, seed=12345):
    u = np.zeros((abi.nvars(cfg), abi.ncells(cfg)), dtype=np.float64)
    rc = lib().orc_ic_cells(C.byref(cfg), int(ic_kind), C.c_uint64(seed), u.ctypes.data)
    if rc != 0:
        raise RuntimeError(rc)
    return u


class OracleSolver:
    """CPU oracle mirror of Solver (construct, IC, evalRHS, TakeStep, Solve)."""

    def __init__(self, cfg):
        self.cfg = cfg
        self.nv = abi.nvars(cfg)
        self.n = abi.ncells(cfg)
        self.h = lib().orc_create(C.byref(cfg))
        if not self.h:
            raise RuntimeError("orc_create failed")

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def init_ic(self, ic_kind, seed=12345):
        rc = lib().orc_init_ic(self.h, int(ic_kind), C.c_uint64(seed))
        assert rc == 0

    def set_state(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64).reshape(self.nv, self.n)
        assert lib().orc_set_state(self.h, u.ctypes.data) == 0

    def get_state(self):
        u = np.empty((self.nv, self.n), dtype=np.float64)
        assert lib().orc_get_state(self.h, u.ctypes.data) == 0
        return u

    def eval_rhs(self, t=0.0):
        r = np.empty((self.nv, self.n), dtype=np.float64)
        mv = C.c_double()
        assert lib().orc_eval_rhs(self.h, float(t), r.ctypes.data, C.addressof(mv)) == 0
        return r, mv.value

    def take_step(self):
        info = abi.KfvmStepInfo()
        assert lib().orc_take_step(self.h, C.byref(info)) == 0
        return info

    def solve(self, max_steps):
        info = abi.KfvmStepInfo()
        n = C.c_int64()
        assert lib().orc_solve(self.h, int(max_steps), C.byref(n), C.byref(info)) == 0
        return n.value, info

    def time_dt(self):
        t, dt = C.c_double(), C.c_double()
        lib().orc_get_time(self.h, C.addressof(t), C.addressof(dt))
        return t.value, dt.value

    def flow_stats(self):
        out = np.zeros(3, dtype=np.float64)
        n = C.c_int32()
        assert lib().orc_flow_stats(self.h, out.ctypes.data, C.addressof(n)) == 0
        return out[:n.value].copy()

    def apply_forcing(self, modes, edot, ratio):
        """Random forcing with the given mode table [n][dim][3]; returns the strength."""
        m = np.ascontiguousarray(modes, dtype=np.float64)
        s = C.c_double()
        assert lib().orc_apply_forcing(self.h, m.ctypes.data, m.shape[0], float(edot), float(ratio),
                                       C.addressof(s)) == 0
        return s.value

    def set_time(self, t, dt):
        assert lib().orc_set_time(self.h, float(t), float(dt)) == 0

    def set_user_bc(self, fn):
        """User boundary conditions on host buffers: fn(kind, face, time, inner, outer)
        with float64 numpy arrays of shape (NV, points), as kfvm.Solver.set_user_bc."""
        nv = self.nv

        def cb(user, kind, face, time, inner, outer, npts, stream):
            try:
                n = int(npts) * nv
                a = np.ctypeslib.as_array((C.c_double * n).from_address(inner)).reshape(nv, -1)
                b = np.ctypeslib.as_array((C.c_double * n).from_address(outer)).reshape(nv, -1)
                fn(int(kind), int(face), float(time), a, b)
                return 0
            except Exception as e:  # noqa: BLE001
                self.user_bc_error = e
                return 1

        self._user_bc = abi.USER_BC_FN(cb)
        self.user_bc_error = None
        assert lib().orc_set_user_bc(self.h, self._user_bc, None) == 0

    def set_exchange(self, transport):
        """Install a host-buffer transport for the exchange faces of a decomposed domain."""
        self._transport = transport
        assert lib().orc_set_exchange(self.h, transport.exchange_fn, transport.allreduce_fn, None) == 0

    def keep_faces(self, on=True):
        assert lib().orc_keep_faces(self.h, 1 if on else 0) == 0

    def faces(self, d):
        c = self.cfg
        nz = c.nz if c.dim == 3 else 1
        fd = [c.nx + (d == 0), c.ny + (d == 1), nz + (d == 2)]
        nqf = c.nq if c.dim == 2 else c.nq * c.nq
        out = np.empty((2, nqf, self.nv, fd[2] * fd[1] * fd[0]), dtype=np.float64)
        assert lib().orc_get_faces(self.h, int(d), out.ctypes.data) == 0
        return out

    def flags(self):
        a = np.empty(self.n, dtype=np.uint8)
        th = np.empty(self.n, dtype=np.float64)
        assert lib().orc_get_flags(self.h, a.ctypes.data, th.ctypes.data) == 0
        return a, th

    def weno_departure(self):
        """max_{s,v} |omega_{s,v} - gamma_s| of every cell (label of the learned indicator)."""
        out = np.empty(self.n, dtype=np.float64)
        assert lib().orc_weno_departure(self.h, out.ctypes.data) == 0
        return out

    def set_indicator(self, ind):
        assert lib().orc_set_indicator(self.h, int(ind)) == 0
