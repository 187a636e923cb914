"""Python front end of libkfvm_b200.so (the C ABI in include/kfvm_b200.h).

Mirrors the reference's Solver operator boundary (slug-cfd/kfvm-kokkos
src/Solver.H:118-160): construct with a run configuration, set an initial
condition, evalRHS, TakeStep, Solve.  Every call goes to the sm_100a CUDA path;
there is no CPU fallback -- if the library or a GPU is missing the calls raise.
"""
import ctypes as C
import os

import numpy as np

import kfvm_abi as abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libkfvm_b200.so")
_LIB = None


class KfvmError(RuntimeError):
    pass


# kernel classes of kfvm_get_timing (enum kfvm_kernel_class)
KCLASS = ["bc_fill", "compact", "flag", "recon", "heavy", "riemann", "stage", "other"]


def lib():
    """Load the in-tree CUDA library (built by build.py); raises if it is absent."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise KfvmError(f"{LIB_PATH} is missing: run kfvm-kokkos_b200/build.py")
        L = C.CDLL(LIB_PATH)
        P, I32, I64, D = C.c_void_p, C.c_int32, C.c_int64, C.c_double
        L.kfvm_default_config.argtypes = [C.POINTER(abi.KfvmConfig)]
        L.kfvm_default_config.restype = None
        L.kfvm_stencil_build.argtypes = [C.POINTER(abi.KfvmConfig), C.POINTER(abi.KfvmStencil)]
        L.kfvm_create.argtypes = [C.POINTER(abi.KfvmConfig), C.POINTER(P)]
        L.kfvm_destroy.argtypes = [P]
        L.kfvm_destroy.restype = None
        L.kfvm_init_ic.argtypes = [P, I32, C.c_uint64]
        L.kfvm_set_state.argtypes = [P, P]
        L.kfvm_get_state.argtypes = [P, P]
        L.kfvm_eval_rhs.argtypes = [P, D, P, P]
        L.kfvm_take_step.argtypes = [P, C.POINTER(abi.KfvmStepInfo)]
        L.kfvm_err_est.argtypes = [P, P, P, P, P]
        L.kfvm_err_est_noalloc.argtypes = [I32, P, P, I64, D, D, P, P]
        L.kfvm_solve.argtypes = [P, I32, C.POINTER(I64), C.POINTER(abi.KfvmStepInfo)]
        L.kfvm_get_time.argtypes = [P, P, P]
        L.kfvm_set_time.argtypes = [P, D, D]
        L.kfvm_set_indicator.argtypes = [P, I32]
        L.kfvm_set_precision.argtypes = [P, I32]
        L.kfvm_get_faces.argtypes = [P, I32, P]
        L.kfvm_get_flags.argtypes = [P, P, P]
        L.kfvm_last_stage_ms.argtypes = [P, P]
        L.kfvm_get_stream.argtypes = [P, C.POINTER(C.c_void_p)]
        L.kfvm_set_timing.argtypes = [P, I32]
        L.kfvm_get_timing.argtypes = [P, P, P]
        L.kfvm_get_launch_count.argtypes = [P, C.POINTER(I64)]
        L.kfvm_last_error.restype = C.c_char_p
        _LIB = L
    return _LIB


def _check(rc, what):
    if rc != 0:
        msg = lib().kfvm_last_error().decode(errors="replace")
        raise KfvmError(f"{what} failed ({rc}): {msg}")


def err_est_noalloc(eq, u_dev_ptr, uhat_dev_ptr, n, atol, rtol, out_dev_ptr, stream=0):
    """kfvm_err_est_noalloc: error estimate into out_dev (2 doubles) without allocating."""
    _check(lib().kfvm_err_est_noalloc(int(eq), C.c_void_p(u_dev_ptr), C.c_void_p(uhat_dev_ptr),
                                      int(n), float(atol), float(rtol), C.c_void_p(out_dev_ptr),
                                      C.c_void_p(stream)), "kfvm_err_est_noalloc")


def stencil(cfg):
    """Stencil geometry and reconstruction weights (host FP64, LAPACK LU)."""
    st = abi.KfvmStencil()
    _check(lib().kfvm_stencil_build(C.byref(cfg), C.byref(st)), "kfvm_stencil_build")
    return st


class Solver:
    """One solver on the current CUDA device (Solver::Solver .. Solver::Solve)."""

    def __init__(self, cfg):
        self.cfg = cfg
        self.nv = abi.nvars(cfg)
        self.n = abi.ncells(cfg)
        h = C.c_void_p()
        _check(lib().kfvm_create(C.byref(cfg), C.byref(h)), "kfvm_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().kfvm_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def init_ic(self, ic_kind, seed=12345):
        _check(lib().kfvm_init_ic(self.h, int(ic_kind), C.c_uint64(seed)), "kfvm_init_ic")

    def set_state(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64).reshape(self.nv, self.n)
        _check(lib().kfvm_set_state(self.h, u.ctypes.data), "kfvm_set_state")

    def get_state(self, out=None):
        u = out if out is not None else np.empty((self.nv, self.n), dtype=np.float64)
        _check(lib().kfvm_get_state(self.h, u.ctypes.data), "kfvm_get_state")
        return u

    def eval_rhs(self, t=0.0):
        r = np.empty((self.nv, self.n), dtype=np.float64)
        mv = C.c_double()
        _check(lib().kfvm_eval_rhs(self.h, float(t), r.ctypes.data, C.addressof(mv)), "kfvm_eval_rhs")
        return r, mv.value

    def err_est(self, u_dev_ptr, uhat_dev_ptr):
        """Error estimate of two device arrays (SoA interior): (err, posmin)."""
        e, p = C.c_double(), C.c_double()
        _check(lib().kfvm_err_est(self.h, C.c_void_p(u_dev_ptr), C.c_void_p(uhat_dev_ptr),
                                  C.addressof(e), C.addressof(p)), "kfvm_err_est")
        return e.value, p.value

    def take_step(self):
        info = abi.KfvmStepInfo()
        _check(lib().kfvm_take_step(self.h, C.byref(info)), "kfvm_take_step")
        return info

    def solve(self, max_steps):
        info = abi.KfvmStepInfo()
        n = C.c_int64()
        _check(lib().kfvm_solve(self.h, int(max_steps), C.byref(n), C.byref(info)), "kfvm_solve")
        return n.value, info

    def time_dt(self):
        t, dt = C.c_double(), C.c_double()
        _check(lib().kfvm_get_time(self.h, C.addressof(t), C.addressof(dt)), "kfvm_get_time")
        return t.value, dt.value

    def set_time(self, t, dt):
        _check(lib().kfvm_set_time(self.h, float(t), float(dt)), "kfvm_set_time")

    def set_indicator(self, ind):
        _check(lib().kfvm_set_indicator(self.h, int(ind)), "kfvm_set_indicator")

    def set_precision(self, prec):
        """abi.KFVM_PREC_FP64 (default) or abi.KFVM_PREC_TF32X3 (tensor-core stencil sums)."""
        _check(lib().kfvm_set_precision(self.h, int(prec)), "kfvm_set_precision")

    def faces(self, d):
        c = self.cfg
        nz = c.nz if c.dim == 3 else 1
        fd = [c.nx + (d == 0), c.ny + (d == 1), nz + (d == 2)]
        nqf = c.nq if c.dim == 2 else c.nq * c.nq
        out = np.empty((2, nqf, self.nv, fd[0] * fd[1] * fd[2]), dtype=np.float64)
        _check(lib().kfvm_get_faces(self.h, int(d), out.ctypes.data), "kfvm_get_faces")
        return out

    def flags(self):
        a = np.empty(self.n, dtype=np.uint8)
        th = np.empty(self.n, dtype=np.float64)
        _check(lib().kfvm_get_flags(self.h, a.ctypes.data, th.ctypes.data), "kfvm_get_flags")
        return a, th

    def stream_handle(self):
        h = C.c_void_p()
        _check(lib().kfvm_get_stream(self.h, C.byref(h)), "kfvm_get_stream")
        return h.value or 0

    def set_timing(self, on=True):
        _check(lib().kfvm_set_timing(self.h, 1 if on else 0), "kfvm_set_timing")

    def timing(self):
        """Per kernel class: (device ms, launches) since set_timing(True)."""
        ms = np.zeros(len(KCLASS), dtype=np.float64)
        ln = np.zeros(len(KCLASS), dtype=np.int64)
        _check(lib().kfvm_get_timing(self.h, ms.ctypes.data, ln.ctypes.data), "kfvm_get_timing")
        return {k: (float(ms[i]), int(ln[i])) for i, k in enumerate(KCLASS)}

    def launch_count(self):
        n = C.c_int64()
        _check(lib().kfvm_get_launch_count(self.h, C.byref(n)), "kfvm_get_launch_count")
        return n.value

    def last_step_ms(self):
        ms = C.c_double()
        _check(lib().kfvm_last_stage_ms(self.h, C.addressof(ms)), "kfvm_last_stage_ms")
        return ms.value
