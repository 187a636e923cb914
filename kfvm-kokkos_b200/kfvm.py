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
        L.kfvm_selftest_wait.argtypes = [D, C.POINTER(I32), C.POINTER(D)]
        L.kfvm_selftest_rcp.argtypes = [I64, C.c_uint64, C.POINTER(I64), C.POINTER(D)]
        L.kfvm_mlp_num_weights.argtypes = [I32]
        L.kfvm_mlp_init_weights.argtypes = [P, C.c_uint64]
        L.kfvm_mlp_set_weights.argtypes = [P, P, I64]
        L.kfvm_mlp_get_weights.argtypes = [P, P, I64]
        L.kfvm_mlp_reserve.argtypes = [P, I64]
        L.kfvm_mlp_collect.argtypes = [P, D, D, C.c_uint64, C.POINTER(I64), C.POINTER(I64)]
        L.kfvm_mlp_get_samples.argtypes = [P, I64, I64, P, P, P]
        L.kfvm_mlp_train.argtypes = [P, I32, I32, D, D, C.c_uint64, C.POINTER(D), C.POINTER(D)]
        L.kfvm_mlp_config.argtypes = [P, D, D, D, D]
        L.kfvm_mlp_probability.argtypes = [P, P]
        L.kfvm_mlp_stats.argtypes = [P, P]
        L.kfvm_get_faces.argtypes = [P, I32, P]
        L.kfvm_get_flags.argtypes = [P, P, P]
        L.kfvm_plotfile_write.argtypes = [C.POINTER(abi.KfvmConfig), C.c_char_p, C.c_char_p, I32, I32, I32, D, D,
                                          P, P, P]
        L.kfvm_plotfile_read.argtypes = [C.POINTER(abi.KfvmConfig), C.c_char_p, P, P, P, C.POINTER(I32),
                                         C.POINTER(D), C.POINTER(D)]
        L.kfvm_write_plotfile.argtypes = [P, C.c_char_p, C.c_char_p, I32, I32, I32]
        L.kfvm_restart.argtypes = [P, C.c_char_p, C.POINTER(I32)]
        L.kfvm_set_plot_freq.argtypes = [P, D, I32]
        L.kfvm_last_stage_ms.argtypes = [P, P]
        L.kfvm_get_stream.argtypes = [P, C.POINTER(C.c_void_p)]
        L.kfvm_set_timing.argtypes = [P, I32]
        L.kfvm_get_timing.argtypes = [P, P, P]
        L.kfvm_get_launch_count.argtypes = [P, C.POINTER(I64)]
        L.kfvm_measure_fp64_mma.argtypes = [C.POINTER(D)]
        L.kfvm_get_same_state.argtypes = [P, C.POINTER(C.c_int32), C.POINTER(I64), C.POINTER(I64)]
        L.kfvm_flow_stats.argtypes = [P, P, C.POINTER(I32)]
        L.kfvm_forcing_num_modes.argtypes = [I32]
        L.kfvm_forcing_draw.argtypes = [I32, C.c_uint32, P]
        L.kfvm_set_forcing.argtypes = [P, C.POINTER(abi.KfvmForcing)]
        L.kfvm_apply_forcing.argtypes = [P, P, P, P]
        L.kfvm_block_config.argtypes = [C.POINTER(abi.KfvmConfig), I32, C.POINTER(abi.KfvmConfig),
                                        C.POINTER(I32)]
        L.kfvm_set_exchange.argtypes = [P, abi.EXCHANGE_FN, abi.ALLREDUCE_FN, P]
        L.kfvm_set_user_bc.argtypes = [P, abi.USER_BC_FN, P]
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


def measure_fp64_mma():
    """kfvm_measure_fp64_mma: FP64 tensor-pipe throughput of this GPU (TFLOP/s)."""
    t = C.c_double()
    _check(lib().kfvm_measure_fp64_mma(C.byref(t)), "kfvm_measure_fp64_mma")
    return t.value


def selftest_wait(limit_s):
    """kfvm_selftest_wait: (gave_up, seconds waited) of a bounded wait that cannot complete."""
    g, w = C.c_int32(), C.c_double()
    _check(lib().kfvm_selftest_wait(float(limit_s), C.byref(g), C.byref(w)), "kfvm_selftest_wait")
    return bool(g.value), w.value


def selftest_rcp(n=1 << 24, seed=5):
    """kfvm_selftest_rcp: (max ulp distance of the Riemann reciprocal from 1/y,
    max relative difference of x * rcp(y) from x / y) over n random doubles."""
    u, q = C.c_int64(), C.c_double()
    _check(lib().kfvm_selftest_rcp(int(n), int(seed), C.byref(u), C.byref(q)), "kfvm_selftest_rcp")
    return u.value, q.value


def forcing_num_modes(dim):
    n = lib().kfvm_forcing_num_modes(int(dim))
    if n < 0:
        _check(n, "kfvm_forcing_num_modes")
    return n


def forcing_draw(dim, seed32):
    """kfvm_forcing_draw: one mode table [n][dim][3] = (k_d, real, imaginary)."""
    m = np.empty((forcing_num_modes(dim), dim, 3), dtype=np.float64)
    _check(lib().kfvm_forcing_draw(int(dim), int(seed32) & 0xFFFFFFFF, m.ctypes.data), "kfvm_forcing_draw")
    return m


def plotfile_write(cfg, directory, base, num, u, weno, theta, time=0.0, time_step=0, dt=0.0, ckpt=False):
    """kfvm_plotfile_write from host arrays: u [nv][n] float64, weno [n] 0/1, theta [n]."""
    nv, n = abi.nvars(cfg), abi.ncells(cfg)
    u = np.ascontiguousarray(u, dtype=np.float64).reshape(nv, n)
    w = np.ascontiguousarray(weno, dtype=np.uint8).reshape(n)
    th = np.ascontiguousarray(theta, dtype=np.float64).reshape(n)
    _check(lib().kfvm_plotfile_write(C.byref(cfg), str(directory).encode(), str(base).encode(), int(num),
                                     1 if ckpt else 0, int(time_step), float(time), float(dt), u.ctypes.data,
                                     w.ctypes.data, th.ctypes.data), "kfvm_plotfile_write")
    return os.path.join(str(directory), f"{base}_{int(num):07d}.xmf")


def plotfile_read(cfg, xmf_path):
    """kfvm_plotfile_read: dict with u [nv][n], weno [n], theta [n], time_step, time, dt."""
    nv, n = abi.nvars(cfg), abi.ncells(cfg)
    u = np.empty((nv, n), dtype=np.float64)
    w = np.empty(n, dtype=np.uint8)
    th = np.empty(n, dtype=np.float64)
    ts, t, h = C.c_int32(), C.c_double(), C.c_double()
    _check(lib().kfvm_plotfile_read(C.byref(cfg), str(xmf_path).encode(), u.ctypes.data, w.ctypes.data,
                                    th.ctypes.data, C.byref(ts), C.byref(t), C.byref(h)), "kfvm_plotfile_read")
    return {"u": u, "weno": w, "theta": th, "time_step": ts.value, "time": t.value, "dt": h.value}


def stencil(cfg):
    """Stencil geometry and reconstruction weights (host FP64, LAPACK LU)."""
    st = abi.KfvmStencil()
    _check(lib().kfvm_stencil_build(C.byref(cfg), C.byref(st)), "kfvm_stencil_build")
    return st


class _CudaBytes:
    """A device byte range in the CUDA array interface, for torch.as_tensor."""

    def __init__(self, ptr, nbytes):
        self.__cuda_array_interface__ = {"shape": (int(nbytes),), "typestr": "|u1",
                                         "data": (int(ptr), False), "version": 3}


def block_config(blocks, rank):
    """Rank `rank`'s configuration of a decomposed domain and the ranks across its six
    faces (-1: none): the reference's LayoutMPI::distributeBlocks.  `blocks` holds
    one block's cells, the whole domain's extents and nb."""
    out = abi.KfvmConfig()
    nbr = (C.c_int32 * 6)()
    _check(lib().kfvm_block_config(C.byref(blocks), int(rank), C.byref(out), nbr), "kfvm_block_config")
    return out, list(nbr)


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
        # at interpreter shutdown the module globals may already be gone
        try:
            self.close()
        except Exception:
            pass

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

    def set_user_bc(self, fn):
        """Install user boundary conditions (the faces configured KFVM_BC_USER):
        fn(kind, face, time, inner, outer) gets the packed inner values and fills
        outer in place, both float64 CUDA tensors of shape (NV, points) with the
        layouts of kfvm_set_user_bc.  fn may raise to fail the step."""
        import torch
        dev = torch.device("cuda", torch.cuda.current_device())

        def cb(user, kind, face, time, inner, outer, npts, stream):
            try:
                nb = int(npts) * self.nv * 8
                a = torch.as_tensor(_CudaBytes(inner, nb), device=dev).view(torch.float64).view(self.nv, -1)
                b = torch.as_tensor(_CudaBytes(outer, nb), device=dev).view(torch.float64).view(self.nv, -1)
                fn(int(kind), int(face), float(time), a, b)
                torch.cuda.current_stream(dev).synchronize()   # the solver's stream reads outer next
                return 0
            except Exception as e:  # noqa: BLE001 - reported through the return code
                self.user_bc_error = e
                return 1

        self._user_bc = abi.USER_BC_FN(cb)
        self.user_bc_error = None
        _check(lib().kfvm_set_user_bc(self.h, self._user_bc, None), "kfvm_set_user_bc")

    def set_exchange(self, transport):
        """Install a transport (decomp.DistExchange or a LocalExchange endpoint) whose
        exchange_fn / allreduce_fn carry this block's boundary data between ranks."""
        self._transport = transport  # the callbacks must outlive the solver's use of them
        _check(lib().kfvm_set_exchange(self.h, transport.exchange_fn, transport.allreduce_fn, None),
               "kfvm_set_exchange")

    def set_indicator(self, ind):
        _check(lib().kfvm_set_indicator(self.h, int(ind)), "kfvm_set_indicator")

    def set_precision(self, prec):
        """abi.KFVM_PREC_FP64 (default) or abi.KFVM_PREC_TF32X3 (tensor-core stencil sums)."""
        _check(lib().kfvm_set_precision(self.h, int(prec)), "kfvm_set_precision")

    # ---- learned troubled-cell indicator
    def mlp_num_weights(self):
        return lib().kfvm_mlp_num_weights(self.cfg.dim)

    def mlp_init(self, seed=1):
        _check(lib().kfvm_mlp_init_weights(self.h, C.c_uint64(seed)), "kfvm_mlp_init_weights")

    def mlp_set_weights(self, w_bf16):
        w = np.ascontiguousarray(w_bf16, dtype=np.uint16)
        _check(lib().kfvm_mlp_set_weights(self.h, w.ctypes.data, w.size), "kfvm_mlp_set_weights")

    def mlp_weights(self):
        w = np.empty(self.mlp_num_weights(), dtype=np.uint16)
        _check(lib().kfvm_mlp_get_weights(self.h, w.ctypes.data, w.size), "kfvm_mlp_get_weights")
        return w

    def mlp_reserve(self, capacity):
        _check(lib().kfvm_mlp_reserve(self.h, int(capacity)), "kfvm_mlp_reserve")

    def mlp_collect(self, tau=0.3, keep=0.1, seed=7):
        n, p = C.c_int64(), C.c_int64()
        _check(lib().kfvm_mlp_collect(self.h, float(tau), float(keep), C.c_uint64(seed), C.byref(n), C.byref(p)),
               "kfvm_mlp_collect")
        return n.value, p.value

    def mlp_samples(self, first, count):
        ni = 2 * (25 if self.cfg.dim == 2 else 125)
        f = np.empty((count, ni), dtype=np.uint16)
        lab = np.empty(count, dtype=np.uint8)
        cells = np.empty(count, dtype=np.int64)
        _check(lib().kfvm_mlp_get_samples(self.h, int(first), int(count), f.ctypes.data, lab.ctypes.data,
                                          cells.ctypes.data), "kfvm_mlp_get_samples")
        return f, lab, cells

    def mlp_train(self, steps, batch=1024, lr=3e-3, pos_weight=4.0, seed=11):
        a, b = C.c_double(), C.c_double()
        _check(lib().kfvm_mlp_train(self.h, int(steps), int(batch), float(lr), float(pos_weight), C.c_uint64(seed),
                                    C.byref(a), C.byref(b)), "kfvm_mlp_train")
        return a.value, b.value

    def mlp_config(self, prob_threshold=0.5, judge_frac=1.0 / 256, tau=0.3, miss_limit=0.25):
        _check(lib().kfvm_mlp_config(self.h, float(prob_threshold), float(judge_frac), float(tau),
                                     float(miss_limit)), "kfvm_mlp_config")

    def mlp_probability(self):
        out = np.empty(self.n, dtype=np.float32)
        _check(lib().kfvm_mlp_probability(self.h, out.ctypes.data), "kfvm_mlp_probability")
        return out

    def mlp_stats(self):
        out = np.zeros(6, dtype=np.int64)
        _check(lib().kfvm_mlp_stats(self.h, out.ctypes.data), "kfvm_mlp_stats")
        keys = ["judged", "troubled", "missed", "false_alarm", "fallback_events", "fallback_steps_left"]
        return dict(zip(keys, out.tolist()))

    def faces(self, d):
        c = self.cfg
        nz = c.nz if c.dim == 3 else 1
        fd = [c.nx + (d == 0), c.ny + (d == 1), nz + (d == 2)]
        nqf = c.nq if c.dim == 2 else c.nq * c.nq
        out = np.empty((2, nqf, self.nv, fd[0] * fd[1] * fd[2]), dtype=np.float64)
        _check(lib().kfvm_get_faces(self.h, int(d), out.ctypes.data), "kfvm_get_faces")
        return out

    def write_plotfile(self, directory, base, num, ckpt=False, time_step=0):
        """kfvm_write_plotfile: the current state as an XDMF + binary file set; returns the .xmf path."""
        _check(lib().kfvm_write_plotfile(self.h, str(directory).encode(), str(base).encode(), int(num),
                                         1 if ckpt else 0, int(time_step)), "kfvm_write_plotfile")
        return os.path.join(str(directory), f"{base}_{int(num):07d}.xmf")

    def restart(self, xmf_path):
        """kfvm_restart from a checkpoint; returns its time step."""
        ts = C.c_int32()
        _check(lib().kfvm_restart(self.h, str(xmf_path).encode(), C.byref(ts)), "kfvm_restart")
        return ts.value

    def flow_stats(self):
        """kfvm_flow_stats: volume-averaged kinetic energy, enstrophy (GLM-MHD: and
        current helicity) of the current state."""
        out = np.zeros(3, dtype=np.float64)
        n = C.c_int32()
        _check(lib().kfvm_flow_stats(self.h, out.ctypes.data, C.byref(n)), "kfvm_flow_stats")
        return out[:n.value].copy()

    def set_forcing(self, forcing):
        """kfvm_set_forcing with an abi.KfvmForcing (None disables)."""
        _check(lib().kfvm_set_forcing(self.h, C.byref(forcing) if forcing is not None else None),
               "kfvm_set_forcing")

    def apply_forcing(self, modes=None):
        """kfvm_apply_forcing: force the current state once (a new draw when modes is
        None); returns (mode table used, strength)."""
        dim = self.cfg.dim
        out = np.empty((forcing_num_modes(dim), dim, 3), dtype=np.float64)
        mi = None if modes is None else np.ascontiguousarray(modes, dtype=np.float64)
        s = C.c_double()
        _check(lib().kfvm_apply_forcing(self.h, None if mi is None else mi.ctypes.data, out.ctypes.data,
                                        C.byref(s)), "kfvm_apply_forcing")
        return out, s.value

    def set_plot_freq(self, plot_freq, plot_num):
        _check(lib().kfvm_set_plot_freq(self.h, float(plot_freq), int(plot_num)), "kfvm_set_plot_freq")

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

    def same_state(self):
        """(on, sampled, equal) of the equal-state Riemann variant."""
        on, n, e = C.c_int32(), C.c_int64(), C.c_int64()
        _check(lib().kfvm_get_same_state(self.h, C.byref(on), C.byref(n), C.byref(e)), "kfvm_get_same_state")
        return bool(on.value), n.value, e.value

    def last_step_ms(self):
        ms = C.c_double()
        _check(lib().kfvm_last_stage_ms(self.h, C.addressof(ms)), "kfvm_last_stage_ms")
        return ms.value
