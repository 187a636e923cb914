"""User boundary conditions written once for both back ends (numpy arrays on the
oracle, CUDA tensors on the CUDA path): the callbacks of kfvm_set_user_bc.

Cell layout: inner / outer are (NV, 2 * positions): [v][layer][position], layer h
of inner = interior cell h (low side) or n - 2 + h (high side), layer h of outer
= halo cell h - 2 (low) or n + h (high).  Face layout: [q][v][point], the
same buffer viewed as (NQF, NV, points).
"""
import kfvm_abi as abi

# the reflecting and no-slip coefficient tables (src/physics/*/*_BCCoeffs.H)
def wall_coefs(bc, axis, nv):
    c = [1.0] * nv
    if bc == abi.KFVM_BC_REFLECTING:
        c[1 + axis] = -1.0
        if nv == 9:
            c[5 + axis] = -1.0
    elif bc == abi.KFVM_BC_NOSLIP:
        c[1] = c[2] = c[3] = -1.0
        if nv == 9:
            c[5 + axis] = -1.0
    return c


def mirror_wall(bcs, nv, nqf, log=None):
    """A user function that reproduces the built-in outflow / reflecting / no-slip
    faces: halo cell -1 - m mirrors interior cell m with the wall's sign flips
    (so halo layer h takes interior layer 1 - h on both sides), and the outer face
    state is the inner one with the same flips.  bcs[face] = built-in type."""
    def fn(kind, face, time, inner, outer):
        if log is not None:
            log.append((kind, face, time))
        c = wall_coefs(bcs[face], face // 2, nv)
        if kind == abi.KFVM_USER_CELLS:
            a = inner.reshape(nv, 2, -1)
            b = outer.reshape(nv, 2, -1)
            for v in range(nv):
                b[v, 0] = c[v] * a[v, 1]
                b[v, 1] = c[v] * a[v, 0]
        else:
            a = inner.reshape(nqf, nv, -1)
            b = outer.reshape(nqf, nv, -1)
            for v in range(nv):
                b[:, v] = c[v] * a[:, v]
    return fn


def inflow(state, nqf, nv):
    """Supersonic inflow: a fixed state in every halo cell and outer face point of
    the faces it serves (the DoubleMach problem's western boundary, as a user writes
    it in UserBCs.H)."""
    def fn(kind, face, time, inner, outer):
        if kind == abi.KFVM_USER_CELLS:
            b = outer.reshape(nv, -1)
        else:
            b = outer.reshape(nqf, nv, -1)
        for v in range(nv):
            if kind == abi.KFVM_USER_CELLS:
                b[v] = state[v]
            else:
                b[:, v] = state[v]
    return fn
