"""Pins of the CPU oracle (no GPU needed).

The reference ships no tests or golden outputs, so the oracle is pinned by what
the reference itself defines: its quadrature and RK tables (extracted from its
source text into tests/golden/reference_tables.json), the self-checks its weight
code carries (polynomial reproduction, as in the unused testPV of
src/stencil/Stencil.cpp:250-277, and the symmetry mapping), conservation, and
the convergence study of its isentropic-vortex example
(exec/Hydro/IsenVort/sweepN.sh, l1Errors.py).
"""
import json
import math
import os

import numpy as np
import pytest

import kfvm_abi as abi

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "reference_tables.json")))


@pytest.mark.parametrize("nq", [1, 2, 3])
def test_quadrature_tables(nq, oracle_lib):
    ab, wt, _ = oracle_lib.tables(nq, abi.KFVM_RK_SSP4_3_2)
    assert ab == GOLD["quad"][str(nq)]["ab"]
    assert wt == GOLD["quad"][str(nq)]["wt"]


@pytest.mark.parametrize("rk,name", [(abi.KFVM_RK_SSP4_3_2, "SSP4_3_2"),
                                     (abi.KFVM_RK_SSP10_4_3, "SSP10_4_3"),
                                     (abi.KFVM_RK_THREESTARP, "ThreeStarP"),
                                     (abi.KFVM_RK_FOURSTARP, "FourStarP")])
def test_rk_tables(rk, name, oracle_lib):
    _, _, t = oracle_lib.tables(2, rk)
    g = GOLD["rk"][name]
    assert t["nStages"] == g["nStages"]
    for k in ("gam1", "gam2", "gam3", "delta", "beta", "bhat", "c"):
        assert t[k] == g[k], k
    for k in ("bhatfsal", "ep1", "ep2"):
        assert t[k] == g[k], k


def _mono_avg(p, x):
    return ((x + 0.5) ** (p + 1) - (x - 0.5) ** (p + 1)) / (p + 1)


def _degrees(dim, tot):
    out = []
    for t in range(tot + 1):
        for i in range(t + 1):
            if dim == 2:
                out.append((i, t - i, 0))
            else:
                for j in range(t - i + 1):
                    out.append((i, j, t - i - j))
    return out


def _stencil(dim, oracle_lib, lfac=5.0, n=16):
    name = "isentropic_vortex" if dim == 2 else "sod3d"
    cfg, _ = abi.workload(name, scale=n)
    cfg.lfac = lfac
    return cfg, oracle_lib.stencil(cfg)


def _sub_offsets(st, s, dim):
    off = np.array(st.off)[:, :st.n_cells].T.astype(float)
    if s < 2:
        m = st.n_cells if s == 0 else st.n_cells_ctr
        return off[:m]
    idx = np.array(st.sub_idx)[s - 2, :st.n_cells_bias]
    return off[idx]


@pytest.mark.parametrize("dim", [2, 3])
def test_face_weights_reproduce_polynomials(dim, oracle_lib):
    """Face-point weights of each substencil reproduce the point values of the
    monomials in its polynomial space (degree 3 full, 1 central/biased)."""
    cfg, st = _stencil(dim, oracle_lib)
    fw = np.array(st.face_w)
    nqf = st.nqf
    ab = GOLD["quad"]["2"]["ab"]
    for s in range(st.n_sub):
        deg = 3 if s == 0 else 1
        offs = _sub_offsets(st, s, dim)
        m = len(offs)
        for f in range(2 * dim):
            for q in range(nqf):
                a = ab[q] if dim == 2 else ab[q // 2]
                b = 0.0 if dim == 2 else ab[q % 2]
                pt = [[-0.5, a, b], [0.5, a, b], [a, -0.5, b], [a, 0.5, b], [a, b, -0.5], [a, b, 0.5]][f]
                w = fw[s, f, q, :m]
                for (p0, p1, p2) in _degrees(dim, deg):
                    avg = np.array([_mono_avg(p0, o[0]) * _mono_avg(p1, o[1]) *
                                    (_mono_avg(p2, o[2]) if dim == 3 else 1.0) for o in offs])
                    exact = pt[0] ** p0 * pt[1] ** p1 * (pt[2] ** p2 if dim == 3 else 1.0)
                    assert abs(w @ avg - exact) < 1e-8, (s, f, q, (p0, p1, p2))


@pytest.mark.parametrize("dim", [2, 3])
def test_derivative_weights_keep_reference_functional(dim, oracle_lib):
    """Derivative weights of the full stencil reproduce the reference's derivative
    functional of each monomial.  That functional (Monomials.cpp:29) passes its
    recursion arguments swapped, so d2/dx2 of x^3 at 0 evaluates to 3, not 0;
    the weights must carry that quirk (scaled by dx^px dy^py dz^pz)."""
    cfg, st = _stencil(dim, oracle_lib)
    dw = np.array(st.deriv_w)
    offs = _sub_offsets(st, 0, dim)
    h = [(cfg.xup - cfg.xlo) / cfg.nx, (cfg.yup - cfg.ylo) / cfg.ny,
         (cfg.zup - cfg.zlo) / (cfg.nz if dim == 3 else 1)]

    def nderiv(p, N, x):  # the reference's recursion, swap included
        if N == 0:
            return x ** p
        if N > p:
            return 0.0
        return p * nderiv(p - 1, int(x), float(N - 1))

    dset = _degrees(dim, 2 if dim == 2 else 3)[1:]
    for i, Nd in enumerate(dset):
        w = dw[0, i, :st.n_cells]
        scl = h[0] ** Nd[0] * h[1] ** Nd[1] * (h[2] ** Nd[2] if dim == 3 else 1.0)
        for (p0, p1, p2) in _degrees(dim, 3):
            avg = np.array([_mono_avg(p0, o[0]) * _mono_avg(p1, o[1]) *
                            (_mono_avg(p2, o[2]) if dim == 3 else 1.0) for o in offs])
            want = nderiv(p0, Nd[0], 0.0) * nderiv(p1, Nd[1], 0.0) * \
                (nderiv(p2, Nd[2], 0.0) if dim == 3 else 1.0)
            assert abs(w @ avg - scl * want) < 1e-6 * max(1.0, abs(scl * want)), (Nd, (p0, p1, p2))
    # the quirk itself: second x-derivative of x^3 at the centre is 3, not 0
    assert nderiv(3, 2, 0.0) == 3.0


@pytest.mark.parametrize("dim", [2, 3])
def test_symmetry_mapped_weights(dim, oracle_lib):
    """Weights copied through the reference's symmetry maps equal direct mirrors:
    the east face of the full stencil is the x-reflection of the west face."""
    cfg, st = _stencil(dim, oracle_lib)
    fw = np.array(st.face_w)
    off = np.array(st.off)[:, :st.n_cells].T
    mirror = [int(np.where((off == [-o[0], o[1], o[2]]).all(axis=1))[0][0]) for o in off]
    w_west = fw[0, 0, :st.nqf, :st.n_cells]
    w_east = fw[0, 1, :st.nqf, :st.n_cells]
    assert np.array_equal(w_east, w_west[:, mirror])


def test_stencil_geometry(oracle_lib):
    """Cell counts of StencilInfo.H:22-84 for radius 2."""
    for dim, counts in ((2, (13, 5, 5, 6, 4, 5)), (3, (33, 7, 11, 8, 6, 19))):
        _, st = _stencil(dim, oracle_lib)
        assert (st.n_cells, st.n_cells_ctr, st.n_cells_bias, st.n_sub, st.n_bias, st.n_indic) == counts


@pytest.mark.parametrize("name,scale", [("kelvin_helmholtz", 32), ("orszag_tang", 32),
                                        ("taylor_green", 10)])
def test_oracle_conservation(name, scale, oracle_lib):
    cfg, ic = abi.workload(name, scale=scale, steps=3)
    s = oracle_lib.OracleSolver(cfg)
    s.init_ic(ic)
    u0 = s.get_state().sum(axis=1)
    s.solve(cfg.max_steps)
    u1 = s.get_state().sum(axis=1)
    # Navier-Stokes: the reference adds u.(div tau) to the energy equation
    # (NavierStokes_K.H:385-404), which is not a flux difference, so only mass and
    # momentum are conserved there
    nchk = 4 if cfg.eq == abi.KFVM_EQ_NAVIERSTOKES else len(u0)
    assert np.all(np.abs(u1 - u0)[:nchk] <= 1e-12 * np.abs(u0).max())


def _vortex_exact(cfg, t):
    """Cell averages (8x8 Gauss) of the vortex advected by (t, t) on the periodic box."""
    g = (cfg.gamma)
    n = cfg.nx
    L = cfg.xup - cfg.xlo
    dx = L / n
    xg, wg = np.polynomial.legendre.leggauss(8)
    xg, wg = xg / 2, wg / 2
    xc = cfg.xlo + dx * (np.arange(n) + 0.5)
    X = (xc[:, None] + dx * xg[None, :]).ravel()
    W = np.outer(np.ones(n), wg).ravel()
    x = X[None, :] - t
    y = X[:, None] - t
    x = (x - cfg.xlo) % L + cfg.xlo
    y = (y - cfg.ylo) % L + cfg.ylo
    beta = 5.0
    r2 = x ** 2 + y ** 2
    T = 1.0 - (g - 1) * beta ** 2 / (8 * g * math.pi ** 2) * np.exp(1 - r2)
    rho = T ** (1 / (g - 1))
    ww = np.outer(W, W)
    avg = (rho * ww).reshape(n, 8, n, 8).sum(axis=(1, 3))
    return avg  # [y][x]


@pytest.mark.parametrize("nq", [2, 3])
def test_isentropic_vortex_convergence(nq, oracle_lib):
    """Density L1 error against the advected exact solution drops at high order
    (the reference's convergence sweep, exec/Hydro/IsenVort/sweepN.sh), with the
    2- and the 3-point Gauss rule."""
    errs = []
    for n in (32, 64):
        cfg, ic = abi.workload("isentropic_vortex", scale=n, steps=10000)
        cfg.nq = nq
        cfg.final_time = 0.5
        cfg.atol = cfg.rtol = 1e-8
        s = oracle_lib.OracleSolver(cfg)
        s.init_ic(ic)
        s.solve(cfg.max_steps)
        t, _ = s.time_dt()
        assert abs(t - 0.5) < 1e-12
        rho = s.get_state()[0].reshape(n, n)
        errs.append(np.abs(rho - _vortex_exact(cfg, t)).mean())
    eoc = math.log2(errs[0] / errs[1])
    assert eoc > 3.0, (errs, eoc)


def _walls(cfg, names):
    codes = {"periodic": abi.KFVM_BC_PERIODIC, "outflow": abi.KFVM_BC_OUTFLOW,
             "reflecting": abi.KFVM_BC_REFLECTING, "noslip": abi.KFVM_BC_NOSLIP}
    for f, n in enumerate(names):
        cfg.bc[f] = codes[n]
    return cfg


@pytest.mark.parametrize("name,scale,walls", [
    ("kelvin_helmholtz", 24, ["periodic", "periodic", "reflecting", "reflecting"] + ["periodic"] * 2),
    ("sod3d", 10, ["reflecting"] * 6),
    ("taylor_green", 10, ["noslip"] * 6),
])
def test_oracle_walls_conserve_mass(name, scale, walls, oracle_lib):
    """Reflecting and no-slip walls (BoundaryConditions_K.H:75-95, 549-570 with the
    <Eq>_BCCoeffs.H tables) pass no mass: the mirrored states give a zero contact
    speed, so the total mass stays constant to rounding (outflow would not).
    GLM-MHD is left out: its HLL speeds take min(v_R, v_Roe) in the upper Wu-Shu
    bound as the reference writes it (MHD_GLM_Riemann.H:87), so the mirrored
    states' fan is not symmetric and some mass crosses the wall there too."""
    cfg, ic = abi.workload(name, scale=scale, steps=3)
    _walls(cfg, walls)
    s = oracle_lib.OracleSolver(cfg)
    s.init_ic(ic)
    m0 = s.get_state()[0].sum()
    s.solve(cfg.max_steps)
    u1 = s.get_state()
    assert np.all(np.isfinite(u1))
    assert abs(u1[0].sum() - m0) <= 1e-12 * abs(m0)


@pytest.mark.parametrize("dim,n,rs", [(2, 16, abi.KFVM_RS_LLF), (3, 8, abi.KFVM_RS_HLL)])
def test_oracle_srhydro_conserves_periodic(dim, n, rs, oracle_lib):
    """SRHydro on a periodic smooth flow: D, S and E are conserved to rounding (the
    flux differences telescope) and every state stays admissible: D > 0 and
    E^2 > D^2 + |S|^2 (SRHydro_EOS.H:238-250)."""
    cfg = abi.make_config(dim, abi.KFVM_EQ_SRHYDRO, n, n, n, gamma=5.0 / 3.0, rs=rs, cfl=0.8, steps=4)
    s = oracle_lib.OracleSolver(cfg)
    s.init_ic(abi.KFVM_IC_SMOOTH_WAVE)
    u0 = s.get_state()
    s.solve(cfg.max_steps)
    u1 = s.get_state()
    assert np.all(np.isfinite(u1))
    tot0, tot1 = u0.sum(axis=1), u1.sum(axis=1)
    scale = np.abs(u0).sum(axis=1)
    assert np.all(np.abs(tot1 - tot0) <= 1e-12 * scale), (tot1 - tot0) / scale
    assert np.all(u1[0] > 0.0)
    assert np.all(u1[4] ** 2 > u1[0] ** 2 + (u1[1:4] ** 2).sum(axis=0))


def test_oracle_sr_shock_tube_plateaus(oracle_lib):
    """SRShockTube (exec/SRHydro/SRShockTube) before the waves reach the outflow
    ends: mass is conserved, the undisturbed states keep their initial values, and
    D stays between the two initial densities (the limiter bounds face values, so
    cell averages may cross the bounds by rounding-sized amounts of the RK stages)."""
    cfg, ic = abi.workload("sr_shock_tube", scale=64, steps=12)
    s = oracle_lib.OracleSolver(cfg)
    s.init_ic(ic)
    u0 = s.get_state()
    s.solve(cfg.max_steps)
    u1 = s.get_state().reshape(5, 4, 4, 64)
    assert abs(u1[0].sum() - u0[0].sum()) <= 1e-12 * u0[0].sum()
    d = u1[0, 0, 0]
    assert np.all(u1[0] == u1[0, :1, :1])           # uniform across y and z
    assert d[0] == 10.0 and d[-1] == 1.0
    assert d.min() >= 1.0 - 1e-6 and d.max() <= 10.0 + 1e-6
    assert np.all(np.diff(d) <= 1e-6)               # D falls from left to right
