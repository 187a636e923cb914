"""CPU checks of the learned indicator's checkers: the oracle's label (WENO
weight departure) and the numpy feature / BF16 helpers."""
import numpy as np

import kfvm_abi as abi
import mlp_ref


def test_departure_zero_on_uniform_and_large_at_a_jump(oracle_lib):
    import oracle
    cfg, ic = abi.workload("sod3d", scale=16, steps=1)
    o = oracle.OracleSolver(cfg)
    o.init_ic(ic)
    dep = o.weno_departure().reshape(16, 16, 16)
    # the sphere of radius 0.2 about the centre: cells far from its surface are uniform
    x = (np.arange(16) + 0.5) / 16 - 0.5
    r = np.sqrt(x[:, None, None] ** 2 + x[None, :, None] ** 2 + x[None, None, :] ** 2)
    far = np.abs(r - 0.2) > 0.2
    near = np.abs(r - 0.2) < 0.5 / 16
    assert dep[far].max() == 0.0
    assert dep[near].max() > 0.3
    assert (dep >= 0).all() and (dep <= 1).all()
    del o


def test_departure_small_on_smooth_flow(oracle_lib):
    import oracle
    cfg, ic = abi.workload("taylor_green", scale=16, steps=1)
    o = oracle.OracleSolver(cfg)
    o.init_ic(ic)
    assert o.weno_departure().max() < 0.3
    del o


def test_bf16_helpers_and_features():
    x = np.array([1.0, -2.5, 3.14159, 1e-3, 0.0], dtype=np.float32)
    b = mlp_ref.f32_to_bf16(x)
    y = mlp_ref.bf16_to_f32(b)
    assert np.all(np.abs(y - x) <= np.abs(x) * 2.0 ** -8)
    assert mlp_ref.bf16_to_f32(mlp_ref.f32_to_bf16(np.float32(1.0)))[()] == 1.0
    # a density ramp in x: features are the normalised ramp, pressure flat
    cfg = abi.make_config(2, abi.KFVM_EQ_HYDRO, 8, 8, bc="outflow")
    n = 64
    u = np.zeros((5, n))
    xs = np.tile(np.arange(8, dtype=float), 8)
    u[0] = 1.0 + 0.01 * xs
    u[4] = 2.5
    f = mlp_ref.features(u, cfg, [3 * 8 + 4])[0]
    fr = f[:25].reshape(5, 5)
    # max |drho| = 0.02 at rho_c = 1.04: scale 1 / (0.02 + 1e-4 * 1.04)
    s = 0.02 / (0.02 + 1e-4 * 1.04)
    assert np.allclose(fr[2], s * np.array([-1.0, -0.5, 0.0, 0.5, 1.0]), atol=1e-6)
    assert np.allclose(f[25:], 0.0, atol=1e-6)
