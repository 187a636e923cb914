"""The learned troubled-cell indicator on the GPU, checked piece by piece:

* labels (WENO weight departure > tau) against the oracle's restatement,
* features (normalised density / pressure patch, BF16) against numpy,
* the network's probability (first layer on the tensor cores with BF16 features
  and weights, FP32 accumulation) against a float64 numpy forward pass with the
  same BF16 values,
* training (loss falls, troubled cells are recalled on the collected set),
* a run with the indicator in the stage (the judge counts, no failure) whose
  state stays close to the KXRCF run, and, on the isentropic vortex after one
  period, an L1 error against the exact solution within 1.05x of plain FP64.
"""
import numpy as np
import pytest

import kfvm_abi as abi
import mlp_ref

pytestmark = pytest.mark.gpu

TAU = 0.3


def _solver(cfg, ic, steps=0, prec=None):
    import kfvm
    s = kfvm.Solver(cfg)
    if prec is not None:
        s.set_precision(prec)
    s.init_ic(ic)
    for _ in range(steps):
        s.take_step()
    return s


@pytest.mark.parametrize("name,scale,steps", [("kelvin_helmholtz", 64, 6), ("sod3d", 20, 3),
                                              ("orszag_tang", 64, 6)])
def test_labels_and_features_match_references(name, scale, steps, product_lib, oracle_lib, gpu):
    import oracle
    cfg, ic = abi.workload(name, scale=scale, steps=steps + 2)
    s = _solver(cfg, ic, steps)
    u = s.get_state()
    n = abi.ncells(cfg)
    s.mlp_reserve(n)
    cnt, npos = s.mlp_collect(tau=TAU, keep=1.0, seed=3)
    assert cnt == n
    feats, lab, cells = s.mlp_samples(0, cnt)
    assert sorted(cells.tolist()) == list(range(n))
    o = oracle.OracleSolver(cfg)
    o.set_state(u)
    dep = o.weno_departure()[cells]
    clear = np.abs(dep - TAU) > 1e-9
    assert np.array_equal(lab[clear].astype(bool), dep[clear] > TAU), name
    assert npos == int(lab.sum())
    if name != "orszag_tang":
        assert npos > 0, name
    # features: numpy in float64 then FP32, rounded to BF16
    pick = np.arange(0, cnt, max(1, cnt // 400))
    ref = mlp_ref.f32_to_bf16(mlp_ref.features(u, cfg, cells[pick]))
    got = feats[pick]
    ulp = np.abs(mlp_ref.bf16_to_f32(got) - mlp_ref.bf16_to_f32(ref))
    scale_ = np.maximum(np.abs(mlp_ref.bf16_to_f32(ref)), 1e-30)
    assert (ulp <= scale_ * 2.0 ** -7 + 1e-30).all(), name
    assert (got == ref).mean() > 0.99, name
    s.close()
    del o


@pytest.mark.parametrize("name,scale", [("kelvin_helmholtz", 48), ("sod3d", 16)])
def test_probability_matches_numpy(name, scale, product_lib, gpu):
    cfg, ic = abi.workload(name, scale=scale, steps=4)
    s = _solver(cfg, ic, 2)
    s.mlp_init(seed=5)
    w = s.mlp_weights()
    assert w.size == s.mlp_num_weights()
    prob = s.mlp_probability()
    u = s.get_state()
    cells = np.arange(0, abi.ncells(cfg), 7)
    # the kernel feeds the tensor cores BF16 features, as training sees them
    x = mlp_ref.bf16_to_f32(mlp_ref.f32_to_bf16(mlp_ref.features(u, cfg, cells)))
    ref = mlp_ref.probability(w, x)
    assert np.abs(prob[cells] - ref).max() < 2e-4, name
    # weights round-trip through the ABI
    s.mlp_set_weights(w)
    assert np.array_equal(s.mlp_weights(), w)
    s.close()


def _trained_kh(scale=128, seed=1):
    """Train on samples of a plain KH run (every 8 steps of 32)."""
    cfg, ic = abi.workload("kelvin_helmholtz", scale=scale, steps=40)
    s = _solver(cfg, ic)
    s.mlp_reserve(400000)
    for step in range(33):
        if step % 8 == 0:
            s.mlp_collect(tau=TAU, keep=0.25, seed=100 + step)
        s.take_step()
    s.mlp_init(seed=seed)
    l0, l1 = s.mlp_train(600, batch=1024, lr=3e-3, pos_weight=4.0, seed=seed)
    return s, cfg, l0, l1


def test_training_learns_the_labels(product_lib, gpu):
    s, cfg, l0, l1 = _trained_kh()
    assert np.isfinite(l0) and np.isfinite(l1)
    assert l1 < 0.6 * l0, (l0, l1)
    n, npos = s.mlp_collect(tau=TAU, keep=0.0, seed=9)   # adds the positives of the last state
    feats, lab, _ = s.mlp_samples(0, n)
    p = mlp_ref.probability(s.mlp_weights(), mlp_ref.bf16_to_f32(feats))
    pos = lab == 1
    recall = (p[pos] > 0.5).mean()
    assert pos.sum() > 100 and recall > 0.8, (pos.sum(), recall)
    s.close()


def test_learned_indicator_in_the_stage(product_lib, gpu):
    trained, cfg, _, _ = _trained_kh()
    w = trained.mlp_weights()
    trained.close()
    cfg, ic = abi.workload("kelvin_helmholtz", scale=128, steps=30)
    ref = _solver(cfg, ic)
    mlp = _solver(cfg, ic)
    mlp.mlp_set_weights(w)
    mlp.mlp_config(prob_threshold=0.5, judge_frac=1.0 / 16, tau=TAU, miss_limit=0.25)
    mlp.set_indicator(abi.KFVM_IND_MLP)
    for _ in range(20):
        ia, ib = ref.take_step(), mlp.take_step()
        assert ib.accepted == 1
        if ia.dt != ib.dt:
            mlp.set_time(*ref.time_dt())   # keep both on the same time levels
    st = mlp.mlp_stats()
    assert st["judged"] > 0 and st["troubled"] > 0, st
    ua, ub = ref.get_state(), mlp.get_state()
    assert np.isfinite(ub).all()
    rel = np.abs(ub - ua)[[0, 4]].sum(axis=1) / np.abs(ua)[[0, 4]].sum(axis=1)
    assert rel.max() < 1e-2, rel
    ref.close()
    mlp.close()


def test_learned_fp32_vortex_error(product_lib, gpu):
    """Learned indicator + FP32 contraction on the isentropic vortex: L1 error
    against the exact solution after one period within 1.05x of plain FP64."""
    trained, _, _, _ = _trained_kh()
    w = trained.mlp_weights()
    trained.close()
    errs = {}
    for form in ("plain", "learned_fp32"):
        cfg, ic = abi.workload("isentropic_vortex", scale=64, steps=100000)
        cfg.final_time = abi.stof(10.0)
        s = _solver(cfg, ic, prec=abi.KFVM_PREC_TF32X3 if form != "plain" else None)
        exact = s.get_state().copy()
        if form != "plain":
            s.mlp_set_weights(w)
            s.set_indicator(abi.KFVM_IND_MLP)
            s.init_ic(abi.KFVM_IC_ISENTROPIC_VORTEX)
        s.solve(cfg.max_steps)
        errs[form] = np.abs(s.get_state() - exact).sum(axis=1)
        s.close()
    for v in (0, 1, 2, 4):
        assert errs["learned_fp32"][v] <= 1.05 * errs["plain"][v], (v, errs)


def test_mlp_arguments(product_lib, gpu):
    import kfvm
    cfg, ic = abi.workload("isentropic_vortex", scale=16, steps=2)
    s = _solver(cfg, ic)
    with pytest.raises(kfvm.KfvmError):
        s.set_indicator(abi.KFVM_IND_MLP)          # no weights yet
    with pytest.raises(kfvm.KfvmError):
        s.mlp_collect()                            # no buffer
    with pytest.raises(kfvm.KfvmError):
        s.mlp_set_weights(np.zeros(10, dtype=np.uint16))
    with pytest.raises(kfvm.KfvmError):
        s.mlp_config(prob_threshold=1.5)
    assert s.mlp_num_weights() == 2721
    s.close()
