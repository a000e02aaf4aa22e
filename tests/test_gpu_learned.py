"""The learned correction of the diagonal step (gccu_lp_*): its device
kernels against the CPU restatement in oracle/mlp.py (loss and gradient over
a training set at 1e-10 relative, sampled rows at 1e-12, the corrected step,
whose perceptron runs in FP32, at 1e-5),
training lowers the loss, and on held-out instances of a small stream of
synthetic CCSD Hamiltonians the learned step reaches |dE| < 1 uEh in fewer
iterations than plain diagonal + DIIS, at the same converged energy."""
import numpy as np
import pytest

import gccu
import learned
import mlp
from cases import random_list

pytestmark = pytest.mark.gpu


@pytest.fixture
def engine(built):
    e = gccu.Engine(0)
    yield e
    e.close()


def _rows(n, seed):
    rng = np.random.default_rng(seed)
    x = np.stack([rng.uniform(0.1, 3.0, n), rng.uniform(0.1, 5.0, n), rng.uniform(-3, 3, n)], 1)
    s = rng.normal(0.0, 0.1, n)
    target = s * rng.uniform(0.0, 1.5, n)
    rows = np.concatenate([x, s[:, None], np.zeros((n, 1))], 1)
    return rows, target


def test_gradient_matches_cpu(engine):
    w = mlp.init_weights(3, out_scale=0.5)
    rows, target = _rows(1000, 4)  # not a multiple of the 128 rows of a block
    engine.lp_set_weights(w)
    engine.lp_load_samples(rows, target)
    g, loss = engine.lp_gradient()
    lref, gref = mlp.loss_and_gradient(w, rows[:, :3], rows[:, 3], target)
    assert abs(loss - lref) <= 1e-12 * abs(lref)
    assert np.max(np.abs(g - gref)) <= 1e-10 * np.max(np.abs(gref))
    assert np.linalg.norm(g - gref) <= 1e-10 * np.linalg.norm(gref)


def test_training_lowers_the_loss(engine):
    # targets a smooth function of the inputs times the plain step: learnable
    rows, _ = _rows(20000, 5)
    target = rows[:, 3] * (0.6 + 0.3 * np.tanh(rows[:, 0] - 0.5 * rows[:, 2]))
    w0 = mlp.init_weights(6)
    engine.lp_set_weights(w0)
    engine.lp_load_samples(rows, target)
    _, l0 = engine.lp_gradient()
    engine.lp_train(300, 1024, 3e-3, seed=7)
    w1 = engine.lp_get_weights()
    _, l1 = engine.lp_gradient()
    assert l1 < 0.5 * l0
    assert l1 == pytest.approx(mlp.loss_and_gradient(w1, rows[:, :3], rows[:, 3], target)[0],
                               rel=1e-12)


def test_step_and_rows_match_cpu(engine):
    from cases import SPACES
    from cc import PPHH
    nsym, norb = SPACES["c2v"]
    engine.register_orbinfo(nsym, norb)
    op = engine.define_operator([PPHH])
    lists = [engine.register_list(op) for _ in range(5)]
    (lo, n), (li, _), (ld, _), (lp, _), (la, _) = lists
    r, d, p, a = (random_list(n, 20), 0.3 + np.abs(random_list(n, 21)), random_list(n, 22),
                  random_list(n, 23))
    d[::7] = -d[::7]
    d[5] = -2e-11  # clamped as in diavc
    for lid, x in ((li, r), (ld, d), (lp, p), (la, a)):
        engine.upload(lid, x)
    w = mlp.init_weights(8, out_scale=0.5)
    engine.lp_set_weights(w)
    for prev, pv in ((lp, p), (0, None)):
        engine.lp_precondition(lo, li, ld, prev, fac=-1.0, shift=0.05)
        got = engine.download(lo, n)
        ref = mlp.step(w, r, d, pv, fac=-1.0, shift=0.05)
        # the perceptron runs in FP32 in the solve's step: its factor to ~1e-6
        assert np.max(np.abs(got - ref)) <= 1e-5 * np.max(np.abs(ref))
    idx = np.random.default_rng(9).choice(n, 50, replace=False)
    rows = engine.lp_rows(li, ld, lp, la, idx, fac=-1.0, shift=0.05)
    x, s = mlp.inputs(r, d, p, fac=-1.0, shift=0.05)
    ref = np.concatenate([x[idx], s[idx, None], a[idx, None]], 1)
    assert np.max(np.abs(rows - ref)) <= 1e-12 * np.max(np.abs(ref))
    with pytest.raises(gccu.GccuError, match="out of range"):
        engine.lp_rows(li, ld, lp, la, [n], fac=-1.0)


def test_learned_step_needs_fewer_iterations(built):
    # a small stream of the benchmark family's distribution: 16 training
    # instances solved with plain diagonal + DIIS (sampled), 8 held out
    insts = learned.stream(24, seed=5000, nocc=(3, 6), nvir=(12, 24))
    rows, targets = [], []
    for inst in insts[:16]:
        e = gccu.Engine(0)
        try:
            smp = learned.Sampler(seed=inst["seed"])
            s = learned.solve(e, inst, sampler=smp)
            if s.history[-1][2] < 1e-8:
                r, t = smp.targets(s)
                rows.append(r)
                targets.append(t)
        finally:
            e.close()
    assert len(rows) >= 12
    e = gccu.Engine(0)
    try:
        w, l0, l1 = learned.train(e, np.concatenate(rows), np.concatenate(targets))
    finally:
        e.close()
    assert l1 < l0
    plain, learn = [], []
    for inst in insts[16:]:
        res = []
        for weights in (None, w):
            e = gccu.Engine(0)
            try:
                s = learned.solve(e, inst, weights=weights)
                res.append((s.history, s.fallbacks))
            finally:
                e.close()
        e_ref = res[0][0][-1][1]
        assert abs(res[1][0][-1][1] - e_ref) < 1e-8  # the same converged energy
        plain.append(learned.iterations_to(res[0][0], e_ref))
        learn.append(learned.iterations_to(res[1][0], e_ref))
    assert None not in plain and None not in learn
    assert np.mean(learn) < np.mean(plain), (plain, learn)
