"""Learned format selector: CPU restatement of the network's gradients
(finite differences), GPU kernels against it, training, and the gain of the
trained selector over the reference's fixed rule on held-out timings."""
import json
import os

import numpy as np
import pytest

from annarchy_b200 import selector as S
from annarchy_b200 import tuning

DATASET = os.path.join(os.path.dirname(S.__file__), "data", "selector_dataset.json")


def _problem(seed=0, n=37, n_in=13, hidden=16, n_out=9):
    rng = np.random.default_rng(seed)
    p = S.init_params(n_in, hidden, n_out, seed)
    x = rng.normal(size=(n, n_in)).astype(np.float32)
    t = rng.normal(size=(n, n_out)).astype(np.float32)
    m = (rng.random((n, n_out)) < 0.6).astype(np.float32)
    return p, x, t, m, n_in, hidden, n_out


def test_reference_gradient_matches_finite_differences():
    p, x, t, m, a, h, o = _problem(n=11, n_in=5, hidden=7, n_out=4)
    p = p.astype(np.float64)
    _, g = S.reference_loss_grad(p, x, t, m, a, h, o)
    eps = 1e-6
    for i in range(0, p.size, 3):
        q = p.copy()
        q[i] += eps
        lp = S.reference_loss_grad(q, x, t, m, a, h, o)[0]
        q[i] -= 2 * eps
        lm = S.reference_loss_grad(q, x, t, m, a, h, o)[0]
        assert abs((lp - lm) / (2 * eps) - g[i]) <= 1e-6 * max(1.0, abs(g[i]))


def test_fit_rejects_wrong_shapes():
    sel = S.Selector(hidden=8, seed=0)
    X = np.zeros((5, sel.n_in))
    with pytest.raises(ValueError):
        sel.fit(X, np.zeros((5, sel.n_out - 1)), np.ones((5, sel.n_out - 1)))


def test_features_and_feasibility():
    import scipy.sparse as sp
    rng = np.random.default_rng(0)
    m = sp.random(2000, 1500, density=0.01, random_state=1, format="csr")
    f = tuning.features(m)
    assert f.shape == (len(tuning.FEATURE_NAMES),) and np.all(np.isfinite(f))
    assert tuning.feasible(m, {"format": "csr"})
    dense_rows = sp.csr_matrix((np.ones(3000), (np.zeros(3000, int), np.arange(3000))),
                               shape=(3000, 3000))
    assert not tuning.feasible(dense_rows, {"format": "ell"})   # one long row: huge padding


def test_heuristic_is_the_reference_rule():
    import scipy.sparse as sp
    short = sp.random(1000, 1000, density=0.05, random_state=2, format="csr")
    long_rows = sp.random(1000, 1000, density=0.3, random_state=3, format="csr")
    assert tuning.heuristic(short) == "sell_1"
    assert tuning.heuristic(short, plastic=True) == "ellr"
    assert tuning.heuristic(long_rows) == "csr"
    assert tuning.heuristic_schedule(short) == {"format": "sell", "sell_sigma": 1}
    assert tuning.schedule_name(tuning.heuristic_schedule(short)) == "sell_1"
    assert tuning.heuristic_schedule(long_rows) == {"format": "csr"}


@pytest.mark.gpu
def test_gpu_gradient_matches_reference():
    p, x, t, m, a, h, o = _problem()
    l_ref, g_ref = S.reference_loss_grad(p, x, t, m, a, h, o)
    l_gpu, g_gpu = S.gpu_loss_grad(p, x, t, m, a, h, o)
    assert abs(l_gpu - l_ref) <= 1e-5 * max(1.0, abs(l_ref))
    np.testing.assert_allclose(g_gpu, g_ref, rtol=1e-4, atol=1e-5 * np.abs(g_ref).max())


@pytest.mark.gpu
def test_gpu_training_fits():
    rng = np.random.default_rng(1)
    sel = S.Selector(hidden=32, seed=3)
    X = rng.normal(size=(200, sel.n_in))
    W = rng.normal(size=(sel.n_in, sel.n_out))
    Y = np.tanh(X @ W) * 0.5
    M = np.ones_like(Y)
    loss0 = float(((Y - Y.mean(0)) ** 2).mean())
    loss = sel.fit(X, Y, M, epochs=1500, lr=3e-3)
    assert loss < 0.1 * loss0
    pred = sel.predict(X)
    assert float(((pred - Y) ** 2).mean()) == pytest.approx(loss, rel=0.2, abs=1e-4)


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(DATASET), reason="no timing dataset collected")
def test_selector_beats_reference_rule_on_held_out_matrices():
    """Trained on timings of one half of the matrices, the selector's
    schedules are faster on the other half than the reference's rule."""
    records = json.load(open(DATASET))
    X, Y, M, tags = S.Selector.table(records)
    # matrices cycle through four structures: hold out every other group of four
    idx = np.array([int(t.split("/")[0].split("_")[1]) for t in tags])
    test = (idx // 4) % 2 == 1
    sel = S.Selector(hidden=64, seed=0)
    sel.fit(X[~test], Y[~test], M[~test], epochs=3000, lr=3e-3)
    choice = sel.choose_index(X[test], M[test])
    reg_mlp = S.regret(choice, Y[test], M[test])
    heur = []
    for j in np.nonzero(test)[0]:
        name = tuning_heuristic_from_record(records, tags[j], X[j])
        heur.append(S.SCHEDULE_NAMES.index(name) if name in S.SCHEDULE_NAMES else 0)
    reg_heur = S.regret(np.array(heur), Y[test], M[test])
    g_mlp = float(np.exp(np.mean(np.log(np.minimum(reg_mlp, 1e3)))))
    g_heur = float(np.exp(np.mean(np.log(np.minimum(reg_heur, 1e3)))))
    print(f"geometric-mean slowdown vs exhaustive: selector {g_mlp:.3f}, reference rule {g_heur:.3f}")
    assert g_mlp < g_heur
    assert g_mlp < 1.25


def tuning_heuristic_from_record(records, tag, feat):
    """The reference's rule from the recorded features: mean row length
    (10**log_mean_row) <= 128 -> SELL, else CSR."""
    mean = 10.0 ** feat[tuning.FEATURE_NAMES.index("log_mean_row")]
    return "sell_1" if mean <= 128 else "csr"
