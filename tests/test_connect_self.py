"""Self-connections of the random connectors follow the reference's rule,
checked against tests/golden/self_connections.npz (made by the reference's
own connectors, tests/golden/make_golden.py). The reference leaves out
pre == post pairs only when pre and post are the same object
(ANNarchy/core/ConnectorMethods.py:283-284, 344-345, 410-411): a view
connected to its own population keeps them, and so do two views of the same
neurons made separately. The device connectors get the same decision
(its exclude_self flag)."""
import os

import numpy as np
import pytest

from annarchy_b200 import Network, Neuron

GOLDEN = np.load(os.path.join(os.path.dirname(__file__), "golden", "self_connections.npz"))

CASES = {
    # key: (kind, population size, pre slice, post slice, argument); as in make_golden.py
    "fp_view_to_pop": ("fixed_probability", 60, (40, 60), None, 0.3),
    "fp_pop_to_view": ("fixed_probability", 60, None, (10, 30), 0.3),
    "fp_pop_to_pop": ("fixed_probability", 60, None, None, 0.3),
    "fp_same_view": ("fixed_probability", 60, (0, 40), "same", 0.3),
    "fp_two_views": ("fixed_probability", 60, (0, 40), (0, 40), 0.3),
    "fnpre_view_to_pop": ("fixed_number_pre", 60, (40, 60), None, 10),
    "fnpre_pop_to_pop": ("fixed_number_pre", 60, None, None, 10),
    "fnpost_view_to_pop": ("fixed_number_post", 60, None, (40, 60), 10),
    "fnpost_pop_to_pop": ("fixed_number_post", 60, None, None, 10),
}


def _build(key, device=False):
    kind, size, pre_sl, post_sl, arg = CASES[key]
    net = Network(dt=0.1, seed=int(GOLDEN[key + "__seed"]))
    if device:
        net.config(precision="double", device_connectors=True)
    pop = net.create(size, Neuron(parameters="r = 0.0"))
    pre = pop if pre_sl is None else pop[pre_sl[0]:pre_sl[1]]
    post = pre if post_sl == "same" else (pop if post_sl is None else pop[post_sl[0]:post_sl[1]])
    proj = net.connect(pre, post, "exc")
    getattr(proj, kind)(arg, 1.0)
    return proj


def _self_pairs(proj):
    m = proj._csr.tocoo()
    return int(np.sum(proj.post_ranks_view[m.row] == proj.pre_ranks[m.col]))


@pytest.mark.parametrize("key", [k for k in CASES if k.startswith("fp_")])
def test_fixed_probability_rows_equal_the_reference(key):
    """Same generator seed, same per-post Bernoulli draws: the dendrites
    (post ranks, sizes, pre ranks) equal the reference's LIL."""
    proj = _build(key)
    post, row_ptr, cols, _ = proj.csr_population_ranks()
    assert np.array_equal(post, GOLDEN[key + "__post"])
    assert np.array_equal(np.diff(row_ptr), GOLDEN[key + "__sizes"])
    assert np.array_equal(cols, GOLDEN[key + "__pre"])
    assert _self_pairs(proj) == int(GOLDEN[key + "__self_pairs"])


@pytest.mark.parametrize("key", [k for k in CASES if k.startswith("fn")])
def test_fixed_number_self_pairs_follow_the_reference(key):
    """fixed_number_pre/post draw differently from the reference; the rule
    is the same: self pairs occur exactly when the reference has some."""
    proj = _build(key)
    want = int(GOLDEN[key + "__self_pairs"])
    got = _self_pairs(proj)
    assert (got > 0) == (want > 0), (got, want)


@pytest.mark.parametrize("key", ["fp_view_to_pop", "fp_pop_to_pop", "fp_same_view",
                                 "fp_two_views", "fnpre_view_to_pop", "fnpre_pop_to_pop"])
def test_device_connector_gets_the_same_decision(key):
    proj = _build(key, device=True)
    assert proj._device_conn["exclude_self"] == (int(GOLDEN[key + "__self_pairs"]) == 0)
