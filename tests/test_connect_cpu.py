"""Device connectors on the CPU: the restated fixed-probability sampler has
the reference connector's distribution (independent Bernoulli pairs), and
the projection API routes large projections to the device connector."""
import numpy as np
import pytest

from annarchy_b200 import Network, Neuron, Uniform
from connect_emulation import fixed_probability, u01


def test_u01_range_and_independence():
    u = u01(7, np.arange(100000), 3, 3)
    assert u.min() >= 0.0 and u.max() < 1.0
    assert abs(u.mean() - 0.5) < 0.005 and abs(u.var() - 1 / 12) < 0.002
    v = u01(7, np.arange(100000), 4, 3)
    assert abs(np.corrcoef(u, v)[0, 1]) < 0.02


@pytest.mark.parametrize("p", [0.02, 0.3, 1.0])
def test_fixed_probability_is_bernoulli(p):
    n_post, n_pre = 3000, 500
    rp, col, w = fixed_probability(n_post, 0, 0, 0, n_pre, p, 12345, False)
    deg = np.diff(rp)
    # in-degree Binomial(n_pre, p)
    assert abs(deg.mean() - n_pre * p) < 4 * np.sqrt(n_pre * p * (1 - p) / n_post) + 1e-9
    if p < 1.0:
        assert abs(deg.var() / (n_pre * p * (1 - p)) - 1.0) < 0.1
    else:
        assert np.all(deg == n_pre)
    # ascending, distinct, in range; pre neurons hit uniformly
    same_row = np.repeat(np.arange(n_post), deg)
    assert np.all((np.diff(col) > 0) | (np.diff(same_row) > 0))
    assert col.min() >= 0 and col.max() < n_pre
    hits = np.bincount(col, minlength=n_pre)
    assert abs(hits.mean() - n_post * p) < 1e-9 + 4 * np.sqrt(n_post * p)
    if 0 < p < 1.0:
        assert abs(hits.var() / (n_post * p * (1 - p)) - 1.0) < 0.25


def test_fixed_probability_self_and_offsets():
    rp, col, _ = fixed_probability(400, 100, 0, 0, 600, 0.5, 3, True)
    rows = np.repeat(np.arange(400), np.diff(rp)) + 100
    assert not np.any(col == rows)
    # rows are keyed by row_offset + row: a shard of rows draws the same rows
    rp2, col2, _ = fixed_probability(150, 250, 150, 0, 600, 0.5, 3, True)
    assert np.array_equal(col2, col[rp[150]:rp[300]])
    assert np.array_equal(np.diff(rp2), np.diff(rp)[150:300])


def test_fixed_probability_weights():
    rp, col, w = fixed_probability(2000, 0, 0, 0, 300, 0.1, 9, False, wkind=1, a=0.2, b=0.5)
    assert w.min() >= 0.2 and w.max() < 0.5 and abs(w.mean() - 0.35) < 0.005
    rp, col, w = fixed_probability(2000, 0, 0, 0, 300, 0.1, 9, False, wkind=2, a=1.0, b=0.1)
    assert abs(w.mean() - 1.0) < 0.005 and abs(w.std() - 0.1) < 0.005


def test_projection_routes_to_device_connector():
    from annarchy_b200.core.backend import CompiledNetwork
    net = Network(dt=0.1, seed=1)
    net.config(precision="float", device_connectors=True)
    a = net.create(1000, Neuron(equations="v = 0.0", spike="v > 1.0"))
    b = net.create(800, Neuron(equations="dv/dt = -v + g_exc", spike="v > 1.0"))
    proj = net.connect(a, b, "exc").fixed_probability(0.05, Uniform(0.1, 0.2))
    assert proj._device_conn["kind"] == "fixed_probability"
    assert proj._device_conn["wkind"] == 1 and not proj._device_conn["exclude_self"]
    be = CompiledNetwork(net, dry=True)
    be.build()
    assert proj._nnz == 40000 and be.layout[proj.id]["post_chunks"] >= 2
