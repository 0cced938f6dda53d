"""Host-side projection, population and network API against the reference:
a connectivity file written by the reference's save_connectivity() loads
into the same dense matrix and receptive fields (fixtures made by
tests/golden/make_golden.py), files written here load back, and the
dendrite, coordinate and accessor helpers."""
import os

import numpy as np
import pytest

from annarchy_b200 import Network, Neuron

HERE = os.path.join(os.path.dirname(__file__), "golden")
META = np.load(os.path.join(HERE, "connectivity_file_meta.npz"))


def _net():
    net = Network(dt=0.5)
    a = net.create((3, 5), Neuron(parameters="r = 0.0"), name="A")
    b = net.create((4, 3), Neuron(equations="r = sum(exc)"), name="B")
    return net, a, b


def test_from_reference_connectivity_file():
    net, a, b = _net()
    p = net.connect(a, b, "exc").from_file(os.path.join(HERE, "connectivity_ref.npz"))
    np.testing.assert_array_equal(p.connectivity_matrix(), META["matrix"])
    np.testing.assert_array_equal(p.receptive_fields(), META["rf"])
    assert p.uniform_delay == 3 and p.nb_synapses == 53


def test_save_connectivity_round_trip(tmp_path):
    net, a, b = _net()
    p = net.connect(a, b, "exc").from_file(os.path.join(HERE, "connectivity_ref.npz"))
    for ext in (".npz", ".gz", ".pkl"):
        path = str(tmp_path / ("c" + ext))
        p.save_connectivity(path)
        net2, a2, b2 = _net()
        q = net2.connect(a2, b2, "exc").from_file(path)
        np.testing.assert_array_equal(q.connectivity_matrix(), META["matrix"])
        assert q.delay == p.delay


def test_dendrites_and_synapses():
    net, a, b = _net()
    p = net.connect(a, b, "exc").from_file(os.path.join(HERE, "connectivity_ref.npz"))
    sizes = p.nb_synapses_per_dendrite()
    assert sum(sizes) == 53 and len(sizes) == p.size
    d = p.dendrite(2)
    m = META["matrix"]
    assert d.pre_ranks == list(np.nonzero(m[2])[0])
    np.testing.assert_array_equal(d.w, m[2][d.pre_ranks])
    assert p.dendrite((0, 2)).post_rank == 2 and p[(0, 2)].size == d.size
    syn = p.synapse(d.pre_ranks[1], 2)
    assert syn.w == m[2, d.pre_ranks[1]]
    syn.w = 5.0
    assert p.connectivity_matrix()[2, d.pre_ranks[1]] == 5.0
    assert p.synapse(int(np.nonzero(m[2] == 0)[0][0]), 2) is None
    assert [x.post_rank for x in p.dendrites] == p.post_ranks
    rf = d.receptive_field()
    assert rf.shape == (3, 5) and rf.ravel()[d.pre_ranks[0]] == d.w[0]


def test_coordinates_and_accessors():
    net, a, b = _net()
    assert a.rank_from_coordinates((2, 3)) == 13 and a.coordinates_from_rank(13) == (2, 3)
    assert a.normalized_coordinates_from_rank(13) == (1.0, float(np.float32(3 / 4)))
    with pytest.raises(ValueError):
        a.rank_from_coordinates((3, 0))
    assert a.dimension == 2
    p = net.connect(a, b, "exc").all_to_all(0.5)
    assert net.get_population("B") is b and net.get_projection(p.name) is p
    assert net.get_projections(post=b) == [p] and net.get_projections(pre=b, suppress_error=True) == []
    assert net.time == 0.0


def test_global_synaptic_attributes():
    """Projection-level parameters and variables read and assign through
    get/set (before compile they are kept for the device arrays)."""
    from annarchy_b200 import Synapse
    net, a, b = _net()
    syn = Synapse(parameters="eta = 0.02 : projection",
                  equations="dbeta/dt = -beta : projection, init=1.0\ndw/dt = eta * beta")
    p = net.connect(a, b, "exc", synapse=syn).all_to_all(0.5)
    assert p.beta == 1.0 and p.eta == 0.02
    p.beta = 0.25
    p.eta = 0.5
    assert "beta" not in p.__dict__ and p.beta == 0.25 and p.get("eta") == 0.5


def test_save_load_semiglobal(tmp_path):
    """Per-dendrite (post-synaptic) variables are saved as one value per
    dendrite and loaded back."""
    from annarchy_b200 import Synapse
    syn = Synapse(parameters="eta = 0.02 : projection",
                  equations=["dalpha/dt = -alpha : postsynaptic", "dw/dt = eta * alpha"])
    net, a, b = _net()
    p = net.connect(a, b, "exc", synapse=syn).all_to_all(0.5)
    p.alpha = np.arange(12.0)
    path = str(tmp_path / "p.npz")
    p.save(path)
    net2, a2, b2 = _net()
    q = net2.connect(a2, b2, "exc", synapse=syn).all_to_all(0.1)
    q.load(path)
    np.testing.assert_array_equal(q.alpha, np.arange(12.0))
    np.testing.assert_array_equal(q.get("w", flat=True), np.full(180, 0.5))
