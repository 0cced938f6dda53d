"""Attribute access of compiled networks: known answers of the reference's
test suite restated against this backend's API and run on the GPU (values
read and written through the device arrays):

* tests_python/Neuron/test_Population1D.py:64-240 - coordinates, local and
  population-level parameters by array, `get`/`set`, neuron and view; init
  values, listings of attributes; reset;
* tests_python/Neuron/test_IndividualNeuron.py:46-80 and
  test_PopulationView.py:46-90 - 2D coordinates, unions of neurons, rows and
  columns of an 8 x 8 population;
* tests_python/RateSynapse/test_Dendrite.py:67-300 - dendrites of a default
  and of an Oja-like synapse: pre ranks, size, weights by dendrite and by
  synapse, postsynaptic and synaptic parameters, get/set by name."""
import numpy as np
import pytest

from annarchy_b200 import Network, Neuron, Parameter, Synapse, Uniform

pytestmark = pytest.mark.gpu


def _pop1d():
    net = Network(dt=1.0, seed=1)
    p1 = net.create(3, Neuron(parameters=dict(tau=Parameter(10, locality="local")),
                              equations="r += t/tau"))
    p2 = net.create(3, Neuron(parameters=dict(tau=10), equations="r += t/tau : init = 1.0"))
    p3 = net.create(3, Neuron(parameters=dict(tau=10, r_init=1.0),
                              equations="r += t/tau : init = r_init"))
    net.compile()
    return net, p1, p2, p3


def test_population_1d_access():
    net, p1, p2, p3 = _pop1d()
    assert tuple(p1.coordinates_from_rank(1)) == (1,)
    assert p1.rank_from_coordinates((1,)) == 1
    np.testing.assert_array_equal(p1.tau, [10.0] * 3)
    np.testing.assert_array_equal(p1.get("tau"), [10.0] * 3)
    assert p1.neuron(1).tau == 10.0
    p1.tau = 5.0
    np.testing.assert_array_equal(p1.tau, [5.0] * 3)
    p1.set({"tau": 7.0})
    np.testing.assert_array_equal(p1.tau, [7.0] * 3)
    p1.neuron(1).tau = 20
    assert p1.neuron(1).tau == 20.0
    p1.tau = 10.0
    p1[1:3].tau = 5.0
    np.testing.assert_array_equal(p1.tau, [10.0, 5.0, 5.0])
    assert p2.tau == 10.0
    assert p1.attributes == ["tau", "r"] and p1.parameters == ["tau"] and p1.variables == ["r"]
    np.testing.assert_array_equal(p1.r, [0.0] * 3)
    assert p1.neuron(0).r == 0.0
    np.testing.assert_array_equal(p2.r, [1.0] * 3)
    np.testing.assert_array_equal(p3.r, [1.0] * 3)
    p1.r = 1.0
    np.testing.assert_array_equal(p1.r, [1.0] * 3)
    p1.r = 0.0
    p1[1:3].r = 2.0
    np.testing.assert_array_equal(p1.r, [0.0, 2.0, 2.0])
    p1.r = Uniform(0.0, 1.0).get_values(3)
    assert np.all((np.asarray(p1.r) >= 0.0) & (np.asarray(p1.r) <= 1.0))
    p1.set({"r": 1.0})
    np.testing.assert_array_equal(p1.r, [1.0] * 3)
    # reset: back to the values after compile()
    p1.tau = 5.0
    net.reset()
    np.testing.assert_array_equal(p1.tau, [10.0] * 3)
    np.testing.assert_array_equal(p1.r, [0.0] * 3)
    net.close()


def test_individual_neurons_and_views_2d():
    net = Network(dt=1.0, seed=1)
    pop = net.create((8, 8), Neuron(parameters="tau = 10", equations="r += 1/tau * t"))
    net.compile()
    trio = pop[2, 2] + pop[3, 3] + pop[4, 4]
    np.testing.assert_array_equal(trio.r, [0.0] * 3)
    trio.r = 1.0
    np.testing.assert_array_equal((pop[2, 2] + pop[3, 3] + pop[4, 4]).r, [1.0] * 3)
    assert pop[2, 4].rank == 20
    net.reset()
    np.testing.assert_array_equal(pop[:, 2].r, np.zeros(8))
    pop[:, 2].r = 1.0
    np.testing.assert_array_equal(pop[:, 2].r, np.ones(8))
    np.testing.assert_array_equal(pop[:, 4].ranks, [4, 12, 20, 28, 36, 44, 52, 60])
    np.testing.assert_array_equal(pop[2, :].ranks, [16, 17, 18, 19, 20, 21, 22, 23])
    assert isinstance(pop[2, :].ranks, np.ndarray)
    net.close()


def _dendrite_net(synapse=None):
    net = Network(dt=1.0, seed=1)
    pop1 = net.create(5, Neuron(parameters="tau = 10", equations="r += 1/tau * t"))
    pop2 = net.create(8, Neuron(parameters="tau = 10: population",
                                equations="r += 1/tau * t: init = 1.0"))
    proj = net.connect(pre=pop1, post=pop2, target="exc", synapse=synapse)
    proj.all_to_all(weights=1.0, force_multiple_weights=True)
    net.compile()
    return net, proj


def test_dendrites_of_the_default_synapse():
    net, proj = _dendrite_net()
    with pytest.raises(Exception):
        proj.dendrite(14)
    assert list(proj.dendrite(5).pre_ranks) == [0, 1, 2, 3, 4]
    assert proj.dendrite(3).size == 5
    np.testing.assert_array_equal(proj.dendrite(7).w, [1.0] * 5)
    proj.dendrite(6).w = 2.0
    np.testing.assert_array_equal(proj.dendrite(6).w, [2.0] * 5)
    proj.dendrite(6)[2].w = 3.0
    np.testing.assert_array_equal(proj.dendrite(6).w, [2.0, 2.0, 3.0, 2.0, 2.0])
    net.close()


def test_dendrites_of_a_learning_synapse():
    oja = Synapse(parameters="""
        tau = 5000.0 : postsynaptic
        alpha = 8.0
    """, equations="tau * dw/dt = pre.r * post.r - alpha * post.r^2 * w")
    net, proj = _dendrite_net(oja)
    assert list(proj.dendrite(5).pre_ranks) == [0, 1, 2, 3, 4]
    assert proj.dendrite(3).size == 5
    np.testing.assert_array_equal(proj.dendrite(1).tau, 5000.0)
    np.testing.assert_array_equal(proj.dendrite(0).alpha, [8.0] * 5)
    np.testing.assert_array_equal(proj.dendrite(7).w, [1.0] * 5)
    proj.tau = 6000.0
    np.testing.assert_array_equal(proj.dendrite(0).tau, 6000.0)
    old = np.asarray(proj.tau, dtype=float).copy()
    old[1] = 7000.0
    proj.dendrite(1).tau = 7000.0
    np.testing.assert_array_equal(proj.dendrite(1).tau, 7000.0)
    np.testing.assert_array_equal(proj.tau, old)
    proj.dendrite(4).alpha = 9.0
    np.testing.assert_array_equal(proj.dendrite(4).alpha, [9.0] * 5)
    proj.dendrite(4)[1].alpha = 10.0
    np.testing.assert_array_equal(proj.dendrite(4).alpha, [9.0, 10.0, 9.0, 9.0, 9.0])
    proj.dendrite(6).w = 2.0
    proj.dendrite(6)[2].w = 3.0
    np.testing.assert_array_equal(proj.dendrite(6).w, [2.0, 2.0, 3.0, 2.0, 2.0])
    new = np.asarray(proj.tau, dtype=float).copy()
    new[2] = 7500.0
    proj.dendrite(2).set({"tau": 7500})
    np.testing.assert_array_equal(proj.tau, new)
    np.testing.assert_array_equal(proj.dendrite(1).get("tau"), 7000.0)
    net.close()


def _sparse_4x8():
    from scipy import sparse
    wm = sparse.lil_matrix((4, 8))
    for i in range(8):
        wm[1, i] = 0.2
    for i in range(2, 6):
        wm[3, i] = 0.5
    return wm.T


@pytest.mark.parametrize("modified", [False, True])
def test_projection_access(modified):
    """Weights, dendrites, size and post ranks of a from_sparse projection;
    with a synapse holding local, postsynaptic and projection-level
    parameters and a variable initialised from a parameter
    (tests_python/RateSynapse/test_Projection.py:15-230)."""
    net = Network(dt=1.0, seed=1)
    simple = Neuron(parameters="r=0")
    syn = Synapse(parameters="""
        loc_var        = 5000.0
        semi_glob_var  = 8.0    : postsynaptic
        glob_var       = 8.0    : projection
    """, equations="""
        dx/dt = -x              : init = loc_var
        dw/dt = -w
    """) if modified else None
    proj = net.connect(net.create(8, simple), net.create(4, simple), "exc", synapse=syn)
    proj.from_sparse(_sparse_4x8())
    net.compile()
    np.testing.assert_allclose(proj.w[0], 0.2)
    np.testing.assert_allclose(proj.w[1], 0.5)
    np.testing.assert_allclose(proj.dendrite(1).w, 0.2)
    np.testing.assert_allclose(proj.dendrite(3).w, 0.5)
    assert proj.size == 2 and list(proj.post_ranks) == [1, 3]
    if modified:
        np.testing.assert_array_equal(proj.loc_var[0], 5000.0)
        np.testing.assert_array_equal(proj.get("loc_var")[1], 5000.0)
        np.testing.assert_array_equal(proj.x[0], 5000.0)
        np.testing.assert_array_equal(proj.semi_glob_var, 8.0)
        np.testing.assert_array_equal(proj.get("glob_var"), 8.0)
    net.close()


def test_custom_connectivity_from_function():
    """Diagonal bands built by user functions returning a LILConnectivity,
    without delay, with a uniform delay of 2 ms and with per-synapse delays
    DiscreteUniform(1, 5) (tests_python/RateSynapse/
    test_RateCustomConnectivity.py:15-200); the sums of the band through
    the projection without delay are checked after two steps."""
    from annarchy_b200 import DiscreteUniform, LILConnectivity

    def band(pre, post, dt, weight, delay=None):
        syn = LILConnectivity(dt=dt)
        for post_rk in post.ranks:
            ranks = [r for r in (post_rk - 1, post_rk, post_rk + 1) if r in pre.ranks]
            if delay is None:
                d = [0]
            elif isinstance(delay, (int, float)):
                d = [delay]
            else:
                d = delay.get_values(len(ranks))
            syn.add(post_rk, ranks, [weight] * len(ranks), d)
        return syn

    net = Network(dt=1.0, seed=1)
    pop1 = net.create(5, Neuron(equations="r = 1"))
    pop2 = net.create(5, Neuron(equations="r = sum(exc)"))
    p0 = net.connect(pre=pop1, post=pop2, target="exc")
    p0.from_function(method=band, weight=0.1)
    p1 = net.connect(pre=pop1, post=pop2, target="exc2")
    p1.from_function(method=band, weight=0.1, delay=2)
    p2 = net.connect(pre=pop1, post=pop2, target="exc3")
    p2.from_function(method=band, weight=0.1, delay=DiscreteUniform(1, 5))
    net.compile()
    assert p0.delay == 1.0 and p1.delay == 2.0
    assert [list(d.pre_ranks) for d in p0.dendrites] == [[0, 1], [0, 1, 2], [1, 2, 3], [2, 3, 4],
                                                          [3, 4]]
    net.simulate(2)
    np.testing.assert_allclose(np.ravel(pop2.r), [0.2, 0.3, 0.3, 0.3, 0.2], rtol=1e-12)
    net.close()
