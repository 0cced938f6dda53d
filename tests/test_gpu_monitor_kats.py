"""Monitor known answers of the reference's test suite
(ANNarchy tests_python/Neuron/test_Monitor.py:15-340), run through this
backend on the GPU: recording of a population, of views (slices, a union of
single neurons, a slice plus one neuron), a period of 10 steps, a monitor
created stopped and started later, pause/resume, spike recording with and
without a refractory period. The network also holds a rate-coded projection
whose synaptic equation is `w = t`, as the reference's test network does."""
import numpy as np
import pytest

from annarchy_b200 import Network, Neuron, Synapse

pytestmark = pytest.mark.gpu

RAMP = Neuron(equations="r = t")
COUNT_TO_5 = Neuron(equations="v = v + 1.0", spike="v == 5.0", reset="v = 3.0")
COUNT_TO_3_REFRACTORY = Neuron(equations="v = v + 1.0", spike="v == 3.0", reset="v = 1.0 ",
                               refractory=3.0)
W_EQUALS_T = Synapse(parameters="""
    tau = 5000.0
    alpha = 8.0
""", equations="w = t")


def _network(precision):
    net = Network(dt=1.0, seed=1)
    net.config(precision=precision)
    pop1 = net.create(3, RAMP)
    pop2 = net.create(5, RAMP)
    pop3 = net.create(3, COUNT_TO_5)
    pop4 = net.create(3, COUNT_TO_3_REFRACTORY)
    mons = dict(
        m=net.monitor(pop1, "r"),
        n=net.monitor(pop1[:2], "r"),
        o=net.monitor(pop1, "r", period=10.0),
        p=net.monitor(pop1, "r", start=False),
        q=net.monitor(pop1[0] + pop1[2], "r"),
        r=net.monitor(pop2[:2] + pop2.neuron(4), "r"),
        s=net.monitor(pop3, ["v", "spike"]),
        t=net.monitor(pop4, ["v", "spike"]),
    )
    net.connect(pre=pop1, post=pop2, target="exc", synapse=W_EQUALS_T).all_to_all(weights=1.0)
    net.compile()
    return net, mons


def _ramp(steps, width, first=0, every=1):
    return np.repeat(np.arange(first, first + steps * every, every, dtype=float)[:, None], width, 1)


@pytest.mark.parametrize("precision", ("double", "float"))
def test_population_and_view_recordings(precision):
    net, m = _network(precision)
    net.simulate(10)
    np.testing.assert_array_equal(m["m"].get(reshape=False)["r"], _ramp(10, 3))
    np.testing.assert_array_equal(m["n"].get(reshape=False)["r"], _ramp(10, 2))
    np.testing.assert_array_equal(m["q"].get(reshape=False)["r"], _ramp(10, 2))
    np.testing.assert_array_equal(m["r"].get(reshape=False)["r"], _ramp(10, 3))
    net.close()


def test_period_of_ten_steps():
    net, m = _network("double")
    net.simulate(100)
    np.testing.assert_array_equal(m["o"].get(reshape=False)["r"], _ramp(10, 3, every=10))
    net.close()


def test_monitor_started_later_and_paused():
    net, m = _network("double")
    net.simulate(10)
    m["p"].start()
    m["m"].pause()
    net.simulate(10)
    m["m"].resume()
    np.testing.assert_array_equal(m["p"].get(reshape=False)["r"], _ramp(10, 3, first=10))
    # m recorded steps 0-9, paused for 10-19
    np.testing.assert_array_equal(m["m"].get(reshape=False)["r"], _ramp(10, 3))
    net.close()


def test_pause_then_resume():
    net, m = _network("double")
    m["m"].pause()
    net.simulate(10)
    m["m"].resume()
    net.simulate(10)
    np.testing.assert_array_equal(m["m"].get()["r"], _ramp(10, 3, first=10))
    net.close()


def test_rank_and_step_access():
    net, m = _network("double")
    net.simulate(10)
    data = m["m"].get(reshape=False)["r"]
    np.testing.assert_array_equal(data[5, :], [5.0, 5.0, 5.0])
    np.testing.assert_array_equal(data[:, 1], np.arange(10.0))
    net.close()


@pytest.mark.parametrize("precision", ("double", "float"))
def test_spikes_and_refractory_recordings(precision):
    net, m = _network(precision)
    net.simulate(10)
    assert m["s"].get("spike")[0] == [4, 6, 8]
    t = m["t"].get(reshape=False)
    np.testing.assert_array_equal(t["v"][:, 0], [1, 2, 1, 1, 1, 1, 2, 1, 1, 1])
    np.testing.assert_array_equal(t["v"], np.repeat(t["v"][:, :1], 3, 1))
    assert t["spike"][1] == [2, 7]
    net.close()
