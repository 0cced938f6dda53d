"""simulate_until on the device: the run ends after the first step at which
the populations' stop conditions hold (all of them with "and", any with
"or"), or after max_duration; the step is the one a host restatement of the
same Euler recursion finds, and monitors hold exactly the steps run."""
import numpy as np
import pytest

from annarchy_b200 import Network, Neuron

pytestmark = pytest.mark.gpu

DT = 0.1


def _first_rate_step(thr):
    r, k = 0.0, 0
    while True:
        k += 1
        r = r + DT * ((1.5 - r) / 10.0)
        if r > thr:
            return k


def _first_spike_step(I):
    v, k = 0.0, 0
    while True:
        k += 1
        v = v + DT * (-v + I)
        if v > 1.0:
            return k


def _net(cond_rate, cond_spike, I=2.0):
    net = Network(dt=DT)
    net.config(precision="double")
    a = net.create(50, Neuron(parameters="tau = 10.0", equations="tau * dr/dt + r = 1.5"),
                   stop_condition=cond_rate)
    b = net.create(40, Neuron(parameters=f"I = {I}", equations="dv/dt = -v + I", spike="v > 1.0",
                              reset="v = 0.0"), stop_condition=cond_spike)
    m = net.monitor(a, "r")
    net.compile()
    return net, a, b, m


@pytest.mark.parametrize("cond", ["r > 1.0", "r > 1.0 : all"])
def test_rate_condition(cond):
    net, a, b, m = _net(cond, None)
    k = _first_rate_step(1.0)
    dur = net.simulate_until(1000.0, a)
    assert net.current_step == k and dur == pytest.approx(k * DT)
    assert m.get("r").shape[0] == k
    assert np.all(a.r > 1.0)
    net.close()


def test_spiked_and_operators():
    net, a, b, m = _net("r > 1.0", "spiked : any")
    ks = _first_spike_step(2.0)
    kr = _first_rate_step(1.0)
    assert ks < kr
    dur = net.simulate_until(1000.0, [a, b], operator="or")
    assert net.current_step == ks
    net.close()
    # "and": both at the same step; b spikes every ks steps (reset to 0), a
    # holds from kr on
    net, a, b, m = _net("r > 1.0", "spiked : any")
    want = next(k for k in range(kr, 10 * kr) if k % ks == 0)
    net.simulate_until(1000.0, [a, b], operator="and")
    assert net.current_step == want
    net.close()


def test_max_duration_and_no_condition():
    net, a, b, m = _net("r > 5.0", None)
    dur = net.simulate_until(20.0, a)
    assert net.current_step == 200 and dur == pytest.approx(20.0)
    # a population without a condition in an "and" list ends the run after one step
    net.simulate_until(20.0, b)
    assert net.current_step == 201
    net.close()
