"""Recording the weighted sums of a rate-coded population (`sum(exc)`) on
the device: a constant input gives the same sum at every recorded step, and
r follows the explicit-Euler recursion driven by it."""
import numpy as np
import pytest

from annarchy_b200 import Network, Neuron

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["double", "float"])
def test_sum_monitor(precision):
    net = Network(dt=1.0)
    net.config(precision=precision)
    P = net.create((4, 5), Neuron(parameters="tau = 10.0", equations="tau * dr/dt + r = sum(exc)"))
    inp = net.create(20, Neuron(parameters="r = 1.0"))
    w = np.linspace(0.01, 0.2, 20 * 20).reshape(20, 20)      # (post, pre)
    net.connect(inp, P, "exc").from_matrix(w)
    m = net.monitor(P, ["r", "sum(exc)"], period=2.0)
    net.compile()
    net.simulate(40.0)
    d = m.get()
    s, r = d["sum(exc)"], d["r"]
    assert s.shape == (20, 4, 5) and r.shape == (20, 4, 5)
    want = np.cumsum(w, axis=1)[:, -1].reshape(4, 5)        # ascending pre rank, as summed
    tol = 0 if precision == "double" else 1e-6
    np.testing.assert_allclose(s, np.broadcast_to(want, s.shape), rtol=tol, atol=0)
    # r after step t (recorded at t = 0, 2, 4, ...): r_t = r_{t-1} + (sum - r_{t-1}) / tau
    x = np.zeros((4, 5))
    ref = []
    for t in range(40):
        x = x + (want - x) / 10.0
        if t % 2 == 0:
            ref.append(x.copy())
    np.testing.assert_allclose(r, np.asarray(ref), rtol=1e-12 if precision == "double" else 1e-5)
    assert m.times()["r"]["start"] == [0] and m.times()["r"]["stop"] == [40]
    net.close()
