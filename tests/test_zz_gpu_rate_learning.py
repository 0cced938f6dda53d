"""Rate-coded synaptic learning on the device against the reference's own
run of the same network (tests/golden/rate_learning.npz): semiglobal,
global and local equations, the min bound of w, and enable_learning with a
period and an offset — bit for bit in double precision, within float32
accuracy in single precision."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from make_golden import LEARN_SYNAPSE, learning_inputs  # noqa: E402

from annarchy_b200 import Network, Neuron, Synapse  # noqa: E402
from annarchy_b200 import workloads as wl  # noqa: E402

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "rate_learning.npz"))


def build(precision):
    r_in, w = learning_inputs()
    net = Network(dt=1.0, seed=1)
    net.config(precision=precision)
    inp = net.create(r_in.size, Neuron(parameters="r = 0.0"))
    out = net.create(w.shape[0], Neuron(parameters="tau = 10.0",
                                        equations="tau * dr/dt + r = sum(exc) + sum(mod)"))
    syn = Synapse(**LEARN_SYNAPSE)
    p1 = net.connect(inp, out, "exc", synapse=syn).from_sparse(wl.to_from_sparse(w))
    p2 = net.connect(inp, out, "mod", synapse=syn).from_sparse(wl.to_from_sparse(w * 0.5))
    m = net.monitor(out, "r")
    return net, inp, out, p1, p2, m, r_in


def test_generated_update_compiles():
    from annarchy_b200.runtime import lib as L
    for prec in ("double", "float"):
        net = build(prec)[0]
        mod = net.generate_code()
        assert "proj0_update_global" in mod.source and "proj1_update()" in mod.source
        size, log = L.nvrtc_compile(mod.source, mod.options)
        assert size > 0 and "error" not in log.lower()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["double", "float"])
def test_rate_learning_equals_reference(precision):
    net, inp, out, p1, p2, m, r_in = build(precision)
    net.compile()
    inp.r = r_in
    net.simulate(7.0)
    p2.enable_learning(period=3.0, offset=1.0)
    net.simulate(int(GOLD["steps"]) - 7.0)
    got = dict(r=m.get("r"), w1=p1.get("w", flat=True), w2=p2.get("w", flat=True),
               alpha1=p1.alpha, alpha2=p2.alpha, beta1=p1.beta, beta2=p2.beta)
    for k, v in got.items():
        if precision == "double":
            np.testing.assert_array_equal(np.asarray(v), GOLD[k], err_msg=k)
        else:
            np.testing.assert_allclose(np.asarray(v), GOLD[k], rtol=2e-4, atol=2e-6, err_msg=k)
    # learning off: weights stay, the other variables still update (rate-coded: all stop)
    p1.disable_learning()
    w_before, a_before = p1.get("w", flat=True), p1.alpha.copy()
    net.simulate(10.0)
    np.testing.assert_array_equal(p1.get("w", flat=True), w_before)
    np.testing.assert_array_equal(p1.alpha, a_before)
    p1.update = True
    p1.plasticity = False
    net.simulate(10.0)
    np.testing.assert_array_equal(p1.get("w", flat=True), w_before)
    assert not np.array_equal(p1.alpha, a_before)
    net.close()
