"""Network constants in equations: declared in the generated module (an
attribute of the same name hides them), compiled for sm_100a, and (on the
GPU) changed at run time."""
import numpy as np
import pytest

from annarchy_b200 import Constant, Network, Neuron
from annarchy_b200.runtime import lib as L


def _net(prec="double"):
    net = Network(dt=1.0)
    net.config(precision=prec)
    kappa = net.constant("kappa", 2.0)
    inp = net.create(10, Neuron(parameters="r = 1.0"))
    out = net.create(4, Neuron(equations="r = kappa * sum(exc)"))
    hid = net.create(3, Neuron(parameters="kappa = 5.0", equations="r = kappa"))
    net.connect(inp, out, "exc").all_to_all(0.1)
    return net, kappa, out, hid


def test_constants_compile_and_shadow():
    net, kappa, out, hid = _net()
    mod = net.generate_code()
    assert "__constant__ double kappa;" in mod.source
    size, log = L.nvrtc_compile(mod.source, mod.options)
    assert size > 0 and "error" not in log.lower()
    assert net.get_constant("kappa") is kappa and kappa == 2.0 and kappa.value == 2.0


def test_global_constants_reach_new_networks():
    from annarchy_b200.core.network import GLOBAL_CONSTANTS
    g = Constant("anb_test_gain", 3.0)
    try:
        net = Network(dt=1.0)
        assert net.get_constant("anb_test_gain").value == 3.0
        g.set(4.0)
        assert net.get_constant("anb_test_gain").value == 4.0
    finally:
        GLOBAL_CONSTANTS.pop("anb_test_gain", None)


@pytest.mark.gpu
def test_constant_values_on_device():
    net, kappa, out, hid = _net()
    net.compile()
    net.simulate(2.0)
    np.testing.assert_allclose(out.r, 2.0 * 1.0)      # 10 inputs x 0.1 x kappa
    np.testing.assert_allclose(hid.r, 5.0)           # the parameter hides the constant
    kappa.set(3.0)
    net.simulate(2.0)
    np.testing.assert_allclose(out.r, 3.0)
    net.close()
