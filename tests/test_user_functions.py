"""User functions (ANNarchy tests_python/Common/test_CustomFunc.py:15-95):
a global one from add_function, one in a neuron (nested if/else branches)
and one in a synapse; their host callables return the reference's known
answers, and the network's module carries them as device functions."""
import numpy as np

from annarchy_b200 import Network, Neuron, Synapse, add_function, functions
from annarchy_b200.runtime import lib as L

add_function("glob_pos(x) = pos(x)")
NEURON = Neuron(equations="r = transfer_function(sum(exc), 0.0)",
                functions="transfer_function(x, t) = if x > t: if x > 2*t : (x - 2*t)^2 "
                          "else: x - t else: 0.")
NEURON2 = Neuron(equations="r = glob_pos(sum(exc))")
SYNAPSE = Synapse(equations="w += hebb(pre.r, post.r)", functions="hebb(x, y) = x * y")


def _net(precision="double"):
    net = Network(dt=1.0)
    net.config(dry=True, precision=precision)
    p1 = net.create(10, NEURON)
    p2 = net.create(10, NEURON2)
    proj = net.connect(p1, p1, "exc", SYNAPSE)
    proj.all_to_all(1.0)
    return net, p1, p2, proj


def test_host_callables_give_the_known_answers():
    _, p1, _, proj = _net()
    np.testing.assert_array_equal(
        p1.transfer_function(np.array([0.0, 1.0, 2.0, 3.0]), np.array([2.0, 2.0, 2.0, 2.0])),
        [0, 0, 0, 1])
    np.testing.assert_array_equal(p1.transfer_function([0.0, 1.0, 2.0, 3.0], [2.0] * 4),
                                  [0, 0, 0, 1])
    np.testing.assert_array_equal(proj.hebb(np.arange(4.0), np.arange(4.0)), [0, 1, 4, 9])
    np.testing.assert_array_equal(proj.hebb([0.0, 1.0, 2.0, 3.0], [0.0, 1.0, 2.0, 3.0]),
                                  [0, 1, 4, 9])
    np.testing.assert_array_equal(functions("glob_pos")([-1.0, 2.0]), [0.0, 2.0])


def test_device_functions_in_the_module():
    for precision in ("double", "float"):
        net, p1, _, _ = _net(precision)
        mod = net.generate_code()
        assert "transfer_function(" in mod.source and "hebb(" in mod.source
        assert "glob_pos(" in mod.source
        size, log = L.nvrtc_compile(mod.source, mod.options)
        assert size > 0, log
    r = next(v for v in p1.desc["variables"] if v["name"] == "r")
    assert r["cpp"] == "r%(local_index)s = transfer_function(_sum_exc%(local_index)s, 0.0);"
