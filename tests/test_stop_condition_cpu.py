"""Stop conditions (simulate_until) on the CPU: the generated stop kernels
compile for sm_100a and the networks that have them use the grid engine."""
import pytest

from annarchy_b200 import Network, Neuron
from annarchy_b200.core.backend import CompiledNetwork
from annarchy_b200.runtime import lib as L


def _net(cond_rate, cond_spike):
    net = Network(dt=0.1)
    net.config(precision="float")
    a = net.create(50, Neuron(parameters="tau = 10.0", equations="tau * dr/dt + r = 1.5"),
                   stop_condition=cond_rate)
    b = net.create(40, Neuron(parameters="I = 2.0", equations="dv/dt = -v + I", spike="v > 1.0",
                              reset="v = 0.0"), stop_condition=cond_spike)
    return net, a, b


@pytest.mark.parametrize("cr,cs", [("r > 1.0", "spiked : any"), ("r > 1.0 : all", "v > 0.5 : any"),
                                   ("r < 0.2 : any", "spiked: all")])
def test_stop_kernels_compile(cr, cs):
    net, a, b = _net(cr, cs)
    mod = net.generate_code()
    assert "pop0_stop" in mod.source and "pop1_stop" in mod.source
    size, log = L.nvrtc_compile(mod.source, mod.options)
    assert size > 0 and "error" not in log.lower()
    assert [s[0] for s in mod.stops] == [0, 1]
    assert [s[4] for s in mod.stops] == ["all" in cr, "all" in cs]


def test_stop_conditions_use_the_grid_engine():
    net, a, b = _net("r > 1.0", "spiked : any")
    be = CompiledNetwork(net, dry=True)
    be.build()
    assert be.engine == "grid"
    assert "stop_flags" in be.native.arrays
