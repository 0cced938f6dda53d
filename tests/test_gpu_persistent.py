"""The grid engine's step as one cooperative persistent kernel (grid-wide
barriers between its phases) against the same step launched as a CUDA graph
of separate kernels.

With one constant weight per projection, every conductance receives the same
increment from each of its spiking inputs, so the order of the atomic
additions does not change the result: the two engines must then agree bit
for bit in single precision. With STDP the weights differ per synapse and the
additions' order changes the rounding; the firing rates must still agree."""
import numpy as np
import pytest

from annarchy_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _run(persistent: bool, stdp: bool, steps: int):
    ln = wl.LargeNet(n=40_000, fan_e=80, fan_i=20, w_exc=0.48, w_inh=5.36, steps=steps)
    net, P, mon, _ = wl.build_large_network(ln, "float", stdp=stdp, weight_dtype="float32",
                                            persistent=persistent)
    net.compile()
    assert (net._backend.module.local is not None) == persistent
    net.simulate_steps(steps)
    s, i = mon.spike_arrays()
    out = (s, i, np.asarray(P.v), net.current_step, net._backend.native.device_error())
    net.close()
    return out


def test_persistent_step_equals_graph_step_bit_for_bit():
    a = _run(True, False, 400)
    b = _run(False, False, 400)
    assert a[1].size > 1000                                  # the network is active
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert np.array_equal(a[2], b[2])
    assert a[3] == b[3] == 400 and a[4] == 0


def test_persistent_step_with_stdp_keeps_the_rates():
    a = _run(True, True, 400)
    b = _run(False, True, 400)
    assert a[4] == 0 and a[3] == 400
    ra, rb = a[1].size, b[1].size
    assert rb > 1000 and abs(ra - rb) / rb < 0.05, (ra, rb)
