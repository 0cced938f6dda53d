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


def _self_stdp(persistent: bool, steps: int):
    """2000 neurons, each with one plastic synapse onto itself (one-to-one
    STDP): every spike is a pre and a post event of the same synapse in the
    same step, and every conductance receives at most one increment per
    step, so the engines must agree bit for bit."""
    from annarchy_b200 import Network, STDP
    net = Network(dt=0.1, seed=3)
    net.config(precision="float", engine="grid", persistent=persistent)
    params = dict(wl.COBA_PARAMS)
    params["I"] = 20.0
    P = net.create(2000, wl.coba_neuron(params))
    proj = net.connect(P, P, "exc", synapse=STDP(**wl.STDP_PARAMS)).one_to_one(weights=0.5)
    mon = net.monitor(P, "spike")
    P.v = np.random.default_rng(3).uniform(-60.0, -50.0, 2000)
    net.compile()
    assert (net._backend.module.local is not None) == persistent
    net.simulate_steps(steps // 2)
    w_mid = proj.get("w", flat=True)          # the post events of a run's last step are in
    net.simulate_steps(steps - steps // 2)
    s, i = mon.spike_arrays()
    out = (s, i, np.asarray(P.v), w_mid, proj.get("w", flat=True))
    net.close()
    return out


def test_persistent_fused_stdp_equals_graph_step_bit_for_bit():
    """The persistent engine runs the post events of step t - 1 with the
    transmissions of step t (a synapse whose pre and post neurons both
    spiked gets its post event first, in the same thread): rasters,
    potentials and weights equal the graph of separate kernels, also across
    two runs (the post events of a run's last step complete before it
    returns)."""
    a = _self_stdp(True, 3000)
    b = _self_stdp(False, 3000)
    assert a[1].size > 500
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    assert not np.array_equal(a[3], a[4])     # the weights moved
