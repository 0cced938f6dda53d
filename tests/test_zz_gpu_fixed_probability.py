"""Device-generated fixed-probability connectivity: rows, pre ranks and
weights equal the host restatement of the device's draws synapse by synapse,
and the reduced large network built with it matches the CPU oracle run on
the read-back connectivity."""
import numpy as np
import pytest

import connect_emulation as CE
from annarchy_b200 import workloads as wl
from oracle import oracle as O
from test_gpu_device_connect import readback, small_large_net

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("wdt", ["float64", "float32", "bfloat16"])
def test_device_fixed_probability_equals_host_restatement(wdt):
    """Rows, pre ranks and weights of device-built fixed-probability
    projections equal the host restatement of the same draws (self
    connections excluded on E->E, Normal and Uniform weights)."""
    from annarchy_b200 import Network, Normal, Uniform
    from annarchy_b200.core.backend import from_bf16, to_bf16
    net = Network(dt=0.1, seed=11)
    prec = "double" if wdt == "float64" else "float"
    net.config(precision=prec, engine="grid", device_connectors=True,
               **({} if prec == "double" else {"weight_dtype": wdt}))
    P = net.create(3000, wl.coba_neuron(dict(wl.COBA_PARAMS)))
    Pe, Pi = P[:2400], P[2400:]
    ee = net.connect(Pe, Pe, "exc").fixed_probability(0.03, Normal(0.5, 0.05))
    ie = net.connect(Pi, P, "inh").fixed_probability(0.2, Uniform(1.0, 2.0))
    net.compile()
    nat = net._backend.native
    for proj, n_post, post0, lo, hi, p, wk, a, b, excl in (
            (ee, 2400, 0, 0, 2400, 0.03, 2, 0.5, 0.05, True),
            (ie, 3000, 0, 2400, 3000, 0.2, 1, 1.0, 2.0, False)):
        seed = proj._device_conn["seed"]
        rp, col, w = CE.fixed_probability(n_post, post0, 0, lo, hi, p, seed, excl, wk, a, b)
        k = proj.id
        assert np.array_equal(nat.read(f"proj{k}__row_ptr").astype(np.int64), rp)
        assert np.array_equal(nat.read(f"proj{k}__col").astype(np.int64), col)
        assert proj.nb_synapses == col.size
        got = net._backend.read_projection_attribute(proj, "w")
        if wdt == "float64":
            np.testing.assert_allclose(got, w, rtol=1e-13, atol=0)
        elif wdt == "float32":
            np.testing.assert_allclose(got, w.astype(np.float32), rtol=1e-6, atol=0)
        else:
            np.testing.assert_allclose(got, from_bf16(to_bf16(w)), rtol=1e-2, atol=0)
        assert [len(x) for x in proj.get("w")] == list(np.diff(rp))
    net.close()


def test_device_fixed_probability_exact_vs_oracle():
    """The reduced large network with fixed-probability device connectivity
    (same mean in-degrees, STDP on E->E): the double-precision run equals the
    oracle run on the read-back connectivity."""
    ln = small_large_net()
    net, P, mon, (ee, ei, ie) = wl.build_large_network(ln, "double", stdp=True,
                                                       connector="fixed_probability")
    net.compile()
    mats = [readback(net, p) for p in (ee, ei, ie)]
    deg = np.diff(mats[0].indptr)
    assert deg.min() < deg.max() and abs(deg.mean() - ln.fan_e) < 2.0
    net.simulate_steps(ln.steps)
    s, i = mon.spike_arrays()
    n, ne = ln.n, ln.n_exc
    cn = wl.CobaNet(n, ne, None, None, np.random.default_rng(ln.seed).uniform(-60.0, -50.0, n),
                    params=dict(wl.COBA_PARAMS), steps=ln.steps)
    projs = [O.SpikeProjection(n, mats[0], np.arange(ne), np.arange(ne), 0, stdp=wl.STDP_PARAMS),
             O.SpikeProjection(n, mats[1], np.arange(ne, n), np.arange(ne), 0),
             O.SpikeProjection(n, mats[2], np.arange(n), np.arange(ne, n), 1)]
    ref = O.coba_run(cn, projs)
    assert ref["n_spikes"] > 1000
    assert np.array_equal(s, ref["spike_steps"]) and np.array_equal(i, ref["spike_idx"])
    w = net._backend.read_projection_attribute(ee, "w")
    np.testing.assert_allclose(w, projs[0].w, rtol=0, atol=1e-12)
    np.testing.assert_allclose(P.v, ref["v"], rtol=0, atol=1e-9)
    net.close()
