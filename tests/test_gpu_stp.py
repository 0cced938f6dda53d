"""Short-term plasticity (event-driven x and u updated at every pre-synaptic
spike, transmission w * u * x) on the 400-neuron COBA network against the
reference's own run (tests/golden/stp_small.npz, made by
tests/golden/make_golden.py): in double precision the raster is
bit-identical, and the final state, every synapse's x and u and the g_exc
recorded every 50 steps (after the transmissions, before the update, as
the reference records conductances) agree within 1e-12 (the event-driven
decays call the device's exp(), whose last bit can differ from glibc's);
in single precision the spike count is close."""
import os
import sys

import numpy as np
import pytest

from annarchy_b200 import Network, Synapse
from annarchy_b200 import workloads as wl

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from stp_model import STP_EQUATIONS, STP_PARAMETERS, STP_PRE_SPIKE  # noqa: E402

pytestmark = pytest.mark.gpu


def _run(g, precision):
    cn = wl.coba_net(seed=int(g["seed"]), n=int(g["n"]), p=float(g["p"]), steps=int(g["steps"]))
    assert wl.csr_digest(cn.w_exc) == str(g["digest_exc"])
    net = Network(dt=cn.dt, seed=0)
    net.config(precision=precision)
    P = net.create(cn.n, wl.coba_neuron(cn.params))
    Pe, Pi = P[: cn.n_exc], P[cn.n_exc:]
    stp = Synapse(parameters=STP_PARAMETERS, equations=STP_EQUATIONS, pre_spike=STP_PRE_SPIKE)
    ce = net.connect(Pe, P, "exc", synapse=stp)
    ce.from_sparse(wl.to_from_sparse(cn.w_exc))
    net.connect(Pi, P, "inh").from_sparse(wl.to_from_sparse(cn.w_inh))
    m = net.monitor(P, "spike")
    mg = net.monitor(P, ["g_exc"], period=int(g["g_every"]) * cn.dt)
    net.compile()
    P.v = cn.v0
    net.simulate(int(g["steps"]) * cn.dt)
    s, i = m.spike_arrays()
    out = dict(steps=s, idx=i, v=np.asarray(P.v).copy(), g_exc=np.asarray(P.g_exc).copy(),
               g_inh=np.asarray(P.g_inh).copy(), trace=np.asarray(mg.get("g_exc")),
               x=np.asarray(ce.get("x", flat=True)), u=np.asarray(ce.get("u", flat=True)),
               err=net._backend.native.device_error())
    net.close()
    return out


def test_stp_exact(golden):
    g = golden("stp_small")
    out = _run(g, "double")
    assert out["err"] == 0
    assert np.array_equal(out["steps"], g["spike_steps"])
    assert np.array_equal(out["idx"], g["spike_idx"])
    for k, gk in (("v", "v_final"), ("g_exc", "g_exc_final"), ("g_inh", "g_inh_final"),
                  ("trace", "g_exc_trace"), ("x", "x_final"), ("u", "u_final")):
        assert out[k].shape == g[gk].shape, k
        np.testing.assert_allclose(out[k], g[gk], rtol=1e-12, atol=1e-12, err_msg=k)


def test_stp_float_rates(golden):
    g = golden("stp_small")
    out = _run(g, "float")
    assert out["err"] == 0
    n_ref = g["spike_steps"].size
    assert abs(out["steps"].size - n_ref) <= 0.05 * n_ref, (out["steps"].size, n_ref)
