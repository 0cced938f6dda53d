"""Saving and loading network state in the reference's file layout
(ANNarchy/core/IO.py:340-617): round trips through every format, before and
after compile(), and a state file written by the reference itself
(tests/golden/io_ref_state.npz, made by tests/golden/make_golden.py, which
also checks that the reference loads a file written here)."""
import os

import numpy as np
import pytest
import scipy.sparse as sp

import annarchy_b200 as ann
from annarchy_b200 import workloads as wl

HERE = os.path.dirname(os.path.abspath(__file__))


def _net(cn, w_scale=1.0, delays=True):
    net = ann.Network(dt=cn.dt, seed=1)
    P = net.create(cn.n, wl.coba_neuron(cn.params))
    Pe, Pi = P[: cn.n_exc], P[cn.n_exc:]
    ee = net.connect(Pe, Pe, "exc", synapse=ann.STDP(**wl.STDP_PARAMS))
    ci = net.connect(Pi, P, "inh")
    return net, P, ee, ci


def _fill(cn, ee, ci, scale=1.0):
    w_ee = wl.stdp_matrix(cn, 3, 0.1)
    ee.from_sparse(wl.to_from_sparse(w_ee * scale))
    ci.from_sparse(wl.to_from_sparse(cn.w_inh * scale), delays=0.5)


@pytest.mark.parametrize("ext", [".npz", ".data", ".txt.gz"])
def test_roundtrip_before_compile(tmp_path, ext):
    cn = wl.coba_net(seed=3, n=200, p=0.1)
    net, P, ee, ci = _net(cn)
    _fill(cn, ee, ci)
    P.v = np.linspace(-60, -50, cn.n)
    ee.set({"tau_plus": 20.0})
    f = str(tmp_path / ("state" + ext))
    net.save(f)
    net2, P2, ee2, ci2 = _net(cn)
    net2.load(f)
    assert np.array_equal(P2.v, P.v)
    for a, b in ((ee, ee2), (ci, ci2)):
        assert (a._csr != b._csr).nnz == 0 and np.array_equal(a._csr.data, b._csr.data)
        assert a.post_ranks == b.post_ranks
    assert ci2.delay == pytest.approx(0.5) and ee2.get("tau_plus") == 20.0


def test_saved_layout_matches_reference_keys(tmp_path):
    cn = wl.coba_net(seed=3, n=200, p=0.1)
    net, P, ee, ci = _net(cn)
    _fill(cn, ee, ci)
    f = str(tmp_path / "s.npz")
    net.save(f)
    from annarchy_b200.core.io import load_data
    d = load_data(f)
    assert {"time_step", "net_id", "obj_names", P.name, ee.name, ci.name} <= set(d)
    assert {"name", "geometry", "size", "attributes", "parameters", "variables", "v"} <= set(d[P.name])
    assert {"name", "pre", "post", "target", "post_ranks", "pre_ranks", "delays", "w", "attributes",
            "x", "y", "tau_plus"} <= set(d[ee.name])


def test_load_reference_state_file():
    """A state file written by the reference's Network.save() (an STDP
    network after 50 steps): connectivity, delays, weights, traces and
    neural variables load into the same network built here."""
    ref = os.path.join(HERE, "golden", "io_ref_state.npz")
    meta = np.load(os.path.join(HERE, "golden", "io_ref_meta.npz"))
    cn = wl.coba_net(seed=3, n=200, p=0.1)
    net, P, ee, ci = _net(cn)
    net.load(ref)
    np.testing.assert_array_equal(P.v, meta["v"])
    w = np.concatenate([np.asarray(x) for x in ee.get("w")])
    np.testing.assert_array_equal(w, meta["w_ee"])
    np.testing.assert_array_equal(np.concatenate([np.asarray(x) for x in ee.get("x")]), meta["x_ee"])
    assert ci.delay == pytest.approx(0.5)
    assert ee.nb_synapses == meta["w_ee"].size
    # and the reference loaded a file written by this backend's save()
    assert bool(meta["reference_loaded_ours"])


@pytest.mark.gpu
def test_roundtrip_after_compile(tmp_path):
    cn = wl.coba_net(seed=3, n=200, p=0.1)
    net, P, ee, ci = _net(cn)
    _fill(cn, ee, ci)
    mon = net.monitor(P, "spike")
    net.compile()
    P.v = cn.v0
    net.simulate_steps(300)
    f = str(tmp_path / "after.npz")
    net.save(f)
    w_before = np.concatenate([np.asarray(x) for x in ee.get("w")])
    v_before = P.v.copy()
    net.simulate_steps(100)
    net.load(f)
    assert net.current_step == 300
    np.testing.assert_array_equal(P.v, v_before)
    np.testing.assert_array_equal(np.concatenate([np.asarray(x) for x in ee.get("w")]), w_before)
    net.close()
