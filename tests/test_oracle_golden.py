"""The CPU oracle against the golden fixtures produced by the reference
simulator itself (tests/golden/make_golden.py): bit-exact in double."""
import numpy as np
import pytest

from annarchy_b200 import workloads as wl
from oracle import oracle as O


def test_rate_small_trace_exact(golden):
    g = golden("rate_small")
    rn = wl.rate_net(seed=7, n_in=100, n_out=200, p_in=0.1, p_rec=0.05, steps=100)
    assert wl.csr_digest(rn.w_in) == str(g["digest_in"])
    assert wl.csr_digest(rn.w_rec) == str(g["digest_rec"])
    _, tr = O.rate_run(rn, trace=True)
    assert np.array_equal(tr, g["r_at"])


@pytest.mark.parametrize("threads", [1, 4])
def test_rate_c1_exact(golden, threads):
    g = golden("rate_c1")
    rn = wl.rate_net(seed=42)
    assert wl.csr_digest(rn.w_in) == str(g["digest_in"])
    _, tr = O.rate_run(rn, trace=True, threads=threads)
    assert np.array_equal(tr[g["record_steps"]], g["r_at"])
    assert np.array_equal(tr.sum(axis=1), g["r_sum"])


@pytest.mark.parametrize("name,kw", [
    ("coba_small", dict(seed=7, n=400, p=0.05, steps=2000)),
    ("coba_c2", dict(seed=42, n=4000, p=0.02, steps=10000)),
])
def test_coba_raster_exact(golden, name, kw):
    g = golden(name)
    cn = wl.coba_net(**kw)
    assert wl.csr_digest(cn.w_exc) == str(g["digest_exc"])
    assert wl.csr_digest(cn.w_inh) == str(g["digest_inh"])
    res = O.coba_run(cn)
    assert np.array_equal(res["spike_steps"], g["spike_steps"])
    assert np.array_equal(res["spike_idx"], g["spike_idx"])
    for k in ("v", "g_exc", "g_inh"):
        assert np.array_equal(res[k], g[k + "_final"]), k


def test_coba_threads_identical():
    cn = wl.coba_net(seed=7, n=400, p=0.05, steps=500)
    a = O.coba_run(cn, threads=1)
    b = O.coba_run(cn, threads=4)
    assert np.array_equal(a["spike_idx"], b["spike_idx"]) and np.array_equal(a["v"], b["v"])


def test_stdp_weights_exact(golden):
    g = golden("stdp_small")
    cn = wl.coba_net(seed=11, n=400, p=0.05, steps=2000)
    w_ee = wl.stdp_matrix(cn, 11, 0.05)
    assert wl.csr_digest(w_ee) == str(g["digest_ee"])
    projs = O.coba_projections(cn, w_ee, wl.STDP_PARAMS)
    res = O.coba_run(cn, projs)
    assert np.array_equal(res["spike_steps"], g["spike_steps"])
    assert np.array_equal(res["spike_idx"], g["spike_idx"])
    assert np.array_equal(projs[0].w, g["w_ee_final"])


def test_silent_without_drive():
    """The spiking net as specified (no drive) never fires: the reason the
    benchmark adds I = 20."""
    cn = wl.coba_net(seed=42, n=4000, p=0.02, drive=0.0, steps=2000)
    assert O.coba_run(cn)["n_spikes"] == 0
