"""Device-generated fixed in-degree connectivity and the warp-per-row
kernels of the large plastic network, at reduced size: the double-precision
grid engine matches the CPU oracle run on the same (read-back) connectivity."""
import numpy as np
import pytest
import scipy.sparse as sp

from annarchy_b200 import workloads as wl
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def small_large_net():
    return wl.LargeNet(n=20000, fan_e=80, fan_i=20, w_exc=0.48, w_inh=5.36, steps=400)


def readback(net, proj):
    nat = net._backend.native
    k = proj.id
    rp = nat.read(f"proj{k}__row_ptr").astype(np.int64)
    col = nat.read(f"proj{k}__col")
    w = net._backend.read_projection_attribute(proj, "w")
    pre_lo = int(proj.pre_ranks[0])
    m = sp.csr_matrix((w, col - pre_lo, rp), shape=(len(proj.post_ranks_view), len(proj.pre_ranks)))
    return m


@pytest.mark.parametrize("stdp", [False, True])
def test_device_connectivity_exact_vs_oracle(stdp):
    ln = small_large_net()
    net, P, mon, (ee, ei, ie) = wl.build_large_network(ln, "double", stdp=stdp)
    net.compile()
    mats = [readback(net, p) for p in (ee, ei, ie)]
    # structure: exact in-degree, distinct ascending pre ranks, no self-connection on E->E
    for m, p in zip(mats, (ee, ei, ie)):
        deg = np.diff(m.indptr)
        assert np.all(deg == (ln.fan_e if p is not ie else ln.fan_i))
        assert np.all(np.diff(m.indices)[np.diff(np.repeat(np.arange(m.shape[0]), deg)) == 0] > 0)
    rows = np.repeat(np.arange(mats[0].shape[0]), np.diff(mats[0].indptr))
    assert not np.any(mats[0].indices == rows)
    net.simulate_steps(ln.steps)
    s, i = mon.spike_arrays()
    n, ne = ln.n, ln.n_exc
    cn = wl.CobaNet(n, ne, None, None, np.random.default_rng(ln.seed).uniform(-60.0, -50.0, n),
                    params=dict(wl.COBA_PARAMS), steps=ln.steps)
    projs = [O.SpikeProjection(n, mats[0], np.arange(ne), np.arange(ne), 0,
                               stdp=wl.STDP_PARAMS if stdp else None),
             O.SpikeProjection(n, mats[1], np.arange(ne, n), np.arange(ne), 0),
             O.SpikeProjection(n, mats[2], np.arange(n), np.arange(ne, n), 1)]
    ref = O.coba_run(cn, projs)
    assert ref["n_spikes"] > 1000
    assert np.array_equal(s, ref["spike_steps"]) and np.array_equal(i, ref["spike_idx"])
    if not stdp:
        assert np.array_equal(P.v, ref["v"])
        assert np.array_equal(P.g_exc, ref["g_exc"])
    else:
        w = net._backend.read_projection_attribute(ee, "w")
        np.testing.assert_allclose(w, projs[0].w, rtol=0, atol=1e-12)
        np.testing.assert_allclose(P.v, ref["v"], rtol=0, atol=1e-9)
    net.close()


@pytest.mark.parametrize("static_w,tol", [("float32", 0.03), ("bfloat16", 0.10)])
def test_device_connectivity_fast_rates(static_w, tol):
    """Single precision (float plastic weights, float or bfloat16 static
    weights) over the first 40 ms: firing rate within `tol` of the double run
    (bfloat16 rounds the static weights by up to 0.4 %, which the initial
    transient amplifies), E->E weight histograms close."""
    ln = small_large_net()
    out = {}
    for prec, kw in (("double", {}), ("float", {"weight_dtype": static_w})):
        net, P, mon, (ee, ei, ie) = wl.build_large_network(ln, prec, **kw)
        net.compile()
        net.simulate_steps(ln.steps)
        out[prec] = (mon.spike_arrays()[1].size,
                     np.histogram(net._backend.read_projection_attribute(ee, "w"),
                                  bins=20, range=(0, 1))[0])
        net.close()
    n64, h64 = out["double"]
    n32, h32 = out["float"]
    assert abs(n32 - n64) / n64 < tol, (n32, n64)
    assert np.abs(h32 - h64).sum() / h64.sum() < 2 * tol
