"""CUDA backend vs the reference: bit-exact in double precision (against the
golden fixtures produced by the reference itself and against the oracle),
within stated tolerances in single precision."""
import numpy as np
import pytest

from annarchy_b200 import workloads as wl
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def run_rate(rn, steps, **kw):
    net, pop, mon = wl.build_rate_network(rn, **kw)
    net.compile()
    net.simulate_steps(steps)
    r = mon.get("r")
    net.close()
    return r


def run_coba(cn, steps, **kw):
    net, P, mon = wl.build_coba_network(cn, **kw)
    net.compile()
    net.simulate_steps(steps)
    s, i = mon.spike_arrays()
    out = dict(steps=s, idx=i, v=P.v.copy(), g_exc=P.g_exc.copy(), g_inh=P.g_inh.copy(),
               engine=net.engine)
    out["net"] = net
    return out


def test_rate_small_exact(golden):
    g = golden("rate_small")
    rn = wl.rate_net(seed=7, n_in=100, n_out=200, p_in=0.1, p_rec=0.05, steps=100)
    r = run_rate(rn, 100)
    assert np.array_equal(r, g["r_at"])


def test_rate_c1_exact(golden):
    g = golden("rate_c1")
    rn = wl.rate_net(seed=42)
    r = run_rate(rn, 1000)
    assert np.array_equal(r[g["record_steps"]], g["r_at"])
    assert np.array_equal(r.sum(axis=1), g["r_sum"])


@pytest.mark.parametrize("fmt", ["ell", "ellr", "sell", "bsr", "pcsr"])
def test_rate_formats_exact(golden, fmt):
    """ELL, ELL-R, SELL and BSR sum every row in ascending pre rank:
    bit-identical to CSR."""
    g = golden("rate_small")
    rn = wl.rate_net(seed=7, n_in=100, n_out=200, p_in=0.1, p_rec=0.05, steps=100)
    r = run_rate(rn, 100, storage_format=fmt)
    assert np.array_equal(r, g["r_at"])


def test_rate_hyb_close(golden):
    """HYB adds the ELL part and the COO tail of a row separately (as the
    reference's HYB does): equal to CSR up to rounding."""
    g = golden("rate_small")
    rn = wl.rate_net(seed=7, n_in=100, n_out=200, p_in=0.1, p_rec=0.05, steps=100)
    r = run_rate(rn, 100, storage_format="hyb")
    np.testing.assert_allclose(r, g["r_at"], rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("wdt", ["float32", "bfloat16"])
def test_rate_float(wdt):
    """Single-precision state and accumulation: norm-wise relative error of r
    per step <= 1e-5 against the double oracle fed the same (rounded) weights."""
    rn = wl.rate_net(seed=42, steps=200)
    if wdt == "bfloat16":
        from annarchy_b200.core.backend import from_bf16, to_bf16
        rn.w_in.data = from_bf16(to_bf16(rn.w_in.data))
        rn.w_rec.data = from_bf16(to_bf16(rn.w_rec.data))
    _, ref = O.rate_run(rn, trace=True)
    r = run_rate(rn, 200, precision="float", weight_dtype=wdt)
    err = np.linalg.norm(r - ref, axis=1) / np.linalg.norm(ref, axis=1)
    assert err.max() <= 1e-5, err.max()


@pytest.mark.parametrize("engine", ["grid", "local"])
def test_coba_small_exact(golden, engine):
    g = golden("coba_small")
    cn = wl.coba_net(seed=7, n=400, p=0.05, steps=2000)
    out = run_coba(cn, 2000, engine=engine)
    assert out["engine"] == {"grid": "grid", "local": "cluster"}[engine]
    assert np.array_equal(out["steps"], g["spike_steps"])
    assert np.array_equal(out["idx"], g["spike_idx"])
    for k in ("v", "g_exc", "g_inh"):
        assert np.array_equal(out[k], g[k + "_final"]), k
    out["net"].close()


@pytest.mark.parametrize("graph_steps", [32, 0])
@pytest.mark.parametrize("pdl", [True, False])
def test_coba_small_exact_launch_modes(golden, graph_steps, pdl):
    """The grid engine's plan replayed as CUDA graphs or launched step by
    step, with and without programmatic dependent launch: the reference's
    raster and final state bit for bit in every mode."""
    g = golden("coba_small")
    cn = wl.coba_net(seed=7, n=400, p=0.05, steps=2000)
    out = run_coba(cn, 2000, engine="grid", graph_steps=graph_steps, pdl=pdl)
    assert np.array_equal(out["steps"], g["spike_steps"])
    assert np.array_equal(out["idx"], g["spike_idx"])
    for k in ("v", "g_exc", "g_inh"):
        assert np.array_equal(out[k], g[k + "_final"]), k
    out["net"].close()


def test_rate_c1_float_launch_modes():
    """The float rate net with and without programmatic dependent launch,
    CUDA graphs and step-by-step launches: the same final rates (the float
    sums here add in a fixed order)."""
    rn = wl.rate_net(seed=7, n_in=100, n_out=200, p_in=0.1, p_rec=0.05, steps=100)
    outs = []
    for graph_steps, pdl in ((32, True), (32, False), (0, True)):
        net, pop, _ = wl.build_rate_network(rn, "float", record=False, graph_steps=graph_steps, pdl=pdl)
        net.compile()
        net.simulate_steps(100)
        outs.append(np.asarray(pop.r).copy())
        net.close()
    for r in outs[1:]:
        assert np.array_equal(r, outs[0])


def test_coba_c2_exact(golden):
    g = golden("coba_c2")
    cn = wl.coba_net(seed=42)
    out = run_coba(cn, 10000)
    assert np.array_equal(out["steps"], g["spike_steps"])
    assert np.array_equal(out["idx"], g["spike_idx"])
    for k in ("v", "g_exc", "g_inh"):
        assert np.array_equal(out[k], g[k + "_final"]), k
    out["net"].close()


def test_coba_oracle_other_seed_grid_vs_local():
    cn = wl.coba_net(seed=3, n=1000, p=0.03, steps=1500)
    ref = O.coba_run(cn)
    for engine in ("grid", "local"):
        out = run_coba(cn, 1500, engine=engine)
        assert np.array_equal(out["idx"], ref["spike_idx"]), engine
        assert np.array_equal(out["v"], ref["v"]), engine
        out["net"].close()


def test_stdp_small(golden):
    """Plastic E->E: spikes bit-exact; weights equal up to the last-ulp
    differences of the device exp() against glibc's."""
    g = golden("stdp_small")
    cn = wl.coba_net(seed=11, n=400, p=0.05, steps=2000)
    w_ee = wl.stdp_matrix(cn, 11, 0.05)
    out = run_coba(cn, 2000, stdp_w_ee=w_ee)
    assert np.array_equal(out["steps"], g["spike_steps"])
    assert np.array_equal(out["idx"], g["spike_idx"])
    w = out["net"].projections[0].get("w", flat=True)
    np.testing.assert_allclose(w, g["w_ee_final"], rtol=0, atol=1e-12)
    out["net"].close()


@pytest.mark.parametrize("engine", ["grid", "local"])
def test_coba_float_rates(engine):
    """Single precision: identical rasters over the first steps, firing
    rate within 2 % of the double oracle over 2000 steps."""
    cn = wl.coba_net(seed=42, n=4000, p=0.02, steps=2000)
    ref = O.coba_run(cn)
    out = run_coba(cn, 2000, precision="float", engine=engine)
    n_ref, n = ref["n_spikes"], out["idx"].size
    assert abs(n - n_ref) / n_ref < 0.02, (n, n_ref)
    early = ref["spike_steps"] < 300
    e2 = out["steps"] < 300
    assert np.array_equal(out["idx"][e2], ref["spike_idx"][early])
    out["net"].close()


@pytest.mark.parametrize("fmt", ["csr", "ell", "ellr", "sell", "hyb", "bsr", "pcsr"])
@pytest.mark.parametrize("wdt", ["float32", "bfloat16"])
def test_rate_formats_float(fmt, wdt):
    """Every storage format in single precision: norm-wise relative error of
    r per step <= 1e-5 against the double oracle fed the same weights."""
    rn = wl.rate_net(seed=5, n_in=300, n_out=700, p_in=0.1, p_rec=0.05, steps=50)
    if wdt == "bfloat16":
        from annarchy_b200.core.backend import from_bf16, to_bf16
        rn.w_in.data = from_bf16(to_bf16(rn.w_in.data))
        rn.w_rec.data = from_bf16(to_bf16(rn.w_rec.data))
    _, ref = O.rate_run(rn, trace=True)
    r = run_rate(rn, 50, precision="float", weight_dtype=wdt, storage_format=fmt, bsr_tile=32)
    err = np.linalg.norm(r - ref, axis=1) / np.maximum(np.linalg.norm(ref, axis=1), 1e-30)
    assert err.max() <= 1e-5, err.max()


@pytest.mark.parametrize("wdt", ["float32", "bfloat16"])
def test_rate_pcsr_many_panels(wdt):
    """Panelled CSR with panels of 64 columns (5 panels, atomics between
    panels, CTAs of a few rows) against the double oracle fed the same
    weights: norm-wise relative error <= 1e-5 per step."""
    rn = wl.rate_net(seed=11, n_in=300, n_out=700, p_in=0.1, p_rec=0.05, steps=30)
    if wdt == "bfloat16":
        from annarchy_b200.core.backend import from_bf16, to_bf16
        rn.w_in.data = from_bf16(to_bf16(rn.w_in.data))
        rn.w_rec.data = from_bf16(to_bf16(rn.w_rec.data))
    _, ref = O.rate_run(rn, trace=True)
    r = run_rate(rn, 30, precision="float", weight_dtype=wdt, storage_format="pcsr", pcsr_panel=64)
    err = np.linalg.norm(r - ref, axis=1) / np.maximum(np.linalg.norm(ref, axis=1), 1e-30)
    assert err.max() <= 1e-5, err.max()


def test_rate_powerlaw_binned_csr():
    """Power-law row lengths: heavy rows (CTA per row, compensated) and light
    rows (vector loads) together match the double oracle."""
    import scipy.sparse as sp
    rng = np.random.default_rng(3)
    n = 3000
    lengths = np.minimum((rng.pareto(1.0, n) * 20 + 5).astype(int), n)
    lengths[:3] = [2500, 2800, 3000]
    rows = np.repeat(np.arange(n), lengths)
    cols = np.concatenate([rng.choice(n, L, replace=False) for L in lengths])
    w = rng.normal(0, 0.01, rows.size)
    m = sp.csr_matrix((w, (rows, cols)), shape=(n, n))
    m.sort_indices()
    rn = wl.RateNet(n_in=n, n_out=n, w_in=m, w_rec=sp.csr_matrix((n, n)),
                    r_in=rng.uniform(0, 1, n), steps=20)
    _, ref = O.rate_run(rn, trace=True)
    r = run_rate(rn, 20, precision="float", weight_dtype="float32")
    err = np.linalg.norm(r - ref, axis=1) / np.maximum(np.linalg.norm(ref, axis=1), 1e-30)
    assert err.max() <= 1e-5, err.max()
