"""Batched instances: uneven-size spiking networks in one persistent launch.

CPU: packing, structure checks, generated module compiles for sm_100a.
GPU: every instance bit-exact against its own oracle run in double
precision; firing rates within tolerance in single precision."""
import numpy as np
import pytest

from annarchy_b200 import workloads as wl
from annarchy_b200.core.batch import SMEM_LIMIT
from annarchy_b200.runtime import lib as L


def _cns(sizes, steps, seed=42, p=0.02):
    we = np.linspace(0.2, 1.0, len(sizes))
    wi = np.linspace(2.0, 10.0, len(sizes))[::-1]
    return [wl.coba_net(seed=seed + i, n=int(n), p=p, w_exc=float(we[i]), w_inh=float(wi[i]),
                        steps=steps, skip=True) for i, n in enumerate(sizes)]


def test_skip_generator_matches_bernoulli_density():
    rng = np.random.default_rng(1)
    m = wl.bernoulli_csr_skip(rng, 3000, 2000, 0.02, 1.0)
    assert m.shape == (3000, 2000)
    assert m.has_sorted_indices
    dens = m.nnz / (3000 * 2000)
    assert abs(dens - 0.02) < 0.02 * 0.02          # ~14 sigma for 1.2e5 draws
    # no duplicate entries
    assert m.nnz == m.tocoo().tocsr().nnz
    rows = np.diff(m.indptr)
    assert abs(rows.mean() - 40) < 1 and rows.std() < 10


def _atomic_sets(row_ptr, post):
    """Bank multiplicity of every atomic instruction of the fast delivery:
    positions of one row in the same aligned 128-position block with the
    same index mod 4."""
    worst = []
    for b, e in zip(row_ptr[:-1], row_ptr[1:]):
        q = np.arange(b, e)
        rel = q - (b & ~3)
        sets = (rel // 128) * 4 + rel % 4
        for s in np.unique(sets):
            worst.append(np.bincount(post[q[sets == s]] % 32).max())
    return np.array(worst)


def test_bank_interleave_permutes_rows_and_spreads_banks():
    rng = np.random.default_rng(3)
    lens = rng.integers(0, 400, 60)
    lens[:3] = (0, 1, 5)
    row_ptr = np.zeros(61, dtype=np.int64)
    np.cumsum(lens, out=row_ptr[1:])
    post = np.concatenate([np.sort(rng.choice(8000, n, replace=False)) for n in lens]).astype(np.int32)
    perm = L.bank_interleave(row_ptr, post)
    # a permutation within every row
    for b, e in zip(row_ptr[:-1], row_ptr[1:]):
        assert sorted(perm[b:e].tolist()) == list(range(b, e))
    before, after = _atomic_sets(row_ptr, post), _atomic_sets(row_ptr, post[perm])
    assert after.sum() < 0.7 * before.sum() and after.mean() < 2.0
    with pytest.raises(L.BackendError):
        L.bank_interleave(np.array([0, 5, 3]), np.zeros(5, dtype=np.int32))


@pytest.mark.parametrize("prec,wd", [("float", "bfloat16"), ("float", "float32"), ("double", None)])
def test_batch_module_compiles(prec, wd):
    cns = _cns([300, 1000, 2500, 777, 4000, 8000], 10)
    b, _ = wl.build_batch(cns, prec, wd, dry=True, ctas=4)
    b.compile()
    size, log = L.nvrtc_compile(b.module.source, b.module.options)
    assert size > 0 and "error" not in log.lower()
    assert b.smem <= SMEM_LIMIT


def test_batch_packing():
    sizes = np.random.default_rng(0).integers(1000, 8001, 40)
    cns = _cns(sizes, 10)
    b, _ = wl.build_batch(cns, "float", "bfloat16", dry=True, ctas=16)
    b.compile()
    # every instance in exactly one CTA, CTAs within the shared-memory limit
    assert sorted(b.order.tolist()) == list(range(len(cns)))
    assert b.smem <= SMEM_LIMIT
    load = b.cta_load
    biggest = max(s + 0.01 * c.nnz for s, c in zip(sizes, cns))
    assert load.max() <= load.mean() + biggest
    # slot tables agree with the instances
    n_tab = np.array([cns[i].n for i in b.order])
    assert np.array_equal(np.cumsum(n_tab)[:-1], b.goff[0][1:])
    # the shared-memory ranges of the instances of a CTA do not overlap
    soff = b.native_soff
    cta = b.cta
    for c in range(b.n_cta):
        spans = sorted((soff[s].min(), soff[s].min() + b.inst_bytes[b.order[s]])
                       for s in range(cta[c], cta[c + 1]))
        for (a0, a1), (b0, _) in zip(spans, spans[1:]):
            assert a1 <= b0
        assert spans[-1][1] <= b.smem


def test_batch_rejects_other_structures():
    cns = _cns([300, 400], 10)
    b, members = wl.build_batch(cns, "float", dry=True)
    members[1][0].monitor(members[1][1], "v")
    with pytest.raises(ValueError):
        b.compile()


def test_batch_rejects_oversize_instance():
    cns = _cns([300, 9000], 10, p=0.002)
    b, _ = wl.build_batch(cns, "double", dry=True)
    with pytest.raises(ValueError):
        b.compile()


# ------------------------------------------------------------------- GPU
@pytest.mark.gpu
def test_batch_exact_every_instance_matches_oracle():
    from oracle import oracle as O
    sizes = [200, 1500, 613, 1024, 997, 350, 1300, 64, 800, 1111]
    steps = 1000
    cns = _cns(sizes, steps, p=0.05)
    b, members = wl.build_batch(cns, "double", ctas=4)
    b.compile()
    b.simulate_steps(steps)
    for cn, (net, P, mon) in zip(cns, members):
        ref = O.coba_run(cn)
        s, i = mon.spike_arrays()
        assert ref["n_spikes"] > 0
        assert np.array_equal(s, ref["spike_steps"]) and np.array_equal(i, ref["spike_idx"])
        assert np.array_equal(P.v, ref["v"])
        assert np.array_equal(P.g_exc, ref["g_exc"])
        assert np.array_equal(P.g_inh, ref["g_inh"])
        assert net.current_step == steps
    b.close()


@pytest.mark.gpu
def test_batch_exact_chunked_runs_match_one_run():
    """Several launches (state written back and reloaded) = one launch."""
    cns = _cns([700, 1200, 400], 600, p=0.05)
    outs = []
    for chunks in ([600], [1, 250, 349]):
        b, members = wl.build_batch(cns, "double", ctas=2)
        b.compile()
        for c in chunks:
            b.simulate_steps(c)
        outs.append([(m[2].spike_arrays(), m[1].v.copy()) for m in members])
        b.close()
    for (a, va), (c, vc) in zip(*outs):
        assert np.array_equal(a[0], c[0]) and np.array_equal(a[1], c[1])
        assert np.array_equal(va, vc)


@pytest.mark.gpu
@pytest.mark.parametrize("wd,tol", [("float32", 0.02), ("bfloat16", 0.03)])
def test_batch_float_rates(wd, tol):
    """Single-precision state (float or bfloat16 weights): every instance's
    spike count within `tol` of its double oracle over 2000 steps, and the
    total within 1 %."""
    from oracle import oracle as O
    from annarchy_b200.core.backend import from_bf16, to_bf16
    sizes = [1000, 2500, 4000, 1800, 3300, 1234]
    steps = 2000
    cns = _cns(sizes, steps)
    if wd == "bfloat16":       # the oracle gets the same (rounded) weights
        for cn in cns:
            cn.w_exc.data = from_bf16(to_bf16(cn.w_exc.data))
            cn.w_inh.data = from_bf16(to_bf16(cn.w_inh.data))
    b, members = wl.build_batch(cns, "float", wd, ctas=3)
    b.compile()
    b.simulate_steps(steps)
    tot, tot_ref = 0, 0
    for cn, (net, P, mon) in zip(cns, members):
        ref = O.coba_run(cn)["n_spikes"]
        n = mon.spike_arrays()[1].size
        assert abs(n - ref) <= tol * ref + 5, (cn.n, n, ref)
        tot += n
        tot_ref += ref
    assert abs(tot - tot_ref) / tot_ref < 0.01
    b.close()


@pytest.mark.gpu
def test_batch_reset_reproduces_run():
    cns = _cns([900, 300, 1700], 400, p=0.05)
    b, members = wl.build_batch(cns, "double", ctas=2)
    b.compile()
    b.simulate_steps(400)
    first = [m[2].spike_arrays() for m in members]
    for m in members:
        m[2].get("spike")
    b.reset()
    assert members[0][0].current_step == 0
    b.simulate_steps(400)
    for (s0, r0), m in zip(first, members):
        s1, r1 = m[2].spike_arrays()
        assert np.array_equal(s0, s1) and np.array_equal(r0, r1)
    b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("wd", ["float32", "bfloat16"])
@pytest.mark.parametrize("first_spikes", [(300, 100, 0), (6000, 100, 1500)])
def test_fast_batch_delivers_one_step_of_spikes(wd, first_spikes):
    """The fast delivery of one step's spikes, checked synapse by synapse:
    neurons 0..k-1 of each instance start above threshold and spike at
    step 0; after step 1 every conductance is the sum of the weights of those
    spikes, decayed once. 400 spikes in the CTA take the list the update
    appended them to; 7600 overflow it and are delivered from the spike
    bitmaps in rounds."""
    from annarchy_b200.core.backend import from_bf16, to_bf16
    cns = _cns([6000, 2500, 1500], 10)
    for cn, k in zip(cns, first_spikes):
        cn.v0 = np.full(cn.n, -60.0)
        cn.v0[:k] = -40.0
    b, members = wl.build_batch(cns, "float", wd, ctas=1)
    b.compile()
    assert b.n_cta == 1
    b.simulate_steps(2)
    for cn, k, (net, P, mon) in zip(cns, first_spikes, members):
        spiked = np.zeros(cn.n)
        spiked[:k] = 1.0
        steps, ranks = mon.spike_arrays()
        assert ranks[steps == 0].tolist() == list(range(k))
        we, wi = cn.w_exc.copy(), cn.w_inh.copy()
        if wd == "bfloat16":
            we.data, wi.data = from_bf16(to_bf16(we.data)), from_bf16(to_bf16(wi.data))
        for g, w, pre, tau in ((P.g_exc, we, spiked[:cn.n_exc], cn.params["tau_exc"]),
                               (P.g_inh, wi, spiked[cn.n_exc:], cn.params["tau_inh"])):
            s = w @ pre
            expected = s - 0.1 * s / tau
            np.testing.assert_allclose(np.asarray(g), expected, rtol=2e-6, atol=1e-6)
    b.close()
