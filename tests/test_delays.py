"""Synaptic delays: the reference's known answers (tests_python/RateSynapse/
test_RateDelays.py and SpikeSynapse/test_SpikingDelays.py, read as text),
the oracle's delay queues against a literal restatement of the reference's
algorithm, and the CUDA path against the oracle (bit-exact in double
precision)."""
from collections import deque

import numpy as np
import pytest

import annarchy_b200 as ann
from annarchy_b200 import workloads as wl
from oracle import oracle as orc


# ---------------------------------------------------------------- host logic
def test_delay_conversion_and_property():
    net = ann.Network(dt=0.1)
    a = net.create(10, ann.Neuron(parameters="r = 0.0"))
    b = net.create(10, ann.Neuron(equations="r = sum(ff)"))
    p = net.connect(a, b, "ff")
    p.all_to_all(weights=1.0, delays=1.5)
    assert p.uniform_delay == 15 and p.max_delay == 15 and p.delay == pytest.approx(1.5)
    p.delay = 0.2
    assert p.uniform_delay == 2 and p.max_delay == 15
    with pytest.raises(ValueError):
        p.delay = [[0.1]] * 10
    q = net.connect(a, b, "ff2")
    q.one_to_one(weights=1.0, delays=0.0)
    assert q.uniform_delay == 1 and q.max_delay == 1 and q.delay == pytest.approx(0.1)
    r = net.connect(a, b, "ff3")
    r.one_to_one(weights=1.0, delays=ann.DiscreteUniform(1, 5))    # ms: 10..50 steps
    assert r.uniform_delay == -1 and r.max_delay == 50
    assert all(10 <= s <= 50 for s in r._delay_steps)
    r.delay = [[0.3]] * 10
    assert r.delay == [[pytest.approx(0.3)]] * 10
    with pytest.raises(ValueError):
        r.delay = [[0.3, 0.4]] + [[0.3]] * 9


def _py_coba(cn, steps, d_exc, d_inh):
    """Literal restatement of the reference's step with delays: the
    population's spike queue (push_front after the update, entry d - 1 read by
    a uniform delay d; Population/SingleThreadGenerator.py:425-433), and for
    per-synapse delays the projection's ring of pending (post, synapse) lists
    filled from the previous step's spikes (SingleThread/LIL.py:915-969)."""
    n, ne, dt, prm = cn.n, cn.n_exc, cn.dt, cn.params
    v, ge, gi = cn.v0.astype(float).copy(), np.zeros(n), np.zeros(n)
    rr = np.zeros(n, dtype=int)
    refr = int(cn.refractory / dt)
    projs = []
    for m, off, d, tgt in ((cn.w_exc, 0, d_exc, 0), (cn.w_inh, ne, d_inh, 1)):
        m = m.tocsr()
        rows = [(m.indptr[i], m.indptr[i + 1]) for i in range(n)]
        out = {}                       # pre -> [(post, synapse)], ascending post
        for i, (b, e) in enumerate(rows):
            for j in range(b, e):
                out.setdefault(int(m.indices[j]) + off, []).append((i, j))
        uni = np.ndim(d) == 0
        dmax = int(d or 1) if uni else int(np.max(d))
        ring = None if uni else [[[] for _ in range(n)] for _ in range(dmax)]
        projs.append(dict(w=m.data, out=out, uni=uni, d=d, dmax=dmax, ring=ring, idx=0, tgt=tgt))
    qlen = max(p["dmax"] for p in projs)
    queue = deque([[] for _ in range(qlen)])
    raster = []
    for t in range(steps):
        for p in projs:
            g = ge if p["tgt"] == 0 else gi
            if p["uni"]:
                for pre in queue[max(1, int(p["d"] or 1)) - 1]:
                    for i, j in p["out"].get(pre, []):
                        g[i] += p["w"][j]
            else:
                for pre in queue[0]:
                    for i, j in p["out"].get(pre, []):
                        p["ring"][(p["idx"] + int(p["d"][j]) - 1) % p["dmax"]][i].append(j)
                for i in range(n):
                    for j in p["ring"][p["idx"]][i]:
                        g[i] += p["w"][j]
                    p["ring"][p["idx"]][i].clear()
                p["idx"] = (p["idx"] + 1) % p["dmax"]
        in_ref = np.where(rr > 0, 0, 1)
        for i in range(n):
            _v = (prm["El"] + prm["Erev_exc"] * ge[i] + prm["Erev_inh"] * gi[i] + prm["I"]
                  - ge[i] * v[i] - gi[i] * v[i] - v[i]) / prm["tau"]
            _ge = -ge[i] / prm["tau_exc"]
            _gi = -gi[i] / prm["tau_inh"]
            v[i] += dt * _v * in_ref[i]
            ge[i] += dt * _ge
            gi[i] += dt * _gi
            rr[i] -= 1 - in_ref[i]
        spiked = []
        for i in range(n):
            if in_ref[i] and v[i] > prm["Vt"]:
                v[i] = prm["Vr"]
                spiked.append(i)
                rr[i] = refr
                raster.append((t, i))
        queue.appendleft(spiked)
        queue.pop()
    return raster, v, ge, gi


def _small_coba(seed=3):
    cn = wl.coba_net(seed=seed, n=60, p=0.2, steps=250, w_exc=1.5, w_inh=4.0, drive=22.0)
    return cn


def _oracle_raster(cn, steps, delays):
    out = orc.coba_run(cn, orc.coba_projections(cn, delays=delays), steps=steps)
    return list(zip(out["spike_steps"].tolist(), out["spike_idx"].tolist())), out


@pytest.mark.parametrize("kind", ["uniform", "per_synapse"])
def test_oracle_spike_delays_match_reference_algorithm(kind):
    cn = _small_coba()
    rng = np.random.default_rng(5)
    if kind == "uniform":
        delays = (7, 3)
    else:
        delays = (rng.integers(1, 9, cn.w_exc.nnz), rng.integers(1, 4, cn.w_inh.nnz))
    ras_py, v, ge, gi = _py_coba(cn, 250, *delays)
    ras_o, out = _oracle_raster(cn, 250, delays)
    assert len(ras_py) > 50
    assert ras_o == ras_py
    assert np.array_equal(out["v"], v) and np.array_equal(out["g_exc"], ge)
    assert np.array_equal(out["g_inh"], gi)


def test_oracle_uniform_equals_equal_per_synapse_delays():
    cn = wl.coba_net(seed=4, n=400, p=0.05, steps=600)
    a = orc.coba_run(cn, orc.coba_projections(cn, delays=(12, 5)), steps=600)
    b = orc.coba_run(cn, orc.coba_projections(
        cn, delays=(np.full(cn.w_exc.nnz, 12), np.full(cn.w_inh.nnz, 5))), steps=600)
    assert a["n_spikes"] > 100
    for k in ("spike_steps", "spike_idx", "v", "g_exc", "g_inh"):
        assert np.array_equal(a[k], b[k])


def _py_rate(rn, steps, d_in, d_rec):
    """The reference's rate-coded step with delays: each population's queue of
    its last max_delay rates (filled with the initial rates; push_front after
    the update), a delay d reading entry d - 1."""
    r = np.zeros(rn.n_out)
    dm = max(int(np.max(d_rec)) if d_rec is not None else 1, 1)
    queue = deque([r.copy() for _ in range(dm)])
    trace = []
    for _ in range(steps):
        s_tot = np.zeros(rn.n_out)
        for m, d, rec in ((rn.w_in, d_in, False), (rn.w_rec, d_rec, True)):
            m = m.tocsr()
            for i in range(rn.n_out):
                s = 0.0
                for j in range(m.indptr[i], m.indptr[i + 1]):
                    c = m.indices[j]
                    if not rec:
                        x = rn.r_in[c]
                    elif d is None or np.ndim(d) == 0:
                        x = queue[max(1, int(d or 1)) - 1][c]
                    else:
                        x = queue[int(d[j]) - 1][c]
                    s += x * m.data[j]
                s_tot[i] += s
        for i in range(rn.n_out):
            _r = (s_tot[i] - r[i]) / rn.tau
            r[i] += rn.dt * _r
            if r[i] < 0.0:
                r[i] = 0.0
        queue.appendleft(r.copy())
        queue.pop()
        trace.append(r.copy())
    return np.array(trace)


@pytest.mark.parametrize("kind", ["uniform", "per_synapse"])
def test_oracle_rate_delays_match_reference_algorithm(kind):
    rn = wl.rate_net(seed=11, n_in=20, n_out=30, p_in=0.3, p_rec=0.3, steps=40)
    d_rec = 4 if kind == "uniform" else np.random.default_rng(2).integers(1, 7, rn.w_rec.nnz)
    tr_py = _py_rate(rn, 40, None, d_rec)
    _, tr = orc.rate_run(rn, 40, trace=True, delays=(None, d_rec))
    assert np.array_equal(tr, tr_py)


# ---------------------------------------------------------------- GPU: known answers
def _kat_net(delays):
    net = ann.Network(dt=1.0)
    # r_t = [-1, 0, 2, 5, 9, 14, 20, ...]
    p1 = net.create(3, ann.Neuron(equations="r = r + t : init = -1"))
    # r = sum(ff): the weighted sum of the step
    p2 = net.create(3, ann.Neuron(equations="r = sum(ff)"))
    proj = net.connect(p1, p2, "ff", synapse=ann.Synapse(psp="pre.r * w"))
    proj.one_to_one(weights=1.0, delays=delays)
    net.compile()
    return net, p2, proj


@pytest.mark.gpu
def test_kat_uniform_delay():
    """test_RateDelays.py:233-302 (test_get_delay, test_set_delay,
    test_configured_delay_local, test_modified_delay_local)."""
    net, p2, proj = _kat_net(10.0)
    np.testing.assert_allclose(proj.delay, 10.0)
    net.reset()
    net.simulate(10)
    np.testing.assert_allclose(p2.r, -1.0)
    net.simulate(1)
    np.testing.assert_allclose(p2.r, -1.0)
    net.simulate(4)
    np.testing.assert_allclose(p2.r, 9.0)
    net.reset()
    proj.delay = 5.0
    np.testing.assert_allclose(proj.delay, 5.0)
    net.simulate(5)
    np.testing.assert_allclose(p2.r, -1.0)
    net.simulate(1)
    np.testing.assert_allclose(p2.r, -1.0)
    net.simulate(4)
    np.testing.assert_allclose(p2.r, 9.0)
    proj.delay = 2.0
    np.testing.assert_allclose(proj.delay, 2.0)
    net.close()


@pytest.mark.gpu
def test_kat_nonuniform_delay():
    """test_RateDelays.py:380-410 (test_configured_nonuniform_delay,
    test_modified_nonuniform_delay)."""
    net, p2, proj = _kat_net(ann.DiscreteUniform(1, 5))
    net.reset()
    proj.delay = [[3], [5], [2]]
    net.simulate(5)
    np.testing.assert_allclose(p2.r, [0.0, -1.0, 2.0])
    net.reset()
    proj.delay = [[3], [5], [2]]
    proj.delay = [[3.0], [3.0], [3.0]]
    net.simulate(10)
    np.testing.assert_allclose(p2.r, [20.0, 20.0, 20.0])
    net.close()


# ---------------------------------------------------------------- GPU: parity with the oracle
def _raster(mon):
    s, r = mon.spike_arrays()
    return s, r


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["uniform", "per_synapse"])
def test_coba_delays_bit_exact(kind):
    cn = wl.coba_net(seed=21, n=400, p=0.05, steps=2000)
    rng = np.random.default_rng(8)
    delays = (15, 8) if kind == "uniform" else (rng.integers(1, 21, cn.w_exc.nnz), None)
    ref = orc.coba_run(cn, orc.coba_projections(cn, delays=delays), steps=2000)
    net, pop, mon = wl.build_coba_network(cn, "double", delays=delays)
    net.compile()
    assert net.engine == "grid"
    net.simulate_steps(2000)
    s, r = _raster(mon)
    assert ref["n_spikes"] > 500
    assert np.array_equal(s, ref["spike_steps"]) and np.array_equal(r, ref["spike_idx"])
    assert np.array_equal(pop.v, ref["v"]) and np.array_equal(pop.g_exc, ref["g_exc"])
    assert np.array_equal(pop.g_inh, ref["g_inh"])
    # reset: the same run again
    net.reset()
    net.simulate_steps(2000)
    s2, r2 = _raster(mon)
    assert np.array_equal(s2, s) and np.array_equal(r2, r)
    net.close()


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["uniform", "per_synapse"])
def test_coba_delays_float(kind):
    """Fast mode: same firing rate as the double oracle within 3 % over 2000
    steps, identical raster over the first 200 steps."""
    cn = wl.coba_net(seed=21, n=400, p=0.05, steps=2000)
    rng = np.random.default_rng(8)
    delays = (15, 8) if kind == "uniform" else (rng.integers(1, 21, cn.w_exc.nnz), None)
    ref = orc.coba_run(cn, orc.coba_projections(cn, delays=delays), steps=2000)
    net, pop, mon = wl.build_coba_network(cn, "float", delays=delays)
    net.compile()
    net.simulate_steps(2000)
    s, r = _raster(mon)
    assert abs(s.size - ref["n_spikes"]) <= 0.03 * ref["n_spikes"]
    early = ref["spike_steps"] < 200
    assert np.array_equal(s[s < 200], ref["spike_steps"][early])
    assert np.array_equal(r[s < 200], ref["spike_idx"][early])
    net.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["double", "float"])
@pytest.mark.parametrize("kind", ["uniform", "per_synapse"])
def test_rate_delays(precision, kind):
    """Rate net 100 -> 200 with delayed input and recurrent projections:
    double bit-exact, float <= 1e-5 norm-wise relative error per step."""
    rn = wl.rate_net(seed=9, n_in=100, n_out=200, p_in=0.1, p_rec=0.05, steps=200)
    rng = np.random.default_rng(4)
    delays = (3, 5) if kind == "uniform" else (None, rng.integers(1, 7, rn.w_rec.nnz))
    _, tr = orc.rate_run(rn, 200, trace=True, delays=delays)
    net, pop, mon = wl.build_rate_network(rn, precision, delays=delays)
    net.compile()
    net.simulate_steps(200)
    got = mon.get("r")
    if precision == "double":
        assert np.array_equal(got, tr)
    else:
        err = np.linalg.norm(got - tr, axis=1) / np.maximum(np.linalg.norm(tr, axis=1), 1e-30)
        assert err.max() <= 1e-5, err.max()
    net.close()
