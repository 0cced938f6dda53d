"""Generate the golden fixtures in this folder by running the reference
simulator (ANNarchy 5.0.3) itself, in its single-thread CPU build.

Run from the repository root, in a container that has the reference
sources, g++, cmake and the pybind11 wheel in an offline wheelhouse:

    python tests/golden/make_golden.py            # all cases
    python tests/golden/make_golden.py coba_small # one case

Paths (environment variables, with their defaults):

    ANB_REFERENCE    the reference's source tree (read only)   /root/reference
    ANB_GOLDEN_WORK  scratch folder for the build and networks  /tmp/anb_golden
    ANB_WHEELHOUSE   offline wheelhouse holding pybind11        /opt/wheelhouse

Set-up, done once under the scratch folder (nothing is written to the
reference tree and no reference source enters this repository):

1. copy the reference sources to <work>/src and build its Cython extensions
   there (``setup.py build_ext --inplace``);
2. install pybind11 from the offline wheelhouse into <work>/pb;
3. put ``refshim/`` on PYTHONPATH: an own ``nanobind`` stand-in whose CMake
   config builds the reference's generated wrapper as a pybind11 module, and
   empty ``h5py``/``matplotlib`` modules that the reference imports but these
   cases do not use.

Every network is compiled with ``-march=native -O3 -ffp-contract=off`` so
that no multiply-add is contracted: the fixtures are the IEEE-754 double
results of the reference's own operation order. All random arrays come from
``annarchy_b200.workloads`` (seeded numpy) and are injected through
``from_sparse`` and attribute arrays, so the same inputs can be rebuilt on any
machine with the same numpy.
"""
from __future__ import annotations

import json
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("ANB_REFERENCE", "/root/reference")
WORK = os.environ.get("ANB_GOLDEN_WORK", "/tmp/anb_golden")
WHEELHOUSE = os.environ.get("ANB_WHEELHOUSE", "/opt/wheelhouse")
SRC = os.path.join(WORK, "src")
PB = os.path.join(WORK, "pb")
FLAGS = "-march=native -O3 -ffp-contract=off"


def setup_env() -> dict:
    os.makedirs(WORK, exist_ok=True)
    if not os.path.isdir(SRC):
        shutil.copytree(REF, SRC)
    if not os.path.exists(os.path.join(SRC, ".built")):
        subprocess.check_call([sys.executable, "setup.py", "build_ext", "--inplace"], cwd=SRC,
                              stdout=subprocess.DEVNULL)
        open(os.path.join(SRC, ".built"), "w").close()
    if not os.path.isdir(os.path.join(PB, "pybind11")):
        subprocess.check_call([sys.executable, "-m", "pip", "install", "--no-index", "--quiet",
                               "--find-links", WHEELHOUSE, "--target", PB, "pybind11"])
    env = dict(os.environ)
    env["PYTHONPATH"] = os.pathsep.join([SRC, os.path.join(HERE, "refshim"), PB, REPO])
    env["ANB_PYBIND11_INCLUDE"] = os.path.join(PB, "pybind11", "include")
    return env


# ---------------------------------------------------------------------------
# Cases (executed in a child process with the reference importable)
# ---------------------------------------------------------------------------

def _spikes_to_arrays(spk: dict):
    import numpy as np
    steps, idx = [], []
    for n, ts in spk.items():
        steps.extend(ts)
        idx.extend([n] * len(ts))
    steps = np.asarray(steps, dtype=np.int64)
    idx = np.asarray(idx, dtype=np.int64)
    order = np.lexsort((idx, steps))
    return steps[order].astype(np.int32), idx[order].astype(np.int32)


def _coba_neuron(ann, params):
    from annarchy_b200 import workloads as wl
    return ann.Neuron(parameters=dict(params), equations=list(wl.COBA_EQUATIONS),
                      spike=wl.COBA_SPIKE, reset=wl.COBA_RESET, refractory=wl.COBA_REFRACTORY)


def case_rate(name, seed, n_in, n_out, p_in, p_rec, steps, record_steps):
    import numpy as np
    import ANNarchy as ann
    from annarchy_b200 import workloads as wl
    rn = wl.rate_net(seed=seed, n_in=n_in, n_out=n_out, p_in=p_in, p_rec=p_rec, steps=steps)
    net = ann.Network(dt=rn.dt, seed=seed)
    net.config(num_threads=1)
    inp = net.create(n_in, ann.Neuron(parameters="r=0.0"))
    li = ann.Neuron(parameters=dict(tau=rn.tau), equations="tau*dr/dt + r = sum(exc) : min=0.0")
    pop = net.create(n_out, li)
    p1 = net.connect(inp, pop, "exc")
    p1.from_sparse(wl.to_from_sparse(rn.w_in), storage_format="csr")
    p2 = net.connect(pop, pop, "exc")
    p2.from_sparse(wl.to_from_sparse(rn.w_rec), storage_format="csr")
    m = net.monitor(pop, "r")
    net.compile(directory=os.path.join(WORK, "net_" + name), compiler_flags=FLAGS, silent=True)
    inp.r = rn.r_in
    net.simulate(steps * rn.dt)
    r = np.asarray(m.get("r"))
    out = dict(seed=seed, n_in=n_in, n_out=n_out, p_in=p_in, p_rec=p_rec, steps=steps,
               digest_in=wl.csr_digest(rn.w_in), digest_rec=wl.csr_digest(rn.w_rec),
               record_steps=np.asarray(record_steps, dtype=np.int64),
               r_at=r[record_steps], r_sum=r.sum(axis=1), r_final=r[-1])
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)


def case_coba(name, seed, n, p, steps, v_every, stdp=False):
    import numpy as np
    import ANNarchy as ann
    from annarchy_b200 import workloads as wl
    cn = wl.coba_net(seed=seed, n=n, p=p, steps=steps)
    net = ann.Network(dt=cn.dt, seed=seed)
    net.config(num_threads=1)
    P = net.create(n, _coba_neuron(ann, cn.params))
    Pe, Pi = P[: cn.n_exc], P[cn.n_exc:]
    extra = {}
    if stdp:
        # plastic E->E (weights U[0, 0.5]), static E->I and I->all
        rng = np.random.default_rng(seed + 1000)
        w_ee = wl.bernoulli_csr(rng, cn.n_exc, cn.n_exc, p, lambda k: rng.uniform(0.0, 0.5, k))
        w_ei = cn.w_exc[cn.n_exc:]
        syn = ann.STDP(**wl.STDP_PARAMS)
        ee = net.connect(Pe, Pe, "exc", synapse=syn)
        ee.from_sparse(wl.to_from_sparse(w_ee), storage_format="csr")
        ei = net.connect(Pe, Pi, "exc")
        ei.from_sparse(wl.to_from_sparse(w_ei), storage_format="csr")
        extra.update(digest_ee=wl.csr_digest(w_ee), digest_ei=wl.csr_digest(w_ei))
    else:
        ce = net.connect(Pe, P, "exc")
        ce.from_sparse(wl.to_from_sparse(cn.w_exc), storage_format="csr")
    ci = net.connect(Pi, P, "inh")
    ci.from_sparse(wl.to_from_sparse(cn.w_inh), storage_format="csr")
    m = net.monitor(P, ["spike"])
    mv = net.monitor(P, ["v"], period=v_every * cn.dt) if v_every else None
    net.compile(directory=os.path.join(WORK, "net_" + name), compiler_flags=FLAGS, silent=True)
    P.v = cn.v0
    net.simulate(steps * cn.dt)
    s_steps, s_idx = _spikes_to_arrays(m.get("spike"))
    out = dict(seed=seed, n=n, p=p, steps=steps, digest_exc=wl.csr_digest(cn.w_exc),
               digest_inh=wl.csr_digest(cn.w_inh), spike_steps=s_steps, spike_idx=s_idx,
               v_final=np.asarray(P.v), g_exc_final=np.asarray(P.g_exc),
               g_inh_final=np.asarray(P.g_inh), **extra)
    if mv is not None:
        out["v_every"] = v_every
        out["v_trace"] = np.asarray(mv.get("v"))
    if stdp:
        out["w_ee_final"] = np.concatenate([np.asarray(d, dtype=np.float64) for d in ee.w])
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)


def case_io(name):
    """A state file written by the reference's Network.save(): an STDP
    network (plastic E->E, I->all with a uniform 0.5 ms delay) after 50 steps
    (io_ref_state.npz), and the values to expect when it is loaded
    (io_ref_meta.npz)."""
    import numpy as np
    import ANNarchy as ann
    from annarchy_b200 import workloads as wl
    cn = wl.coba_net(seed=3, n=200, p=0.1)
    net = ann.Network(dt=cn.dt, seed=1)
    net.config(num_threads=1)
    P = net.create(cn.n, _coba_neuron(ann, cn.params))
    Pe, Pi = P[: cn.n_exc], P[cn.n_exc:]
    ee = net.connect(Pe, Pe, "exc", synapse=ann.STDP(**wl.STDP_PARAMS))
    ee.from_sparse(wl.to_from_sparse(wl.stdp_matrix(cn, 3, 0.1)), storage_format="csr")
    ci = net.connect(Pi, P, "inh")
    ci.from_sparse(wl.to_from_sparse(cn.w_inh), delays=0.5, storage_format="csr")
    net.compile(directory=os.path.join(WORK, "net_" + name), compiler_flags=FLAGS, silent=True)
    P.v = cn.v0
    net.simulate(50 * cn.dt)
    net.save(os.path.join(HERE, "io_ref_state.npz"))
    meta = dict(v=np.asarray(P.v), w_ee=np.concatenate([np.asarray(d, dtype=np.float64) for d in ee.w]),
                x_ee=np.concatenate([np.asarray(d, dtype=np.float64) for d in ee.x]))
    # the other direction: a file written by this backend's save() (same
    # network, halved weights, other potentials) loaded by the reference
    import annarchy_b200 as b2
    ours = b2.Network(dt=cn.dt, seed=1)
    Q = ours.create(cn.n, wl.coba_neuron(cn.params))
    oee = ours.connect(Q[: cn.n_exc], Q[: cn.n_exc], "exc", synapse=b2.STDP(**wl.STDP_PARAMS))
    oee.from_sparse(wl.to_from_sparse(wl.stdp_matrix(cn, 3, 0.1) * 0.5))
    oci = ours.connect(Q[cn.n_exc:], Q, "inh")
    oci.from_sparse(wl.to_from_sparse(cn.w_inh), delays=0.5)
    Q.v = np.linspace(-70.0, -40.0, cn.n)
    path = os.path.join(WORK, "ours_state.npz")
    ours.save(path)
    net.load(path)
    w_loaded = np.concatenate([np.asarray(d, dtype=np.float64) for d in ee.w])
    w_ours = np.concatenate([np.asarray(d, dtype=np.float64) for d in oee.get("w")])
    meta["reference_loaded_ours"] = bool(np.array_equal(w_loaded, w_ours) and
                                         np.array_equal(np.asarray(P.v), Q.v))
    np.savez_compressed(os.path.join(HERE, "io_ref_meta.npz"), **meta)


def case_parser(name):
    """Description dicts of the reference parser for a set of models."""
    import ANNarchy as ann
    from ANNarchy.parser.AnalyseNeuron import analyse_neuron
    from ANNarchy.parser.AnalyseSynapse import analyse_synapse
    from models_catalog import NEURONS, SYNAPSES
    net = ann.Network(dt=0.1)
    res = {"neurons": {}, "synapses": {}}
    for key, spec in NEURONS.items():
        d = analyse_neuron(ann.Neuron(**spec), net.id)
        res["neurons"][key] = _digest_desc(d)
    for key, spec in SYNAPSES.items():
        d = analyse_synapse(ann.Synapse(**spec), net.id)
        res["synapses"][key] = _digest_desc(d)
    with open(os.path.join(HERE, name + ".json"), "w") as f:
        json.dump(res, f, indent=1, sort_keys=True)


def _digest_desc(d):
    keep = {}
    keep["type"] = d.get("type")
    keep["local"] = list(d.get("local", []))
    keep["global"] = list(d.get("global", []))
    keep["semiglobal"] = list(d.get("semiglobal", []))
    keep["targets"] = list(d.get("targets", []))
    keep["variables"] = [dict(name=v["name"], cpp=v.get("cpp"), switch=v.get("switch"),
                              bounds=v.get("bounds", {}), init=v.get("init"),
                              locality=v.get("locality"), method=v.get("method"))
                         for v in d.get("variables", [])]
    keep["parameters"] = [dict(name=v["name"], init=v.get("init"), locality=v.get("locality"))
                          for v in d.get("parameters", [])]
    if d.get("spike"):
        keep["spike_cond"] = d["spike"]["spike_cond"]
        keep["spike_reset"] = [r["cpp"] for r in d["spike"]["spike_reset"]]
    if "refractory" in d:
        keep["refractory"] = d["refractory"]
    for k in ("pre_spike", "post_spike"):
        if d.get(k):
            keep[k] = [v["cpp"] for v in d[k]]
    if d.get("psp"):
        keep["psp"] = d["psp"].get("cpp")
    return keep


def case_connect_patterns(name):
    """Gaussian and difference-of-Gaussians connectivity built by the
    reference's connector code (ANNarchy/cython_ext/Connector.pyx:433-575)
    for 1-, 2- and 3-D geometries: per pattern the post ranks, the pre ranks
    and weights of every dendrite (concatenated) and the dendrite sizes."""
    import numpy as np
    import ANNarchy as ann
    from ANNarchy.cython_ext.Connector import dog, gaussian
    net = ann.Network(dt=0.1, seed=1)
    neuron = ann.Neuron(parameters="r = 0.0")
    pats = {
        "g2_self": ("gaussian", (12, 10), None, dict(amp=1.0, sigma=0.3, limit=0.01)),
        "g2_map": ("gaussian", (15, 9), (8, 6), dict(amp=2.5, sigma=0.2, limit=0.05)),
        "g1": ("gaussian", (40,), (30,), dict(amp=1.0, sigma=0.1, limit=0.01)),
        "g3_self": ("gaussian", (5, 4, 3), None, dict(amp=0.7, sigma=0.35, limit=0.02)),
        "dog2_self": ("dog", (12, 10), None, dict(amp_pos=1.0, sigma_pos=0.2, amp_neg=0.5,
                                                  sigma_neg=0.5, limit=0.01)),
        "dog2_map": ("dog", (10, 10), (7, 9), dict(amp_pos=1.5, sigma_pos=0.15, amp_neg=1.0,
                                                   sigma_neg=0.3, limit=0.02)),
    }
    out = {}
    for key, (kind, g_pre, g_post, kw) in pats.items():
        pre = net.create(g_pre, neuron)
        post = pre if g_post is None else net.create(g_post, neuron)
        allow = g_post is not None
        if kind == "gaussian":
            lil = gaussian(pre, post, kw["amp"], kw["sigma"], 0.0, kw["limit"], allow, "lil", "post_to_pre")
        else:
            lil = dog(pre, post, kw["amp_pos"], kw["sigma_pos"], kw["amp_neg"], kw["sigma_neg"], 0.0,
                      kw["limit"], allow, "lil", "post_to_pre")
        out[key + "__post"] = np.asarray(list(lil.post_rank), dtype=np.int64)
        out[key + "__sizes"] = np.asarray([len(r) for r in lil.pre_rank], dtype=np.int64)
        out[key + "__pre"] = np.concatenate([np.asarray(r, dtype=np.int64) for r in lil.pre_rank])
        out[key + "__w"] = np.concatenate([np.asarray(w, dtype=np.float64) for w in lil.w])
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)


def spike_dict_fixture(seed=5, n=40, steps=2000):
    """A seeded raster (dict rank -> ascending steps, some neurons silent)
    for the spike-analysis fixtures."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out = {}
    for k in range(n):
        rate = 0.0 if k % 7 == 3 else rng.uniform(0.001, 0.05)
        steps_k = np.nonzero(rng.random(steps) < rate)[0] + 200
        out[k] = [int(t) for t in steps_k]
    return out


def case_spike_analysis(name):
    """The reference's spike-analysis functions (ANNarchy/core/Monitor.py:
    1091-1330, cython_ext/Transformations.pyx:23-108) on a seeded raster at
    dt = 0.1 ms."""
    import numpy as np
    import ANNarchy as ann
    from ANNarchy.core import Monitor as M
    import ANNarchy.cython_ext.Transformations as T
    ann.setup(dt=0.1)
    spikes = spike_dict_fixture()
    out = {"ranks": np.asarray(list(spikes), dtype=np.int64),
           "sizes": np.asarray([len(v) for v in spikes.values()], dtype=np.int64),
           "steps": np.concatenate([np.asarray(v, dtype=np.int64) for v in spikes.values()])}
    t, r = M.raster_plot(spikes, dt=0.1)
    out["raster_t"], out["raster_r"] = t, r
    out["hist_dt"] = M.histogram(spikes, dt=0.1)
    out["hist_05"] = M.histogram(spikes, bins=0.5, dt=0.1)
    out["hist_pn"] = M.histogram(spikes, bins=1.0, per_neuron=True, dt=0.1)
    out["hist_win"] = M.histogram(spikes, bins=0.5, recording_window=(100, 2400), dt=0.1)
    out["isi"] = np.asarray(M.inter_spike_interval(spikes, dt=0.1))
    isi_pn = M.inter_spike_interval(spikes, ranks=[1, 2, 5, 9], per_neuron=True, dt=0.1)
    out["isi_pn_keys"] = np.asarray(sorted(isi_pn), dtype=np.int64)
    out["isi_pn_vals"] = np.concatenate([np.asarray(isi_pn[k]) for k in sorted(isi_pn)])
    out["cv"] = np.asarray(M.coefficient_of_variation(spikes, dt=0.1))
    out["cv_ranks"] = np.asarray(M.coefficient_of_variation(spikes, ranks=[0, 4, 8, 12], dt=0.1))
    out["mean_fr"] = np.float64(M.mean_fr(spikes, dt=0.1))
    out["mean_fr_dur"] = np.float64(M.mean_fr(spikes, duration=2500, dt=0.1))
    for smooth in (0.0, 5.0):
        for start, stop in ((0, 2300), (150, 2250)):
            key = f"{int(smooth)}_{start}"
            out["srate_" + key] = T.smoothed_rate({"data": spikes, "start": start, "stop": stop}, smooth)
            out["prate_" + key] = T.population_rate({"data": spikes, "start": start, "stop": stop},
                                                    smooth)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)


LEARN_SYNAPSE = dict(
    parameters="eta = 0.02 : projection\ntau_alpha = 20.0 : projection",
    equations="""
        tau_alpha * dalpha/dt + alpha = pos(post.r - 0.5) : postsynaptic
        dbeta/dt = -0.01 * beta : projection, init=1.0
        dw/dt = eta * beta * pre.r * post.r - alpha * post.r^2 * w : min=0.0
    """)


def learning_inputs(seed=9, n_in=30, n_out=20):
    """Rates of the input population and the (pre, post) weight matrix of the
    rate-coded learning case."""
    import numpy as np
    from annarchy_b200 import workloads as wl
    rng = np.random.default_rng(seed)
    r_in = rng.uniform(0.0, 1.0, n_in)
    w = wl.bernoulli_csr(rng, n_out, n_in, 0.4, lambda k: rng.uniform(0.0, 0.3, k))
    return r_in, w


def case_rate_learning(name, steps=200):
    """A rate-coded network whose synapses learn (semiglobal, local and
    global equations; min bound on w), one projection updating every step and
    one every 3 steps from an offset (enable_learning(period, offset))."""
    import numpy as np
    import ANNarchy as ann
    from annarchy_b200 import workloads as wl
    r_in, w = learning_inputs()
    net = ann.Network(dt=1.0, seed=1)
    net.config(num_threads=1)
    inp = net.create(r_in.size, ann.Neuron(parameters="r = 0.0"))
    out = net.create(w.shape[0], ann.Neuron(parameters="tau = 10.0",
                                            equations="tau * dr/dt + r = sum(exc) + sum(mod)"))
    syn = ann.Synapse(**LEARN_SYNAPSE)
    p1 = net.connect(inp, out, "exc", synapse=syn)
    p1.from_sparse(wl.to_from_sparse(w), storage_format="csr")
    p2 = net.connect(inp, out, "mod", synapse=syn)
    p2.from_sparse(wl.to_from_sparse(w * 0.5), storage_format="csr")
    m = net.monitor(out, "r")
    net.compile(directory=os.path.join(WORK, "net_" + name), compiler_flags=FLAGS, silent=True)
    inp.r = r_in
    net.simulate(7.0)
    p2.enable_learning(period=3.0, offset=1.0)
    net.simulate((steps - 7) * 1.0)
    out_d = dict(r=np.asarray(m.get("r")),
                 w1=np.concatenate([np.asarray(d, dtype=np.float64) for d in p1.w]),
                 w2=np.concatenate([np.asarray(d, dtype=np.float64) for d in p2.w]),
                 alpha1=np.asarray(p1.alpha, dtype=np.float64), alpha2=np.asarray(p2.alpha, dtype=np.float64),
                 beta1=np.float64(p1.beta), beta2=np.float64(p2.beta), steps=np.int64(steps))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out_d)


def case_connectivity_file(name):
    """A connectivity file written by the reference's
    Projection.save_connectivity() (ragged dendrites, a uniform delay), its
    dense connectivity matrix and receptive fields."""
    import numpy as np
    import ANNarchy as ann
    from annarchy_b200 import workloads as wl
    rng = np.random.default_rng(17)
    w = wl.bernoulli_csr(rng, 12, 15, 0.3, lambda k: rng.uniform(0.1, 1.0, k))
    net = ann.Network(dt=0.5, seed=1)
    net.config(num_threads=1)
    a = net.create((3, 5), ann.Neuron(parameters="r = 0.0"))
    b = net.create((4, 3), ann.Neuron(equations="r = sum(exc)"))
    p = net.connect(a, b, "exc")
    p.from_sparse(wl.to_from_sparse(w), delays=1.5, storage_format="lil")
    net.compile(directory=os.path.join(WORK, "net_" + name), compiler_flags=FLAGS, silent=True)
    p.save_connectivity(os.path.join(HERE, "connectivity_ref.npz"))
    np.savez_compressed(os.path.join(HERE, name + "_meta.npz"), matrix=p.connectivity_matrix(),
                        rf=p.receptive_fields())


def case_self_connections(name):
    """Which self-synapses the reference's random connectors keep. The
    decision is made on the objects connected (ConnectorMethods.py:283-284,
    344-345, 410-411): a view connected to its own population, or two views
    of the same neurons made separately, keep pre == post pairs; the same
    object on both sides drops them. Per case: the network seed, then the
    LIL that the reference's connector builds from a generator seeded like
    the network's (its post ranks, dendrite sizes and concatenated pre
    ranks) for fixed_probability, and the number of pre == post pairs for
    fixed_number_pre and fixed_number_post (whose draws differ from this
    backend's, so only their self-pair rule is compared)."""
    import numpy as np
    import ANNarchy as ann
    neuron = ann.Neuron(parameters="r = 0.0")
    out = {}
    cases = {
        # key: (kind, seed, population size, pre slice, post slice, argument)
        "fp_view_to_pop": ("fixed_probability", 3, 60, (40, 60), None, 0.3),
        "fp_pop_to_view": ("fixed_probability", 4, 60, None, (10, 30), 0.3),
        "fp_pop_to_pop": ("fixed_probability", 5, 60, None, None, 0.3),
        "fp_same_view": ("fixed_probability", 6, 60, (0, 40), "same", 0.3),
        "fp_two_views": ("fixed_probability", 7, 60, (0, 40), (0, 40), 0.3),
        "fnpre_view_to_pop": ("fixed_number_pre", 8, 60, (40, 60), None, 10),
        "fnpre_pop_to_pop": ("fixed_number_pre", 9, 60, None, None, 10),
        "fnpost_view_to_pop": ("fixed_number_post", 10, 60, None, (40, 60), 10),
        "fnpost_pop_to_pop": ("fixed_number_post", 11, 60, None, None, 10),
    }
    for key, (kind, seed, size, pre_sl, post_sl, arg) in cases.items():
        net = ann.Network(dt=0.1, seed=seed)
        pop = net.create(size, neuron)
        pre = pop if pre_sl is None else pop[pre_sl[0]:pre_sl[1]]
        if post_sl == "same":
            post = pre
        else:
            post = pop if post_sl is None else pop[post_sl[0]:post_sl[1]]
        proj = net.connect(pre, post, "exc")
        getattr(proj, kind)(arg, 1.0)
        lil = proj._connection_method(proj.pre, proj.post, np.random.default_rng(seed),
                                      *proj._connection_args)
        post_r = np.asarray(list(lil.post_rank), dtype=np.int64)
        pre_r = [np.asarray(r, dtype=np.int64) for r in lil.pre_rank]
        out[key + "__seed"] = np.int64(seed)
        out[key + "__self_pairs"] = np.int64(sum(int(np.sum(r == p)) for p, r in zip(post_r, pre_r)))
        if kind == "fixed_probability":
            out[key + "__post"] = post_r
            out[key + "__sizes"] = np.asarray([len(r) for r in pre_r], dtype=np.int64)
            out[key + "__pre"] = np.concatenate(pre_r) if pre_r else np.zeros(0, np.int64)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)


def case_stp(name, seed, n, p, steps, g_every):
    """The COBA network with its excitatory projection through short-term
    plasticity: raster, final state, the per-synapse x and u, and g_exc
    recorded every g_every steps (the reference records conductances right
    after the transmissions, before the neurons' update)."""
    import numpy as np
    import ANNarchy as ann
    from annarchy_b200 import workloads as wl
    from stp_model import STP_EQUATIONS, STP_PARAMETERS, STP_PRE_SPIKE
    cn = wl.coba_net(seed=seed, n=n, p=p, steps=steps)
    net = ann.Network(dt=cn.dt, seed=seed)
    net.config(num_threads=1)
    P = net.create(n, _coba_neuron(ann, cn.params))
    Pe, Pi = P[: cn.n_exc], P[cn.n_exc:]
    stp = ann.Synapse(parameters=STP_PARAMETERS, equations=STP_EQUATIONS, pre_spike=STP_PRE_SPIKE)
    ce = net.connect(Pe, P, "exc", synapse=stp)
    ce.from_sparse(wl.to_from_sparse(cn.w_exc), storage_format="csr")
    ci = net.connect(Pi, P, "inh")
    ci.from_sparse(wl.to_from_sparse(cn.w_inh), storage_format="csr")
    m = net.monitor(P, ["spike"])
    mg = net.monitor(P, ["g_exc"], period=g_every * cn.dt)
    net.compile(directory=os.path.join(WORK, "net_" + name), compiler_flags=FLAGS, silent=True)
    P.v = cn.v0
    net.simulate(steps * cn.dt)
    s_steps, s_idx = _spikes_to_arrays(m.get("spike"))
    out = dict(seed=seed, n=n, p=p, steps=steps, g_every=g_every,
               digest_exc=wl.csr_digest(cn.w_exc), digest_inh=wl.csr_digest(cn.w_inh),
               spike_steps=s_steps, spike_idx=s_idx, v_final=np.asarray(P.v),
               g_exc_final=np.asarray(P.g_exc), g_inh_final=np.asarray(P.g_inh),
               g_exc_trace=np.asarray(mg.get("g_exc")),
               x_final=np.concatenate([np.asarray(d, dtype=np.float64) for d in ce.x]),
               u_final=np.concatenate([np.asarray(d, dtype=np.float64) for d in ce.u]))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)


def case_spiking_continuous(name, steps=30):
    """A spiking synapse with equations evaluated every step (decaying pre-
    and post-traces set at pre- and post-synaptic spikes, w their sum), the
    network of the reference's test_SpikingContinuousUpdate: the synapse's
    w and traces after every step."""
    import numpy as np
    import ANNarchy as ann
    net = ann.Network(dt=1.0, seed=1)
    net.config(num_threads=1)
    pre_n = ann.Neuron(equations="mp=t", spike="(modulo(t,3))")
    post_n = ann.Neuron(equations="mp=t", spike="(modulo(t,5))")
    syn = ann.Synapse(pre_spike="pre_trace=pre.mp : init=0.0",
                      post_spike="post_trace=post.mp : init=0.0",
                      equations="""
                          post_trace = post_trace -1 : min=0.0
                          pre_trace = pre_trace -1 : min=0.0
                          w = post_trace + pre_trace
                      """)
    p0 = net.create(1, pre_n)
    p1 = net.create(1, post_n)
    proj = net.connect(p0, p1, "exc", syn)
    proj.all_to_all(weights=0.0)
    net.compile(directory=os.path.join(WORK, "net_" + name), compiler_flags=FLAGS, silent=True)
    rows = []
    for _ in range(steps):
        net.simulate(1)
        rows.append([float(np.ravel(proj.w)[0]), float(np.ravel(proj.pre_trace)[0]),
                     float(np.ravel(proj.post_trace)[0])])
    np.savez_compressed(os.path.join(HERE, name + ".npz"), steps=steps,
                        w_pre_post=np.asarray(rows))


def case_covariance(name, steps=3):
    """The covariance rule with the pre/post population means
    (models_catalog "covariance"): six pre neurons with random rates, two
    post neurons with rates 1 and 3, weights after each step."""
    import numpy as np
    import ANNarchy as ann
    from models_catalog import SYNAPSES
    net = ann.Network(dt=1.0, seed=1)
    net.config(num_threads=1)
    neuron = ann.Neuron(parameters="r=0")
    pre = net.create(6, neuron)
    post = net.create(2, neuron)
    proj = net.connect(pre, post, "exc", synapse=ann.Synapse(**SYNAPSES["covariance"]))
    proj.all_to_all(weights=1.0)
    net.compile(directory=os.path.join(WORK, "net_" + name), compiler_flags=FLAGS, silent=True)
    pr = np.random.default_rng(9).random(6)
    pre.r = pr
    post.r = np.array([1.0, 3.0])
    ws = []
    for _ in range(steps):
        net.simulate(1)
        ws.append(np.array([np.asarray(d, dtype=np.float64) for d in proj.w]))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), pre_r=pr, post_r=np.array([1.0, 3.0]),
                        w=np.asarray(ws))


CASES = {
    "parser_strings": (case_parser, dict()),
    "rate_small": (case_rate, dict(seed=7, n_in=100, n_out=200, p_in=0.1, p_rec=0.05, steps=100,
                                   record_steps=list(range(100)))),
    "rate_c1": (case_rate, dict(seed=42, n_in=1000, n_out=4000, p_in=0.1, p_rec=0.02, steps=1000,
                                record_steps=[0, 1, 9, 99, 499, 998, 999])),
    "coba_small": (case_coba, dict(seed=7, n=400, p=0.05, steps=2000, v_every=50)),
    "coba_c2": (case_coba, dict(seed=42, n=4000, p=0.02, steps=10000, v_every=0)),
    "stdp_small": (case_coba, dict(seed=11, n=400, p=0.05, steps=2000, v_every=0, stdp=True)),
    "io": (case_io, {}),
    "connect_patterns": (case_connect_patterns, {}),
    "spike_analysis": (case_spike_analysis, {}),
    "rate_learning": (case_rate_learning, {}),
    "connectivity_file": (case_connectivity_file, {}),
    "self_connections": (case_self_connections, {}),
    "stp_small": (case_stp, dict(seed=5, n=400, p=0.05, steps=2000, g_every=50)),
    "spiking_continuous": (case_spiking_continuous, {}),
    "covariance": (case_covariance, {}),
}


def main():
    if len(sys.argv) > 2 and sys.argv[1] == "--run":
        fn, kw = CASES[sys.argv[2]]
        fn(sys.argv[2], **kw)
        return
    env = setup_env()
    names = sys.argv[1:] or list(CASES)
    for nm in names:
        print("golden:", nm, flush=True)
        subprocess.check_call([sys.executable, os.path.abspath(__file__), "--run", nm], env=env,
                              cwd=WORK)


if __name__ == "__main__":
    main()
