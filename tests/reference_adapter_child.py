"""Child process of tests/test_reference_adapter.py: runs with the reference
(baseline/_ref) and the stand-ins of tests/golden/refshim importable, builds
a network with the reference's own Python API and instantiates it on this
backend through annarchy_b200.reference_module. Prints one JSON line.

    python tests/reference_adapter_child.py dry   # wiring only (no GPU)
    python tests/reference_adapter_child.py run   # simulate on cuda:0
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))


def build(ann, wl, cn):
    net = ann.Network(dt=cn.dt, seed=7)
    P = net.create(cn.n, ann.Neuron(parameters=dict(cn.params), equations=list(wl.COBA_EQUATIONS),
                                    spike=wl.COBA_SPIKE, reset=wl.COBA_RESET,
                                    refractory=wl.COBA_REFRACTORY))
    Pe, Pi = P[: cn.n_exc], P[cn.n_exc:]
    ce = net.connect(Pe, P, "exc")
    ce.from_sparse(wl.to_from_sparse(cn.w_exc), storage_format="csr")
    ci = net.connect(Pi, P, "inh")
    ci.from_sparse(wl.to_from_sparse(cn.w_inh), storage_format="csr")
    m = net.monitor(P, ["spike"])
    mv = net.monitor(P, ["v"], period=50 * cn.dt)
    return net, P, (ce, ci), m, mv


def main():
    mode = sys.argv[1]
    import ANNarchy as ann
    from annarchy_b200 import reference_module as RM
    from annarchy_b200 import workloads as wl
    cn = wl.coba_net(seed=7, n=400, p=0.05, steps=2000)
    net, P, projs, m, mv = build(ann, wl, cn)
    mod = RM.instantiate(net, dry=(mode == "dry"))
    out = {"mode": mode}
    if mode == "dry":
        ours = [mod._projs[p.id] for p in projs]
        ok = True
        for ref_w, pr in zip((cn.w_exc, cn.w_inh), ours):
            post, row_ptr, cols, w = pr.csr_population_ranks()
            m_ = ref_w.tocsr()
            lengths = np.diff(m_.indptr)
            rows = np.nonzero(lengths > 0)[0]
            ok &= np.array_equal(post, rows)
            ok &= np.array_equal(np.diff(row_ptr), lengths[rows])
            ok &= np.array_equal(w, m_.data)
        out.update(csr_equal=bool(ok), refractory_steps=int(mod._pops[P.id].refractory_steps[0]),
                   recording=[bool(x._recording) for x in mod._mons[P.id]],
                   variables=[list(x.variables) for x in mod._mons[P.id]])
    else:
        P.v = cn.v0
        net.simulate(cn.steps * cn.dt)
        spk = m.get("spike")
        steps = np.concatenate([np.asarray(v, dtype=np.int64) for v in spk.values()])
        idx = np.concatenate([np.full(len(v), k, dtype=np.int64) for k, v in spk.items()])
        order = np.lexsort((idx, steps))
        gold = np.load(os.path.join(HERE, "golden", "coba_small.npz"))
        v_trace = np.asarray(mv.get("v"))
        out.update(spikes=int(idx.size),
                   raster_equal=bool(np.array_equal(steps[order], gold["spike_steps"])
                                     and np.array_equal(idx[order], gold["spike_idx"])),
                   v_equal=bool(np.array_equal(np.asarray(P.v), gold["v_final"])),
                   v_trace_equal=bool(np.array_equal(v_trace, gold["v_trace"])),
                   time=int(mod.get_time()))
    print(json.dumps(out))


if __name__ == "__main__":
    main()
