"""Run the reference simulator itself on the benchmark workloads — TEST AND
MEASUREMENT INFRASTRUCTURE ONLY (bench.py's reference arm; never the
backend).

The reference (ANNarchy 5.0.3) is installed, unmodified, in baseline/_ref
(``pip install --no-index --no-build-isolation --no-deps --target
baseline/_ref <copy of the reference sources>``). Its generated wrapper is
built through the nanobind stand-in of tests/golden/refshim (a pybind11
module; nanobind is not installed), with cmake, g++ and nvcc of the machine
this runs on, so the OpenMP build targets the host CPU it is timed on and
the CUDA build targets the GPU there (the reference reads the compute
capability from nvidia-smi, ANNarchy/generator/Utils.py:489-515).

    python oracle/ref_run.py --workload coba --paradigm openmp --threads 8 \
        --steps 5 --warmup 2 --workdir /tmp/ref_build

prints one JSON line: compile time, wall time of every timed simulate()
(1 s of model time for the spiking network, 1000 steps for the rate-coded
one), delivered events (spiking) or synapse count, spike counts and, for
the spiking network, the raster of the first timed run as (step, rank)
digests so the caller can compare it with the oracle.

The network is built as tests/golden/make_golden.py builds it: connectivity
injected with from_sparse (shape pre x post), initial potentials as numpy
arrays, every random array from annarchy_b200.workloads (seeded numpy).
Timing: ``net.reset()`` then ``P.v = v0`` before every run (the reference
uploads dirty host arrays at the start of run() on CUDA), then the wall
time of ``net.simulate()`` alone; the spike monitor records, as in the
reference's own benchmarks.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
REF_SITE = os.path.join(REPO, "baseline", "_ref")
SHIM = os.path.join(REPO, "tests", "golden", "refshim")


def available() -> str | None:
    """None when the reference can be run here, else the reason."""
    if not os.path.isdir(os.path.join(REF_SITE, "ANNarchy")):
        return "the reference is not installed in baseline/_ref"
    for tool in ("cmake", "g++"):
        if subprocess.call(["which", tool], stdout=subprocess.DEVNULL,
                           stderr=subprocess.DEVNULL) != 0:
            return f"{tool} not found"
    return None


def child_env() -> dict:
    import pybind11
    env = dict(os.environ)
    env["PYTHONPATH"] = os.pathsep.join([REF_SITE, SHIM, REPO, env.get("PYTHONPATH", "")])
    env["ANB_PYBIND11_INCLUDE"] = pybind11.get_include()
    # the generated host target includes cuda_runtime.h without the CUDA include path
    cuda_inc = "/usr/local/cuda/include"
    env["CPATH"] = os.pathsep.join([cuda_inc, env.get("CPATH", "")])
    return env


def run(workload: str, paradigm: str, threads: int, steps: int, warmup: int, workdir: str,
        timeout: float = 1200.0) -> dict:
    """Run this file in a child process with the reference importable and
    return its JSON line (raises on failure)."""
    os.makedirs(workdir, exist_ok=True)
    cmd = [sys.executable, os.path.abspath(__file__), "--child", "--workload", workload,
           "--paradigm", paradigm, "--threads", str(threads), "--steps", str(steps),
           "--warmup", str(warmup), "--workdir", workdir]
    p = subprocess.run(cmd, env=child_env(), cwd=workdir, capture_output=True, text=True,
                       timeout=timeout)
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    if p.returncode != 0 or not lines:
        raise RuntimeError(f"reference run failed (rc={p.returncode}): "
                           + (p.stderr or p.stdout)[-2000:])
    return json.loads(lines[-1])


def _digest(a) -> str:
    import numpy as np
    return hashlib.sha1(np.ascontiguousarray(a).tobytes()).hexdigest()[:16]


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


def _config(ann, net, paradigm: str, threads: int, workdir: str) -> dict:
    kw = dict(directory=os.path.join(workdir, f"net_{paradigm}"), silent=True)
    if paradigm == "cuda":
        net.config(paradigm="cuda")
        cfg = os.path.join(workdir, "annarchy.json")
        with open(cfg, "w") as f:
            json.dump({"openmp": {"compiler": "g++", "flags": "-march=native -O3"},
                       "cuda": {"compiler": "nvcc", "flags": "", "device": 0,
                                "path": "/usr/local/cuda"}}, f)
        kw["annarchy_json"] = cfg
    else:
        net.config(num_threads=threads)
        kw["compiler_flags"] = "-march=native -O3"      # the reference's default flags
    return kw


def child_coba(args) -> dict:
    import numpy as np
    import ANNarchy as ann
    from annarchy_b200 import workloads as wl
    cn = wl.coba_net(seed=42)
    net = ann.Network(dt=cn.dt, seed=42)
    kw = _config(ann, net, args.paradigm, args.threads, args.workdir)
    P = net.create(cn.n, ann.Neuron(parameters=dict(cn.params), equations=list(wl.COBA_EQUATIONS),
                                    spike=wl.COBA_SPIKE, reset=wl.COBA_RESET,
                                    refractory=wl.COBA_REFRACTORY))
    Pe, Pi = P[: cn.n_exc], P[cn.n_exc:]
    fmt = "csr"
    net.connect(Pe, P, "exc").from_sparse(wl.to_from_sparse(cn.w_exc), storage_format=fmt)
    net.connect(Pi, P, "inh").from_sparse(wl.to_from_sparse(cn.w_inh), storage_format=fmt)
    m = net.monitor(P, ["spike"])
    t0 = time.perf_counter()
    net.compile(**kw)
    compile_s = time.perf_counter() - t0
    out_deg = cn.out_degree()
    model_ms = wl_steps = 10000
    times, events, spikes, first = [], [], [], None
    for it in range(args.warmup + args.steps):
        net.reset()
        P.v = cn.v0
        t0 = time.perf_counter()
        net.simulate(wl_steps * cn.dt)
        t1 = time.perf_counter()
        s, i = _spikes_to_arrays(m.get("spike"))
        if it >= args.warmup:
            times.append(t1 - t0)
            events.append(int(out_deg[i].sum()))
            spikes.append(int(i.size))
            if first is None:
                first = (s, i)
    del model_ms
    return {"workload": "coba", "paradigm": args.paradigm, "threads": args.threads,
            "compile_s": compile_s, "run_s": times, "events": events, "spikes": spikes,
            "time_steps": wl_steps, "raster_steps": _digest(first[0]),
            "raster_idx": _digest(first[1]), "n_spikes_first": int(first[1].size)}


def child_rate(args) -> dict:
    import numpy as np
    import ANNarchy as ann
    from annarchy_b200 import workloads as wl
    rn = wl.rate_net(seed=42)
    net = ann.Network(dt=rn.dt, seed=42)
    kw = _config(ann, net, args.paradigm, args.threads, args.workdir)
    inp = net.create(rn.r_in.size, ann.Neuron(parameters="r=0.0"))
    pop = net.create(rn.w_rec.shape[0], ann.Neuron(parameters=dict(tau=rn.tau),
                                                   equations="tau*dr/dt + r = sum(exc) : min=0.0"))
    net.connect(inp, pop, "exc").from_sparse(wl.to_from_sparse(rn.w_in), storage_format="csr")
    net.connect(pop, pop, "exc").from_sparse(wl.to_from_sparse(rn.w_rec), storage_format="csr")
    t0 = time.perf_counter()
    net.compile(**kw)
    compile_s = time.perf_counter() - t0
    times, final = [], None
    for it in range(args.warmup + args.steps):
        net.reset()
        inp.r = rn.r_in
        t0 = time.perf_counter()
        net.simulate(rn.steps * rn.dt)
        t1 = time.perf_counter()
        if it >= args.warmup:
            times.append(t1 - t0)
            if final is None:
                final = np.asarray(pop.r, dtype=np.float64)
    return {"workload": "rate", "paradigm": args.paradigm, "threads": args.threads,
            "compile_s": compile_s, "run_s": times, "synapses": int(rn.w_in.nnz + rn.w_rec.nnz),
            "time_steps": int(rn.steps), "mean_r_final": float(final.mean()),
            "r_final_digest": _digest(final)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--child", action="store_true")
    ap.add_argument("--workload", default="coba", choices=("coba", "rate"))
    ap.add_argument("--paradigm", default="openmp", choices=("openmp", "cuda"))
    ap.add_argument("--threads", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--workdir", default="/tmp/anb_ref_run")
    args = ap.parse_args()
    if not args.child:
        print(json.dumps(run(args.workload, args.paradigm, args.threads, args.steps, args.warmup,
                             args.workdir)))
        return
    res = child_coba(args) if args.workload == "coba" else child_rate(args)
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
