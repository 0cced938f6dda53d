"""Sharding a spiking network by post neurons over ranks (one process per
rank, spikes exchanged after every step). Host logic on CPU with gloo; the
sharded simulation on one GPU with two ranks exchanging over gloo (no kernel
waits on another rank): the oracle's raster, and bit for bit the unsharded
run."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from annarchy_b200 import workloads as wl
from annarchy_b200.core.shard import chunk_words, owned_range


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


@pytest.mark.parametrize("n,world", [(400, 2), (1000, 3), (33, 2), (100000, 8), (64, 4)])
def test_owned_ranges_partition(n, world):
    ranges = [owned_range(n, r, world) for r in range(world)]
    assert ranges[0][0] == 0 and ranges[-1][1] == n
    for (a, b), (c, d) in zip(ranges, ranges[1:]):
        assert b == c
    assert all(lo % 32 == 0 for lo, _ in ranges)
    assert all(hi - lo <= 32 * chunk_words(n, world) for lo, hi in ranges)


def _gather_worker(rank, world, port, q):
    import torch.distributed as dist
    from datetime import timedelta
    from annarchy_b200.core.shard import Exchange
    os.environ["MASTER_ADDR"], os.environ["MASTER_PORT"] = "127.0.0.1", str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        ex = Exchange(rank, world)
        out = ex.all_gather(np.full(3, rank + 1, dtype=np.uint32))
        q.put((rank, out.tolist()))
    finally:
        dist.destroy_process_group()


def _run_ranks(target, world, args, timeout=600):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, world, port, *args, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = {}
    try:
        for _ in range(world):
            rank, val = q.get(timeout=timeout)
            results[rank] = val
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    return results


def test_exchange_all_gather_gloo():
    res = _run_ranks(_gather_worker, 2, ())
    assert res[0] == res[1] == [1, 1, 1, 2, 2, 2]


def test_shard_builds_local_rows():
    from annarchy_b200.core.backend import CompiledNetwork
    cn = wl.coba_net(seed=7, n=400, p=0.05, steps=10)
    rows = []
    for rank in (0, 1):
        net = wl.build_coba_network(cn, "double", "grid", record=False)[0]
        net.config(shard=(rank, 2))
        be = CompiledNetwork(net, dry=True)
        be.build()
        lo, hi = be.owned[0]
        rows.append(be.layout[0]["rows"])
        assert (lo, hi) == owned_range(400, rank, 2)
    # E->all rows: all 400 post neurons split between the ranks
    assert sum(rows) == np.count_nonzero(np.diff(cn.w_exc.indptr))


def _coba_worker(rank, world, port, precision, steps, q, backend="gloo"):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"], os.environ["MASTER_PORT"] = "127.0.0.1", str(port)
    if backend == "nccl":
        import torch
        torch.cuda.set_device(0)
    dist.init_process_group(backend, rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        cn = wl.coba_net(seed=21, n=400, p=0.05, steps=steps)
        w_ee = wl.stdp_matrix(cn, 21, 0.05)
        net, P, mon = wl.build_coba_network(cn, precision, "grid", stdp_w_ee=w_ee)
        net.config(shard=(rank, world))
        net.compile()
        net.simulate_steps(steps)
        s, r = mon.spike_arrays()
        lo, hi = net._backend.owned[P.id]
        q.put((rank, (s, r, P.v[lo:hi].copy(), lo, hi)))
        net.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_sharded_coba_stdp_equals_oracle():
    """Two ranks, each owning half of the 400 neurons and their incoming
    synapses (plastic E->E included), exchanging spike bitmaps after every
    step: the union of their rasters is the oracle's over 1000 steps, and
    rasters and potentials equal an unsharded run on the same GPU bit for bit
    (against the oracle the potentials agree to 1e-9: the STDP weights use the
    device's exp(), last-ulp different from the host's)."""
    from oracle import oracle as orc
    steps = 1000
    res = _run_ranks(_coba_worker, 2, ("double", steps))
    cn = wl.coba_net(seed=21, n=400, p=0.05, steps=steps)
    w_ee = wl.stdp_matrix(cn, 21, 0.05)
    projs = orc.coba_projections(cn, stdp_w_ee=w_ee, stdp=dict(wl.STDP_PARAMS))
    ref = orc.coba_run(cn, projs, steps=steps)
    s = np.concatenate([res[r][0] for r in (0, 1)])
    i = np.concatenate([res[r][1] for r in (0, 1)])
    order = np.lexsort((i, s))
    assert ref["n_spikes"] > 200
    assert np.array_equal(s[order], ref["spike_steps"]) and np.array_equal(i[order], ref["spike_idx"])
    net, P, mon = wl.build_coba_network(cn, "double", "grid", stdp_w_ee=w_ee)
    net.compile()
    net.simulate_steps(steps)
    s1, i1 = mon.spike_arrays()
    assert np.array_equal(s[order], s1) and np.array_equal(i[order], i1)
    v_full = P.v.copy()
    net.close()
    for r in (0, 1):
        _, _, v, lo, hi = res[r]
        assert np.array_equal(v, v_full[lo:hi])
        np.testing.assert_allclose(v, ref["v"][lo:hi], rtol=1e-9)


def _nccl_worker(rank, world, port, q):
    _coba_worker(rank, world, port, "double", 600, q, backend="nccl")


@pytest.mark.gpu
def test_sharded_exchange_in_device_memory_over_nccl():
    """The exchange over NCCL gathers the bitmap words in place in device
    memory, ordered on the network's stream (no host copy). One rank on the
    one GPU of this machine (an NCCL group of one): the sharded path, its
    padded bitmap and the in-place gather reproduce the unsharded run bit
    for bit."""
    steps = 600
    res = _run_ranks(_nccl_worker, 1, ())
    cn = wl.coba_net(seed=21, n=400, p=0.05, steps=steps)
    w_ee = wl.stdp_matrix(cn, 21, 0.05)
    net, P, mon = wl.build_coba_network(cn, "double", "grid", stdp_w_ee=w_ee)
    net.compile()
    net.simulate_steps(steps)
    s1, i1 = mon.spike_arrays()
    v_full = P.v.copy()
    net.close()
    s, i, v, lo, hi = res[0]
    assert i1.size > 100
    assert np.array_equal(s, s1) and np.array_equal(i, i1)
    assert (lo, hi) == (0, 400) and np.array_equal(v, v_full)
