"""Copies of the rate-coded 1000 -> 4000 network (input and recurrent
projections) sharing their weights, run as one RateBatch: every step's
weighted sums of all copies come from the tensor-core block product
(tcgen05, csrc/bsr_tc.cu) inside the step's CUDA graph.

Every copy is checked two ways:
* against a numpy restatement of the same arithmetic (weights and the rates
  the product reads rounded to bfloat16, sums and states in float32), within
  1e-4 norm-wise relative error (the tensor cores add the products in their
  own order; a rate that rounds to the other bfloat16 neighbour changes a
  sum by at most 2^-9 of one term);
* against its own double-precision oracle run with the exact weights
  (oracle/anb_oracle.c, the reference's operation order), which bounds the
  error of the bfloat16 storage: below 1e-2 norm-wise after 50 steps."""
import numpy as np
import pytest

from annarchy_b200 import Network, Neuron, RateBatch
from annarchy_b200 import workloads as wl
from annarchy_b200.core.backend import from_bf16, to_bf16

pytestmark = pytest.mark.gpu

STEPS = 50


def _bf(x):
    return from_bf16(to_bf16(np.asarray(x, dtype=np.float32)))


def _numpy_copy(rn, r_in, steps):
    w_in = rn.w_in.copy()
    w_in.data = _bf(w_in.data)
    w_rec = rn.w_rec.copy()
    w_rec.data = _bf(w_rec.data)
    x_in = _bf(r_in)
    r = np.zeros(rn.n_out, dtype=np.float32)
    tau, dt = np.float32(rn.tau), np.float32(rn.dt)
    for _ in range(steps):
        s = (w_in @ x_in + w_rec @ _bf(r)).astype(np.float32)
        r = r + dt * ((s - r) / tau)
        r = np.maximum(r, np.float32(0.0)).astype(np.float32)
    return r


@pytest.mark.parametrize("batch", [32, 128])
def test_rate_batch_matches_every_copy(batch):
    from oracle import oracle as O
    rn = wl.rate_net(seed=42)
    rng = np.random.default_rng(5)
    X = rng.uniform(0.0, 1.0, (batch, rn.n_in))
    tpl = Network(dt=rn.dt, seed=42)
    inp = tpl.create(rn.n_in, Neuron(parameters="r = 0.0"))
    out = tpl.create(rn.n_out, Neuron(parameters=dict(tau=rn.tau),
                                      equations="tau*dr/dt + r = sum(exc) : min=0.0"))
    tpl.connect(inp, out, "exc").from_sparse(wl.to_from_sparse(rn.w_in))
    tpl.connect(out, out, "exc").from_sparse(wl.to_from_sparse(rn.w_rec))
    rb = RateBatch(tpl, batch)
    rb.compile()
    try:
        rb.set(inp, "r", X)
        rb.simulate_steps(STEPS)
        got = rb.get(out, "r")
        assert got.shape == (batch, rn.n_out) and np.all(np.isfinite(got))
        for b in range(0, batch, max(1, batch // 8)):
            want = _numpy_copy(rn, X[b], STEPS)
            err = np.linalg.norm(got[b] - want) / np.linalg.norm(want)
            assert err < 1e-4, (b, err)
            rn_b = wl.RateNet(rn.n_in, rn.n_out, rn.w_in, rn.w_rec, X[b], rn.tau, rn.dt, STEPS)
            exact, _ = O.rate_run(rn_b, steps=STEPS)
            err64 = np.linalg.norm(got[b] - exact) / np.linalg.norm(exact)
            assert err64 < 1e-2, (b, err64)
        # the same rates in every copy give the same result in every copy
        rb.net.reset()
        rb.set(inp, "r", X[0])
        rb.simulate_steps(STEPS)
        same = rb.get(out, "r")
        assert np.array_equal(same, np.broadcast_to(same[0], same.shape))
        assert rb.net._backend.native.device_error() == 0
    finally:
        rb.close()
