"""Copies of one rate-coded network sharing the weights of its projections.

A parameter or input sweep of a rate-coded network runs many copies whose
connectivity and weights are the same; the reference runs each copy as its
own process (Network.parallel_run, ANNarchy/core/Network.py:751-925), each
computing its weighted sums with its own BSR kernel
(ANNarchy/generator/Projection/CUDA/BSR.py:296-392). Here the copies are one
network: every population holds `batch` copies of its neurons (copy-major,
neuron i of copy b at b * size + i), and each step computes the weighted
sums of every projection for all copies at once, Y = X W^T with X the
copies' pre-synaptic rates (batch x n_pre), as one tensor-core product over
the weights stored once as dense 64 x 64 bfloat16 blocks (tcgen05.mma with
the accumulators in tensor memory, csrc/bsr_tc.cu). The neuron updates run
over all copies in one kernel per population; the step is replayed as a
CUDA graph.

    tpl = Network(dt=1.0)                     # the network of one copy
    inp = tpl.create(n_in, Neuron(parameters="r = 0.0"))
    out = tpl.create(n, Neuron(parameters="tau = 10.0",
                               equations="tau * dr/dt + r = sum(exc)"))
    tpl.connect(inp, out, "exc").from_sparse(W)
    rb = RateBatch(tpl, batch=128)
    rb.compile()
    rb.set(inp, "r", X)                       # (128, n_in) or one row for all
    rb.simulate(100.0)
    rb.get(out, "r")                          # (128, n)

Weights are rounded to bfloat16, rates are rounded to bfloat16 as the
product reads them, sums and states are float32.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


class RateBatch:
    def __init__(self, template, batch: int, device: int = 0, graph_steps: int = 32):
        from . import network as N
        if batch % 16 or not 16 <= batch <= 256:
            raise ValueError("batch must be a multiple of 16 between 16 and 256")
        if template.compiled:
            raise RuntimeError("RateBatch: the template network must not be compiled")
        self.template = template
        self.batch = int(batch)
        big = N.Network(dt=template.dt, seed=template._config.get("seed"))
        big.config(precision="float", engine="grid", device=device, graph_steps=graph_steps)
        self.net = big
        self._pop = {}
        for pop in template.populations:
            if pop.neuron_type.type != "rate":
                raise NotImplementedError("RateBatch holds rate-coded populations only")
            self._pop[pop.id] = big.create(self.batch * pop.size, pop.neuron_type, name=pop.name)
        for proj in template.projections:
            if proj.synapse_type.type != "rate" or proj.desc.get("variables"):
                raise NotImplementedError("RateBatch projections are rate-coded weighted sums "
                                          "without synaptic equations")
            if proj.pre is not proj.pre_pop or proj.post is not proj.post_pop:
                raise NotImplementedError("RateBatch projections connect whole populations")
            if proj._csr is None:
                raise RuntimeError(f"projection {proj.name} has no connectivity")
            if proj.max_delay > 1 or proj._delay_steps is not None:
                raise NotImplementedError("RateBatch projections have no synaptic delays")
            bp = big.connect(self._pop[proj.pre_pop.id], self._pop[proj.post_pop.id], proj.target,
                             name=proj.name)
            w = sp.csr_matrix(proj._csr, dtype=np.float64)
            w.sort_indices()
            bp._batched = (self.batch, w)
            bp._storage_format = "bsr_tc"
        self._mon = {}

    # -- construction -----------------------------------------------------------------
    def monitor(self, pop, variables, period: float | None = None):
        """Record `variables` of every copy of `pop` (get() returns arrays
        of shape (records, batch, size))."""
        m = self.net.monitor(self._pop[pop.id], variables, period=period)
        self._mon[id(m)] = pop
        return m

    def compile(self):
        self.net.compile()
        return self

    # -- state ------------------------------------------------------------------------
    def _shape(self, pop):
        return (self.batch, pop.size)

    def set(self, pop, name: str, values):
        """Set attribute `name` of every copy of `pop`: an array (batch,
        size), one row (size,) for all copies, or a scalar."""
        big = self._pop[pop.id]
        if big._locality.get(name) != "local":
            big.set({name: values})
            return
        v = np.broadcast_to(np.asarray(values, dtype=np.float64), self._shape(pop))
        big.set({name: np.ascontiguousarray(v).reshape(-1)})

    def get(self, pop, name: str) -> np.ndarray:
        v = self._pop[pop.id].get(name)
        if np.ndim(v) == 0:
            return v
        return np.asarray(v).reshape(self._shape(pop))

    def sum(self, pop, target: str) -> np.ndarray:
        """Weighted sums of the last step, (batch, size)."""
        return np.asarray(self._pop[pop.id].sum(target)).reshape(self._shape(pop))

    # -- simulation --------------------------------------------------------------------
    def simulate(self, duration: float):
        self.net.simulate(duration)

    def simulate_steps(self, n: int):
        self.net.simulate_steps(int(n))

    def close(self):
        self.net.close()
