"""CPU restatement of rate-coded synaptic learning — TEST INFRASTRUCTURE ONLY.

Only the test suite uses this module; the backend never does. Plain Python
floats (IEEE double) in the reference's operation order, for small networks:

* a step (ANNarchy/generator/Template/OpenMPBaseTemplate.py:131-484): the
  weighted sums of every projection (sequential in CSR order,
  ANNarchy/generator/Projection/OpenMP/CSR.py:177-253), the neuron update,
  then every projection's update_synapse (OpenMP/CSR.py:833-865) when
  learning is on and (t - offset) % period == 0;
* update_synapse (Projection/SingleThreadGenerator.py:1575-1700,
  generator/Utils.py:17-210): the global equations, then per dendrite its
  semiglobal equations followed by the local ones of its synapses, each ODE
  block as all increments then the switches (dt replaced by dt * period) and
  the bounds, the weight's switch only while plasticity is on;
* enable_learning(period, offset) (ANNarchy/core/Projection.py:1440-1489):
  offset steps int(int((now % period + offset) % period) / dt), where `now`
  is the time of the reference's default network (Global.get_time()), 0 for
  networks created with Network().

The equations are those of the learning case of tests/golden/make_golden.py:
  tau_alpha * dalpha/dt + alpha = pos(post.r - 0.5)      : postsynaptic
  dbeta/dt = -0.01 * beta                                : projection
  dw/dt = eta * beta * pre.r * post.r - alpha * post.r^2 * w : min = 0
with an output population tau * dr/dt + r = sum(exc) + sum(mod).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


class LearningProjection:
    """CSR rows (post neurons with synapses), columns = pre ranks."""

    def __init__(self, w: sp.csr_matrix, target: str, eta=0.02, tau_alpha=20.0):
        m = sp.csr_matrix(w)
        m.sort_indices()
        lengths = np.diff(m.indptr)
        self.rows = np.nonzero(lengths > 0)[0].tolist()
        self.row_ptr = [int(x) for x in np.concatenate([[0], np.cumsum(lengths[lengths > 0])])]
        self.col = m.indices.tolist()
        self.w = [float(x) for x in m.data]
        self.target = target
        self.alpha = [0.0] * len(self.rows)
        self.beta = 1.0
        self.eta, self.tau_alpha = float(eta), float(tau_alpha)
        self.period, self.offset, self.plasticity, self.update = 1, 0, True, True

    def enable_learning(self, now_ms: float, dt: float, period: float, offset: float):
        now_ms = 0.0                      # the default network's time
        self.period = int(period / dt)
        rel = now_ms % period + offset
        self.offset = int(int(rel % period) / dt)
        self.update = self.plasticity = True

    def weighted_sums(self, r_pre, n_post):
        out = [0.0] * n_post
        for i, post in enumerate(self.rows):
            s = 0.0
            for j in range(self.row_ptr[i], self.row_ptr[i + 1]):
                s += r_pre[self.col[j]] * self.w[j]
            out[post] = 0.0 + s
        return out

    def update_synapse(self, t, r_pre, r_post, dt):
        if not self.update or (t - self.offset) % self.period != 0:
            return
        _dt = dt * self.period
        _beta = -0.01 * self.beta
        self.beta += _dt * _beta
        beta, eta = self.beta, self.eta
        for i, post in enumerate(self.rows):
            rp = r_post[post]
            _alpha = (-self.alpha[i] + max(rp - 0.5, 0.0)) / self.tau_alpha
            self.alpha[i] += _dt * _alpha
            alpha = self.alpha[i]
            for j in range(self.row_ptr[i], self.row_ptr[i + 1]):
                _w = rp * (-rp * alpha * self.w[j] + r_pre[self.col[j]] * beta * eta)
                if self.plasticity:
                    self.w[j] += _dt * _w
                    if self.w[j] < 0.0:
                        self.w[j] = 0.0


def run(r_in, projections, n_post: int, steps: int, tau: float = 10.0, dt: float = 1.0,
        events=()):
    """Simulate `steps` steps; `events` = [(step, callable(now_ms))] run
    before that step. Returns the recorded r (steps, n_post)."""
    r_pre = [float(x) for x in r_in]
    r = [0.0] * n_post
    rec = []
    todo = sorted(events, key=lambda e: e[0])
    for t in range(steps):
        while todo and todo[0][0] == t:
            todo.pop(0)[1](t * dt)
        sums = {"exc": [0.0] * n_post, "mod": [0.0] * n_post}
        for p in projections:
            s = p.weighted_sums(r_pre, n_post)
            sums[p.target] = [a + b for a, b in zip(sums[p.target], s)]
        for i in range(n_post):
            _r = (sums["exc"][i] + sums["mod"][i] - r[i]) / tau
            r[i] += dt * _r
        for p in projections:
            p.update_synapse(t, r_pre, r, dt)
        rec.append(list(r))
    return np.asarray(rec)
