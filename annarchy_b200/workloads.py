"""Seeded synthetic networks for the benchmark configurations.

Every random array is drawn here from ``numpy.random.default_rng(seed)`` and
injected into a network explicitly (connectivity through ``from_sparse``,
initial states as arrays), because the reference simulator's own
``Uniform``/``Normal`` draw from an unseeded generator unless given ``rng=``
(ANNarchy/core/Random.py:88-92) and two runs of one script differ.

Connectivity is returned as ``scipy.sparse.csr_matrix`` of shape
(post, pre) with column indices ascending in every row: the order in which
the reference's ``from_sparse`` builds each dendrite
(ANNarchy/core/ConnectorMethods.py:763-796). ``to_from_sparse`` gives the
(pre, post) matrix that ``Projection.from_sparse`` takes.

Workloads (sizes and values as in the benchmark configurations):

* ``rate_net``   - constant-rate inputs feeding leaky integrators through a
  Bernoulli-masked input projection and a recurrent projection (the
  1000 -> 4000 rate-coded net, 1000 steps at dt = 1 ms).
* ``coba_net``   - conductance-based LIF network, 80 % excitatory, Bernoulli
  connectivity p = 0.02, constant weights 0.6 / 6.7, v0 ~ U[-60, -50] mV
  (the 4000-neuron spiking net, 10,000 steps at dt = 0.1 ms). A constant
  drive ``I`` is part of the neuron model: without it the network as
  specified never fires.
* ``sweep_matrix`` - 100k-row recurrent matrices with the four connectivity
  structures used for the format study.
* ``batched_coba`` - uneven-size instances of the spiking net for the
  batched sweep.
"""
from __future__ import annotations

import hashlib
from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp


def bernoulli_csr(rng: np.random.Generator, n_post: int, n_pre: int, p: float,
                  weights) -> sp.csr_matrix:
    """(post, pre) matrix whose entries exist independently with probability p.

    ``weights`` is either a scalar or a callable ``f(n) -> ndarray`` that gives
    the values of the n existing entries in row-major order.
    """
    mask = rng.random((n_post, n_pre)) < p
    rows, cols = np.nonzero(mask)
    nnz = rows.size
    if callable(weights):
        data = np.asarray(weights(nnz), dtype=np.float64)
    else:
        data = np.full(nnz, float(weights), dtype=np.float64)
    m = sp.csr_matrix((data, (rows, cols)), shape=(n_post, n_pre))
    m.sort_indices()
    return m


def bernoulli_csr_skip(rng: np.random.Generator, n_post: int, n_pre: int, p: float,
                       weights) -> sp.csr_matrix:
    """Same distribution as bernoulli_csr (every entry independently with
    probability p) drawn in O(nnz): the gaps between consecutive entries of
    the row-major sequence are geometric(p). Row-major order, sorted."""
    total = n_post * n_pre
    pos = np.zeros(0, dtype=np.int64)
    last = -1
    while True:
        k = int(max(1024, (total - last) * p * 1.05 + 64))
        gaps = rng.geometric(p, size=k).astype(np.int64)
        nxt = last + np.cumsum(gaps)
        inside = nxt < total
        pos = np.concatenate([pos, nxt[inside]])
        if not inside.all():
            break
        last = int(nxt[-1])
    rows = pos // n_pre
    cols = (pos % n_pre).astype(np.int32)
    nnz = pos.size
    if callable(weights):
        data = np.asarray(weights(nnz), dtype=np.float64)
    else:
        data = np.full(nnz, float(weights), dtype=np.float64)
    indptr = np.zeros(n_post + 1, dtype=np.int64)
    np.cumsum(np.bincount(rows, minlength=n_post), out=indptr[1:])
    return sp.csr_matrix((data, cols, indptr), shape=(n_post, n_pre))


def to_from_sparse(m: sp.csr_matrix) -> sp.csr_matrix:
    """(post, pre) -> the (pre, post) layout ``Projection.from_sparse`` expects."""
    return m.T.tocsr()


def csr_digest(m: sp.csr_matrix) -> str:
    """Short content hash of a CSR matrix (structure and values)."""
    h = hashlib.sha256()
    h.update(np.asarray(m.indptr, dtype=np.int64).tobytes())
    h.update(np.asarray(m.indices, dtype=np.int64).tobytes())
    h.update(np.asarray(m.data, dtype=np.float64).tobytes())
    return h.hexdigest()[:16]


@dataclass
class RateNet:
    n_in: int
    n_out: int
    w_in: sp.csr_matrix          # (n_out, n_in)
    w_rec: sp.csr_matrix         # (n_out, n_out)
    r_in: np.ndarray             # (n_in,)
    tau: float = 10.0
    dt: float = 1.0
    steps: int = 1000

    @property
    def nnz(self) -> int:
        return int(self.w_in.nnz + self.w_rec.nnz)


def rate_net(seed: int = 42, n_in: int = 1000, n_out: int = 4000,
             p_in: float = 0.1, p_rec: float = 0.02,
             sd_in: float = 0.05, sd_rec: float = 0.02,
             steps: int = 1000) -> RateNet:
    rng = np.random.default_rng(seed)
    w_in = bernoulli_csr(rng, n_out, n_in, p_in, lambda n: rng.normal(0.0, sd_in, n))
    w_rec = bernoulli_csr(rng, n_out, n_out, p_rec, lambda n: rng.normal(0.0, sd_rec, n))
    r_in = rng.uniform(0.0, 1.0, n_in)
    return RateNet(n_in, n_out, w_in, w_rec, r_in, steps=steps)


COBA_PARAMS = dict(El=-60.0, Vr=-60.0, Erev_exc=0.0, Erev_inh=-80.0, Vt=-50.0,
                   tau=20.0, tau_exc=5.0, tau_inh=10.0, I=20.0)
COBA_EQUATIONS = [
    "tau * dv/dt = (El - v) + g_exc * (Erev_exc - v) + g_inh * (Erev_inh - v) + I",
    "tau_exc * dg_exc/dt = - g_exc",
    "tau_inh * dg_inh/dt = - g_inh",
]
COBA_SPIKE = "v > Vt"
COBA_RESET = "v = Vr"
COBA_REFRACTORY = 5.0

STDP_PARAMS = dict(tau_plus=16.8, tau_minus=33.7, A_plus=0.005, A_minus=0.00525,
                   w_min=0.0, w_max=1.0)


@dataclass
class CobaNet:
    n: int
    n_exc: int
    w_exc: sp.csr_matrix         # (n, n_exc): excitatory pre ranks 0..n_exc-1
    w_inh: sp.csr_matrix         # (n, n - n_exc): inhibitory pre ranks n_exc..n-1
    v0: np.ndarray
    params: dict = field(default_factory=lambda: dict(COBA_PARAMS))
    dt: float = 0.1
    steps: int = 10000
    refractory: float = COBA_REFRACTORY

    @property
    def nnz(self) -> int:
        return int(self.w_exc.nnz + self.w_inh.nnz)

    def out_degree(self) -> np.ndarray:
        """Number of efferent synapses of every neuron (over both projections)."""
        deg = np.zeros(self.n, dtype=np.int64)
        deg[: self.n_exc] = np.bincount(self.w_exc.indices, minlength=self.n_exc)
        deg[self.n_exc:] = np.bincount(self.w_inh.indices, minlength=self.n - self.n_exc)
        return deg


def coba_net(seed: int = 42, n: int = 4000, exc_frac: float = 0.8, p: float = 0.02,
             w_exc: float = 0.6, w_inh: float = 6.7, drive: float = 20.0,
             steps: int = 10000, skip: bool = False) -> CobaNet:
    """skip=True draws the connectivity with bernoulli_csr_skip (same
    distribution, O(nnz) time and memory; a different sample)."""
    rng = np.random.default_rng(seed)
    n_exc = int(round(n * exc_frac))
    v0 = rng.uniform(-60.0, -50.0, n)
    gen = bernoulli_csr_skip if skip else bernoulli_csr
    we = gen(rng, n, n_exc, p, w_exc)
    wi = gen(rng, n, n - n_exc, p, w_inh)
    params = dict(COBA_PARAMS)
    params["I"] = float(drive)
    return CobaNet(n, n_exc, we, wi, v0, params=params, steps=steps)


# ---------------------------------------------------------------------------
# 100k-row matrices for the storage-format study
# ---------------------------------------------------------------------------

def sweep_matrix(kind: str, seed: int = 42, n: int = 100_000, mean_nnz: int = 100,
                 sd: float = 0.01) -> sp.csr_matrix:
    """(n, n) recurrent matrices with the four connectivity structures.

    kind: 'uniform' (exactly mean_nnz distinct random columns per row),
    'powerlaw' (Zipf-like row lengths, exponent 2, clipped to [k_min, 20000]
    with k_min chosen so the mean is close to mean_nnz), 'local' (Gaussian
    neighbourhood on a square grid, sigma 5, cutoff 15) or 'blocks' (64x64
    dense blocks at 2 % block density).
    """
    rng = np.random.default_rng(seed)
    if kind == "uniform":
        # exactly mean_nnz distinct columns per row: draw a few more than
        # needed, drop repeats, keep a uniformly random subset of the rest
        k = mean_nnz + 16
        draws = np.sort(rng.integers(0, n, (n, k)), axis=1)
        keys = rng.random((n, k))
        dup = np.zeros_like(draws, dtype=bool)
        dup[:, 1:] = draws[:, 1:] == draws[:, :-1]
        keys[dup] = 2.0
        short = np.nonzero((~dup).sum(axis=1) < mean_nnz)[0]
        pick = np.argpartition(keys, mean_nnz - 1, axis=1)[:, :mean_nnz]
        cols = np.take_along_axis(draws, pick, axis=1)
        for r in short:                       # rare: too many repeats in the draw
            cols[r] = rng.choice(n, mean_nnz, replace=False)
        cols.sort(axis=1)
        indptr = np.arange(0, n * mean_nnz + 1, mean_nnz, dtype=np.int64)
        data = rng.normal(0.0, sd, n * mean_nnz)
        return sp.csr_matrix((data, cols.ravel(), indptr), shape=(n, n))
    if kind == "powerlaw":
        kmax = 20000
        # continuous power law p(k) ~ k^-2 on [kmin, kmax]; mean = kmin*kmax*ln(kmax/kmin)/(kmax-kmin)
        lo, hi = 1.0, float(mean_nnz)
        for _ in range(60):
            mid = 0.5 * (lo + hi)
            m = mid * kmax * np.log(kmax / mid) / (kmax - mid)
            lo, hi = (mid, hi) if m < mean_nnz else (lo, mid)
        kmin = 0.5 * (lo + hi)
        u = rng.random(n)
        k = kmin * kmax / (kmax - u * (kmax - kmin))      # inverse CDF of k^-2
        lengths = np.clip(np.rint(k).astype(np.int64), 1, kmax)
        indptr = np.zeros(n + 1, dtype=np.int64)
        np.cumsum(lengths, out=indptr[1:])
        cols = np.empty(indptr[-1], dtype=np.int64)
        for r in range(n):
            L = lengths[r]
            if L * 4 < n:
                c = np.unique(rng.integers(0, n, int(L * 1.2) + 8))
                while c.size < L:
                    c = np.unique(np.concatenate([c, rng.integers(0, n, L)]))
                c = rng.choice(c, L, replace=False)
            else:
                c = rng.choice(n, L, replace=False)
            c.sort()
            cols[indptr[r]:indptr[r + 1]] = c
        data = rng.normal(0.0, sd, cols.size)
        return sp.csr_matrix((data, cols, indptr), shape=(n, n))
    if kind == "local":
        side = int(round(np.sqrt(n)))
        n = side * side
        sigma, cutoff = 5.0, 15
        offs = [(dy, dx) for dy in range(-cutoff, cutoff + 1) for dx in range(-cutoff, cutoff + 1)
                if dy * dy + dx * dx <= cutoff * cutoff]
        offs = np.array(offs, dtype=np.int64)
        prob = np.exp(-(offs ** 2).sum(1) / (2 * sigma * sigma))
        ys, xs = np.divmod(np.arange(n), side)
        rows_l, cols_l = [], []
        for r0 in range(0, n, 8192):
            r1 = min(n, r0 + 8192)
            ty = ys[r0:r1, None] + offs[None, :, 0]
            tx = xs[r0:r1, None] + offs[None, :, 1]
            ok = (ty >= 0) & (ty < side) & (tx >= 0) & (tx < side)
            ok &= rng.random(ok.shape) < prob[None, :]
            rr, kk = np.nonzero(ok)
            rows_l.append(rr + r0)
            cols_l.append(ty[rr, kk] * side + tx[rr, kk])
        rows = np.concatenate(rows_l)
        cols = np.concatenate(cols_l)
        data = rng.normal(0.0, sd, rows.size)
        m = sp.csr_matrix((data, (rows, cols)), shape=(n, n))
        m.sort_indices()
        return m
    if kind == "blocks":
        bs = 64
        nb = (n + bs - 1) // bs
        n = nb * bs
        bmask = rng.random((nb, nb)) < 0.02
        brow, bcol = np.nonzero(bmask)
        rr = (brow[:, None] * bs + np.arange(bs)[None, :])          # (nblk, 64)
        cc = (bcol[:, None] * bs + np.arange(bs)[None, :])
        rows = np.repeat(rr, bs, axis=1).ravel()
        cols = np.tile(cc, (1, bs)).ravel()
        data = rng.normal(0.0, sd, rows.size)
        m = sp.csr_matrix((data, (rows, cols)), shape=(n, n))
        m.sort_indices()
        return m
    raise ValueError(f"unknown connectivity structure {kind!r}")


def batched_coba(n_instances: int = 256, seed: int = 42, n_min: int = 1000,
                 n_max: int = 8000, steps: int = 5000) -> list[CobaNet]:
    """Uneven-size spiking networks; excitatory increment swept 0.2-1.0 and
    inhibitory increment 2-10 over a square grid, one seed per instance."""
    side = int(np.ceil(np.sqrt(n_instances)))
    we = np.linspace(0.2, 1.0, side)
    wi = np.linspace(2.0, 10.0, side)
    size_rng = np.random.default_rng(seed)
    sizes = size_rng.integers(n_min, n_max + 1, n_instances)
    nets = []
    for i in range(n_instances):
        nets.append(coba_net(seed=seed + i, n=int(sizes[i]), w_exc=float(we[i % side]),
                             w_inh=float(wi[i // side]), steps=steps, skip=True))
    return nets


# ---------------------------------------------------------------------------
# networks built through the public API
# ---------------------------------------------------------------------------

def delay_arg(m: sp.csr_matrix, d, dt: float):
    """Connector `delays` argument for the (post, pre) matrix m: None -> no
    delay, a number -> uniform delay of that many steps, an array -> one
    delay (steps) per synapse in m's CSR order, as a sparse (pre, post)
    matrix of delays in ms."""
    if d is None:
        return 0.0
    if np.ndim(d) == 0:
        return float(d) * dt
    dm = sp.csr_matrix((np.asarray(d, dtype=np.float64) * dt, m.indices, m.indptr), shape=m.shape)
    return to_from_sparse(dm)


def build_rate_network(rn: RateNet, precision: str = "double", record: bool = True,
                       storage_format: str = "csr", delays=(None, None), **config):
    """Input population (constant r) -> leaky integrators, input and
    recurrent projections on target 'exc'; `delays` (input, recurrent) as in
    delay_arg. Returns (net, pop, monitor)."""
    from . import Network, Neuron
    net = Network(dt=rn.dt, seed=0)
    net.config(precision=precision, **config)
    inp = net.create(rn.n_in, Neuron(parameters="r = 0.0"))
    li = Neuron(parameters=dict(tau=rn.tau), equations="tau*dr/dt + r = sum(exc) : min=0.0")
    pop = net.create(rn.n_out, li)
    net.connect(inp, pop, "exc").from_sparse(to_from_sparse(rn.w_in), delay_arg(rn.w_in, delays[0], rn.dt),
                                             storage_format=storage_format)
    net.connect(pop, pop, "exc").from_sparse(to_from_sparse(rn.w_rec), delay_arg(rn.w_rec, delays[1], rn.dt),
                                             storage_format=storage_format)
    mon = net.monitor(pop, "r") if record else None
    inp.r = rn.r_in
    return net, pop, mon


def coba_neuron(params: dict):
    from . import Neuron
    return Neuron(parameters=dict(params), equations=list(COBA_EQUATIONS), spike=COBA_SPIKE,
                  reset=COBA_RESET, refractory=COBA_REFRACTORY)


def build_coba_network(cn: CobaNet, precision: str = "double", engine: str = "auto",
                       record: bool = True, stdp_w_ee: sp.csr_matrix | None = None,
                       delays=(None, None), **config):
    """The spiking net: E->all (exc) and I->all (inh); with a plastic E->E
    matrix: E->E (STDP, exc), E->I (exc), I->all (inh). `delays` (exc, inh)
    of E->all / I->all as in delay_arg. Returns (net, pop, monitor); the
    initial potentials are set after compile()."""
    from . import STDP, Network
    net = Network(dt=cn.dt, seed=0)
    net.config(precision=precision, engine=engine, **config)
    P = net.create(cn.n, coba_neuron(cn.params))
    Pe, Pi = P[: cn.n_exc], P[cn.n_exc:]
    if stdp_w_ee is None:
        net.connect(Pe, P, "exc").from_sparse(to_from_sparse(cn.w_exc),
                                              delay_arg(cn.w_exc, delays[0], cn.dt))
    else:
        net.connect(Pe, Pe, "exc", synapse=STDP(**STDP_PARAMS)).from_sparse(to_from_sparse(stdp_w_ee))
        net.connect(Pe, Pi, "exc").from_sparse(to_from_sparse(cn.w_exc[cn.n_exc:]))
    net.connect(Pi, P, "inh").from_sparse(to_from_sparse(cn.w_inh), delay_arg(cn.w_inh, delays[1], cn.dt))
    mon = net.monitor(P, "spike") if record else None
    P.v = cn.v0
    return net, P, mon


def stdp_matrix(cn: CobaNet, seed: int, p: float) -> sp.csr_matrix:
    """Plastic E->E weights U[0, 0.5] of the plastic test network."""
    rng = np.random.default_rng(seed + 1000)
    return bernoulli_csr(rng, cn.n_exc, cn.n_exc, p, lambda k: rng.uniform(0.0, 0.5, k))


# ---------------------------------------------------------------------------
# large plastic spiking network (device-generated connectivity)
# ---------------------------------------------------------------------------

def build_batch(cns: list[CobaNet], precision: str = "float", weight_dtype: str | None = None,
                record: bool = True, **kw):
    """The spiking nets of `cns` as instances of one Batch (not compiled).
    Returns (batch, [(net, pop, monitor)])."""
    from .core.batch import Batch
    members = [build_coba_network(cn, "double", "grid", record=record) for cn in cns]
    batch = Batch([m[0] for m in members], precision=precision, weight_dtype=weight_dtype, **kw)
    return batch, members


@dataclass
class LargeNet:
    """1M conductance-based LIF neurons (80 % excitatory), every neuron
    receiving 800 excitatory and 200 inhibitory synapses (1e9 in total);
    E->E is plastic (pair-based STDP, float weights), the other projections
    are static. Weights scale the 4000-neuron net's total input to the larger
    in-degree (0.6 x 64/800 and 6.7 x 16/200)."""
    n: int = 1_000_000
    fan_e: int = 800
    fan_i: int = 200
    w_exc: float = 0.048
    w_inh: float = 0.536
    drive: float = 20.0
    seed: int = 42
    steps: int = 1000
    dt: float = 0.1

    @property
    def n_exc(self) -> int:
        return int(round(self.n * 0.8))

    @property
    def nnz(self) -> int:
        return self.n * (self.fan_e + self.fan_i)


def build_large_network(ln: LargeNet, precision: str = "double", stdp: bool = True,
                        record: bool = True, connector: str = "fixed_number_pre", **config):
    """Returns (net, pop, monitor, projections); connectivity is generated on
    the device at compile(): fixed in-degrees, or (connector
    "fixed_probability") independent pairs with the same mean in-degrees."""
    from . import STDP, Network, Uniform
    net = Network(dt=ln.dt, seed=ln.seed)
    # float: Kahan compensation of v only (the conductances only decay)
    config.setdefault("compensate", "auto")
    net.config(precision=precision, engine="grid", device_connectors=True, **config)
    params = dict(COBA_PARAMS)
    params["I"] = float(ln.drive)
    P = net.create(ln.n, coba_neuron(params))
    Pe, Pi = P[: ln.n_exc], P[ln.n_exc:]
    syn = STDP(**STDP_PARAMS) if stdp else None
    if connector == "fixed_probability":
        pe, pi = ln.fan_e / ln.n_exc, ln.fan_i / (ln.n - ln.n_exc)
        ee = net.connect(Pe, Pe, "exc", synapse=syn).fixed_probability(pe, ln.w_exc)
        ei = net.connect(Pe, Pi, "exc").fixed_probability(pe, ln.w_exc)
        ie = net.connect(Pi, P, "inh").fixed_probability(pi, ln.w_inh)
    else:
        ee = net.connect(Pe, Pe, "exc", synapse=syn).fixed_number_pre(ln.fan_e, ln.w_exc)
        ei = net.connect(Pe, Pi, "exc").fixed_number_pre(ln.fan_e, ln.w_exc)
        ie = net.connect(Pi, P, "inh").fixed_number_pre(ln.fan_i, ln.w_inh)
    mon = net.monitor(P, "spike") if record else None
    P.v = np.random.default_rng(ln.seed).uniform(-60.0, -50.0, ln.n)
    return net, P, mon, (ee, ei, ie)
