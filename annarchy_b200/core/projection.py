"""Projections and connector methods.

Connectivity is kept as one CSR matrix per projection, rows = post neurons
of the projection (in ``post_ranks`` order) and columns = pre neurons, with
each row's pre ranks ascending: the order in which the reference builds its
LIL dendrites and hence the order of its CSR rows
(ANNarchy/core/ConnectorMethods.py:763-796, ANNarchy/include/CSRMatrix.hpp:142).
The storage format the kernels read (CSR, ELL, ELL-R, SELL-C-sigma, BSR,
HYB) is derived from it at compile time.

Connector methods (ANNarchy/core/ConnectorMethods.py): from_sparse,
from_matrix, fixed_probability, fixed_number_pre, fixed_number_post,
all_to_all, one_to_one. Weights may be scalars, arrays or random
distributions drawn from the network's seeded generator. Synaptic delays
follow the reference (ANNarchy/core/Projection.py:651-690, 1283-1416): a
delay in ms becomes round(delay / dt) steps; one step (or less) is the
ordinary transmission of the previous step's output; a scalar gives a
uniform delay, a random distribution or a per-synapse array a non-uniform
one. A rate-coded projection with delay d reads the pre-synaptic rates of
step t - d; a spiking one delivers the spikes of step t - d.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from .models import Synapse
from .population import Population, PopulationView
from .random import values as draw

FORMATS = ("csr", "ell", "ellr", "sell", "bsr", "hyb", "pcsr", "auto")


def _ranks(obj):
    return np.asarray(obj.ranks, dtype=np.int64)


def _population(obj):
    return obj.population if isinstance(obj, PopulationView) else obj


class Projection:
    def __init__(self, pre, post, target: str, synapse: Synapse | None = None,
                 name: str | None = None, net=None, proj_id: int = 0, disable_omp=True):
        self.pre = pre
        self.post = post
        self.pre_pop: Population = _population(pre)
        self.post_pop: Population = _population(post)
        self.target = target
        self.net = net
        self.id = proj_id
        self.name = name or f"proj{proj_id}"
        pre_type = self.pre_pop.neuron_type.type
        if synapse is None:
            synapse = Synapse(pre_spike="g_target += w") if pre_type == "spike" else Synapse()
        self.synapse_type = synapse
        self.desc = synapse.desc
        if synapse.type == "spike" and pre_type != "spike":
            raise TypeError("a spiking synapse needs a spiking pre-synaptic population")
        if synapse.type == "rate" and pre_type != "rate":
            raise TypeError("a rate-coded synapse needs a rate-coded pre-synaptic population")
        # reductions of the pre/post populations used by the synapse
        for side, pop in (("pre", self.pre_pop), ("post", self.post_pop)):
            for op in self.desc.get(side + "_global_operations", []):
                pop._add_globalop(op)
        if self.post_pop.neuron_type.type == "rate" and target not in self.post_pop.targets:
            # a rate-coded target the neuron does not sum: its weighted sum is
            # still computed (ANNarchy/core/Projection.py:105-110 adds the
            # target to the population's)
            self.post_pop._add_rate_target(target)
        if self.post_pop.neuron_type.type == "spike" and synapse.type == "spike":
            if target not in self.post_pop.targets:
                # a conductance the neuron only assigns (`g_exc = 0`) is not
                # found by the target extraction (ANNarchy/parser/
                # Extraction.py:686-702 wants a character before `g_`), or the
                # neuron does not mention it: the projection adds its target
                # to the population's, as the reference's does
                # (ANNarchy/core/Projection.py:105-110)
                self.post_pop._add_spike_target(target)
        self.pre_ranks = _ranks(pre)
        self.post_ranks_view = _ranks(post)
        self._csr: sp.csr_matrix | None = None   # (n_post_view, n_pre_view), view-relative
        self._storage_format = "csr"
        self._device_conn = None
        self._nnz = 0
        self._host_attr: dict[str, np.ndarray] = {}
        self.connector_name = None
        self._schedule = None
        self.uniform_delay = 1          # steps; -1 when the delays are per synapse
        self.max_delay = 1              # steps
        self._delay_steps = None        # per synapse (CSR order) for non-uniform delays
        self._global_values: dict[str, float] = {}   # global parameters set before compile()
        self._host_semi: dict[str, np.ndarray] = {}  # post-synaptic (per dendrite) attributes
        # learning switches on the device: plasticity, update, period, offset (steps)
        self._learn_flags = [1, 1, 1, 0]

    # -- properties -------------------------------------------------------------
    @property
    def nb_synapses(self) -> int:
        if getattr(self, "_device_conn", None):
            return int(self._nnz)
        return 0 if self._csr is None else int(self._csr.nnz)

    def __len__(self):
        return self.nb_synapses

    @property
    def size(self) -> int:
        return 0 if self._csr is None else int((np.diff(self._csr.indptr) > 0).sum())

    @property
    def plastic(self) -> bool:
        """Whether the synapses keep per-synapse state updated by events: the
        weight changes, post-spike statements, or pre-spike statements that
        do more than `g_target += w` (short-term plasticity's x and u, a
        transmission scaled by a synaptic variable)."""
        d = self.desc
        if d.get("plasticity") or d.get("post_spike"):
            return True
        if any(v.get("cpp") and v.get("method") != "event-driven" for v in d["variables"]):
            return True                 # synaptic variables updated every step
        for v in d.get("pre_spike", []):
            if v["name"] != "g_target" or v["eq"].replace(" ", "") != "g_target+=w":
                return True
        return False

    @property
    def storage_format(self) -> str:
        return self._storage_format

    def _rng(self):
        return self.net._rng if self.net is not None else np.random.default_rng()

    # -- connectors ---------------------------------------------------------------
    def _dt(self) -> float:
        return self.net.dt if self.net is not None else 1.0

    def _steps(self, ms) -> np.ndarray:
        # Python's round(), as the reference uses; at least one step
        return np.maximum(1, np.array([round(float(v) / self._dt()) for v in np.ravel(ms)],
                                      dtype=np.int64)).astype(np.int32)

    def _set_delays(self, delays, m: sp.csr_matrix, delay_matrix=None):
        """delays: ms as a scalar (uniform), a RandomDistribution (one draw
        per synapse, bounded below by dt) or None; delay_matrix: per-synapse
        delays in ms with the structure of `m` (rows post, columns pre)."""
        from .random import RandomDistribution
        if delay_matrix is not None:
            rows = np.repeat(np.arange(m.shape[0]), np.diff(m.indptr))
            vals = np.asarray(delay_matrix[rows, m.indices]).ravel()
            steps = self._steps(vals)
        elif isinstance(delays, RandomDistribution):
            if getattr(delays, "max", None) is None:
                raise ValueError("a random distribution of delays needs a max value")
            vals = np.maximum(draw(delays, (m.nnz,), self._rng()), self._dt())
            steps = self._steps(vals)
            # history for the distribution's whole range (Projection.py:667)
            dist_max = int(round(float(delays.max) / self._dt()))
        else:
            d = 0.0 if delays is None else float(delays)
            self.uniform_delay = max(1, int(round(d / self._dt())))
            self.max_delay = self.uniform_delay
            self._delay_steps = None
            return
        if self.plastic and self.synapse_type.type == "spike":
            raise NotImplementedError("non-uniform delays of plastic spiking projections "
                                      "are not supported by this backend")
        if steps.size and int(steps.max()) > 63:
            raise NotImplementedError("per-synapse delays are limited to 63 steps by this backend")
        self.uniform_delay = -1
        self._delay_steps = steps
        self.max_delay = max(int(steps.max()) if steps.size else 1,
                             dist_max if delay_matrix is None else 1)

    def _store(self, m: sp.csr_matrix, name, storage_format, delays=0.0, delay_matrix=None):
        m = sp.csr_matrix(m)
        m.sum_duplicates()
        m.sort_indices()
        self._csr = m
        self._set_delays(delays, m, delay_matrix)
        self.connector_name = name
        if storage_format is not None:
            if storage_format not in FORMATS:
                raise ValueError(f"unknown storage format {storage_format!r}")
            self._storage_format = storage_format
        n_dend = int(np.count_nonzero(np.diff(m.indptr)))
        params = {q["name"]: q for q in self.desc["parameters"]}
        # parameters first: a variable may take its initial value from one
        for v in self.desc["parameters"] + self.desc["variables"]:
            init = v["init"]
            if isinstance(init, str):
                src = params.get(init)
                if src is None:
                    raise ValueError(f"init value {init!r} of {v['name']} is not a parameter")
                init = self._host_attr.get(init, self._host_semi.get(init, src["init"]))
            if v["locality"] == "local" and v["name"] != "w":
                self._host_attr[v["name"]] = np.broadcast_to(
                    np.asarray(init, dtype=np.float64), (m.nnz,)).copy()
            elif v["locality"] == "semiglobal":
                self._host_semi[v["name"]] = np.broadcast_to(
                    np.asarray(init, dtype=np.float64), (n_dend,)).copy()
        return self

    def from_function(self, method, storage_format=None, storage_order=None, **args):
        """Connectivity returned by a user function method(pre, post, dt,
        **args) as a LILConnectivity (ANNarchy/core/ConnectorMethods.py:
        456-530)."""
        syn = method(self.pre, self.post, self._dt(), **args)
        if not isinstance(syn, LILConnectivity):
            raise TypeError("the connection method must return a LILConnectivity")
        syn.validate()
        delays = ([[syn.uniform_delay]] * len(syn.post_rank) if syn.uniform_delay != -1
                  else syn.delay)
        self._from_lil(syn.post_rank, syn.pre_rank, syn.w, delays, syn.requires_sorting)
        self.connector_name = "User-defined"
        if storage_format is not None:
            if storage_format not in FORMATS:
                raise ValueError(f"unknown storage format {storage_format!r}")
            self._storage_format = storage_format
        return self

    connect_with_func = from_function

    def _weights(self, weights, nnz):
        return draw(weights, (nnz,), self._rng())

    def from_sparse(self, weights, delays=0.0, storage_format=None, storage_order=None):
        """weights: scipy sparse matrix of shape (pre, post); delays: ms, a
        scalar or a sparse matrix of the same shape."""
        w = sp.csr_matrix(weights)
        if w.shape != (len(self.pre_ranks), len(self.post_ranks_view)):
            raise ValueError(f"from_sparse(): expected shape {(len(self.pre_ranks), len(self.post_ranks_view))}, "
                             f"got {w.shape}")
        if sp.issparse(delays):
            return self._store(w.T.tocsr(), "Sparse connectivity matrix", storage_format, None,
                               sp.csr_matrix(delays).T.tocsr())
        return self._store(w.T.tocsr(), "Sparse connectivity matrix", storage_format, delays)

    connect_from_sparse = from_sparse

    def _from_lil(self, post_ranks, pre_ranks, w, delays, requires_sorting: bool = False):
        """Connectivity as the reference's generated module receives it
        (init_from_lil, ANNarchy/generator/NanoBind/Projection.py:20-60;
        built by ANNarchy/cython_ext/Connector.pyx:93-170): post population
        ranks, per post the pre population ranks, weights (one value or one
        per synapse) and delays in steps (one or one per synapse). Rows may
        come unsorted when requires_sorting; pre ranks are sorted per row
        with their weights and delays."""
        post_ranks = [int(r) for r in post_ranks]
        if len(pre_ranks) != len(post_ranks) or len(w) != len(post_ranks):
            raise ValueError("init_from_lil: post_ranks, pre_ranks and w differ in length")
        if requires_sorting:
            order = sorted(range(len(post_ranks)), key=lambda i: post_ranks[i])
        else:
            order = range(len(post_ranks))
        post_pos = {int(r): i for i, r in enumerate(self.post_ranks_view)}
        pre_pos = {int(r): i for i, r in enumerate(self.pre_ranks)}
        rows, cols, vals, dsteps = [], [], [], []
        for i in order:
            pr = np.asarray(pre_ranks[i], dtype=np.int64)
            if post_ranks[i] not in post_pos:
                raise ValueError(f"init_from_lil: post rank {post_ranks[i]} is not in the projection")
            ww = np.asarray(w[i], dtype=np.float64)
            ww = np.full(pr.size, float(ww.reshape(-1)[0])) if ww.size == 1 else ww
            dd = np.asarray(delays[i] if delays is not None and len(delays) > i else [0],
                            dtype=np.int64)
            dd = np.full(pr.size, int(dd.reshape(-1)[0]) if dd.size else 0) if dd.size <= 1 else dd
            if ww.size != pr.size or dd.size != pr.size:
                raise ValueError(f"init_from_lil: row {i} has {pr.size} ranks, {ww.size} weights "
                                 f"and {dd.size} delays")
            try:
                c = np.fromiter((pre_pos[int(r)] for r in pr), dtype=np.int64, count=pr.size)
            except KeyError as e:
                raise ValueError(f"init_from_lil: pre rank {e.args[0]} is not in the projection")
            rows.append(np.full(pr.size, post_pos[post_ranks[i]], dtype=np.int64))
            cols.append(c)
            vals.append(ww)
            dsteps.append(dd)
        cat = (lambda a, dt: np.concatenate(a) if a else np.zeros(0, dt))
        rows, cols = cat(rows, np.int64), cat(cols, np.int64)
        vals, dsteps = cat(vals, np.float64), cat(dsteps, np.int64)
        shape = (len(self.post_ranks_view), len(self.pre_ranks))
        m = sp.csr_matrix((vals, (rows, cols)), shape=shape)
        if dsteps.size and np.unique(dsteps).size > 1:
            dm = sp.csr_matrix((dsteps * self._dt(), (rows, cols)), shape=shape)
            return self._store(m, "From LIL", None, None, dm)
        d = float(dsteps[0]) * self._dt() if dsteps.size else 0.0
        return self._store(m, "From LIL", None, d)

    def from_matrix(self, weights, delays=0.0, pre_post=False, storage_format=None,
                    storage_order=None):
        """weights: dense (post, pre) array (or (pre, post) with pre_post=True);
        entries that are None/NaN mean no synapse."""
        W = np.array(weights, dtype=object if np.asarray(weights).dtype == object else np.float64)
        if pre_post:
            W = W.T
        if W.dtype == object:
            mask = np.vectorize(lambda x: x is not None)(W)
            W = np.where(mask, W, 0.0).astype(np.float64)
        else:
            mask = ~np.isnan(W)
            W = np.nan_to_num(W)
        rows, cols = np.nonzero(mask)
        m = sp.csr_matrix((W[rows, cols], (rows, cols)), shape=W.shape)
        if np.ndim(delays) == 2:
            D = np.asarray(delays, dtype=np.float64)
            return self._store(m, "Connectivity matrix", storage_format, None, D.T if pre_post else D)
        return self._store(m, "Connectivity matrix", storage_format, delays)

    def _drops_self(self, allow_self_connections: bool) -> bool:
        """Whether a random connector leaves out the pairs with pre rank ==
        post rank. The reference allows them as soon as pre and post are
        different objects (ANNarchy/core/ConnectorMethods.py:283-284,
        344-345, 410-411 compare the objects, not their populations): a view
        connected to its own population keeps its self-synapses, and so do
        two views of the same neurons made separately. all_to_all alone
        compares the populations (ConnectorMethods.py:105-112)."""
        return not allow_self_connections and self.pre is self.post

    def _self_mask(self, rows, cols):
        if self.pre_pop is not self.post_pop:
            return np.ones(rows.shape, dtype=bool)
        return self.post_ranks_view[rows] != self.pre_ranks[cols]

    def all_to_all(self, weights, delays=0.0, allow_self_connections=False,
                   force_multiple_weights=False, storage_format=None, storage_order=None):
        npost, npre = len(self.post_ranks_view), len(self.pre_ranks)
        rows = np.repeat(np.arange(npost), npre)
        cols = np.tile(np.arange(npre), npost)
        if not allow_self_connections:
            keep = self._self_mask(rows, cols)
            rows, cols = rows[keep], cols[keep]
        w = self._weights(weights, rows.size)
        m = sp.csr_matrix((w, (rows, cols)), shape=(npost, npre))
        return self._store(m, "All-to-All", storage_format, delays)

    def one_to_one(self, weights=1.0, delays=0.0, force_multiple_weights=False,
                   storage_format=None, storage_order=None):
        n = min(len(self.post_ranks_view), len(self.pre_ranks))
        rows = np.arange(n)
        w = self._weights(weights, n)
        m = sp.csr_matrix((w, (rows, rows)), shape=(len(self.post_ranks_view), len(self.pre_ranks)))
        return self._store(m, "One-to-One", storage_format, delays)

    # -- distance-based patterns ------------------------------------------------
    @staticmethod
    def _pattern_coords(geometry) -> np.ndarray:
        """(size, dim) normalized coordinates of every rank as the reference's
        pattern connectors compute them (ANNarchy/cython_ext/Connector.pyx:
        464-489 with Coordinates.pyx:122-199): 1-D rank / (size - 1) in
        double; 2-D and 3-D row-major indices / (extent - 1) rounded to
        float32 (0 along an extent of 1); more dimensions in double."""
        geometry = tuple(int(g) for g in np.atleast_1d(geometry))
        size = int(np.prod(geometry))
        ranks = np.arange(size)
        if len(geometry) == 1:
            if size < 2:
                raise ValueError("distance-based patterns need more than one neuron along a 1-D "
                                 "geometry")
            return (ranks / float(size - 1))[:, None]
        idx = np.stack(np.unravel_index(ranks, geometry), axis=1).astype(np.float64)
        if len(geometry) > 3:
            if min(geometry) < 2:
                raise ValueError("distance-based patterns need extents above 1 beyond 3-D")
            return idx / (np.asarray(geometry, dtype=np.float64) - 1.0)
        den = np.asarray([g - 1.0 if g > 1 else 1.0 for g in geometry])
        out = (idx / den).astype(np.float32).astype(np.float64)
        out[:, np.asarray(geometry) <= 1] = 0.0
        return out

    def _pattern(self, kind: str, weight_of, limit_of, delays, allow_self_connections,
                 storage_format, name):
        """Rows of a distance-based pattern: every (post, pre) pair whose
        float32 value passes the limit, pre ranks ascending. The squared
        distance accumulates in float32 over the pre population's
        dimensions, each term in double (Coordinates.pyx:10-48)."""
        from .population import PopulationView
        if isinstance(self.pre, PopulationView) or isinstance(self.post, PopulationView):
            raise ValueError(f"{kind} connector is only possible on whole populations, "
                             "not PopulationViews")
        if self.pre_pop is not self.post_pop:
            allow_self_connections = True
        pre_c = self._pattern_coords(self.pre_pop.geometry)
        post_c = self._pattern_coords(self.post_pop.geometry)
        dim = pre_c.shape[1]
        if post_c.shape[1] < dim:
            raise ValueError(f"{kind} connector: the post-synaptic geometry has fewer dimensions "
                             "than the pre-synaptic one")
        npost, npre = post_c.shape[0], pre_c.shape[0]
        if self._device_ok(npost * npre // 10):
            # generated on the device at compile() (anb_connect_distance_pattern)
            self._device_delays(delays)
            self._device_conn = dict(kind="pattern", pattern=kind, post_c=post_c, pre_c=pre_c,
                                     exclude_self=not allow_self_connections, name=name,
                                     storage_format=storage_format, delays=delays,
                                     **self._pattern_params)
            self._nnz = 0                                  # known after compile()
            self.connector_name = name + " (device)"
            if storage_format is not None:
                self._storage_format = storage_format
            return self
        rows_l, cols_l, w_l = [], [], []
        block = max(1, 4_000_000 // max(npre, 1))
        for r0 in range(0, npost, block):
            r1 = min(npost, r0 + block)
            if dim == 1:
                d = ((pre_c[None, :, 0] - post_c[r0:r1, None, 0]) ** 2).astype(np.float32)
            else:
                d = np.zeros((r1 - r0, npre), dtype=np.float32)
                for k in range(dim):
                    term = (pre_c[None, :, k] - post_c[r0:r1, None, k]) ** 2
                    d = (d.astype(np.float64) + term).astype(np.float32)
            value = weight_of(d.astype(np.float64)).astype(np.float32)
            keep = limit_of(value.astype(np.float64))
            if not allow_self_connections:           # the same population: pre rank == post rank
                rr = np.arange(r0, min(r1, npre))
                keep[rr - r0, rr] = False
            rows, cols = np.nonzero(keep)
            rows_l.append(rows + r0)
            cols_l.append(cols)
            w_l.append(value[rows, cols].astype(np.float64))
        rows = np.concatenate(rows_l)
        cols = np.concatenate(cols_l)
        m = sp.csr_matrix((np.concatenate(w_l), (rows, cols)), shape=(npost, npre))
        return self._store(m, name, storage_format, delays)

    def gaussian(self, amp, sigma, delays=0.0, limit=0.01, allow_self_connections=False,
                 storage_format=None):
        """Gaussian pattern (ANNarchy/core/ConnectorMethods.py:144-198,
        cython_ext/Connector.pyx:433-502): post neuron i receives pre neuron
        j with weight amp * exp(-d2 / (2 sigma^2)), d2 the squared distance of
        their normalized coordinates, when that weight exceeds limit * amp;
        amp and sigma in float32, the weight rounded to float32."""
        a32, s32 = np.float32(amp), np.float32(sigma)
        den = 2.0 * float(np.float32(s32 * s32))
        a = float(a32)
        self._pattern_params = dict(pkind=0, a_pos=a, den_pos=den, a_neg=0.0, den_neg=1.0,
                                    threshold=float(limit) * a)
        return self._pattern("Gaussian", lambda d: a * np.exp(-d / den),
                             lambda v: v > float(limit) * a, delays, allow_self_connections,
                             storage_format, "Gaussian")

    connect_gaussian = gaussian

    def dog(self, amp_pos, sigma_pos, amp_neg, sigma_neg, delays=0.0, limit=0.01,
            allow_self_connections=False, storage_format=None):
        """Difference-of-Gaussians pattern (ANNarchy/core/ConnectorMethods.py:
        201-260, cython_ext/Connector.pyx:504-575): weight amp_pos *
        exp(-d2 / (2 sigma_pos^2)) - amp_neg * exp(-d2 / (2 sigma_neg^2)),
        kept when |weight| exceeds limit * |amp_pos - amp_neg| (the
        difference taken in float32)."""
        ap, an = float(np.float32(amp_pos)), float(np.float32(amp_neg))
        sp_, sn = np.float32(sigma_pos), np.float32(sigma_neg)
        dp, dn = 2.0 * float(np.float32(sp_ * sp_)), 2.0 * float(np.float32(sn * sn))
        span = abs(float(np.float32(np.float32(amp_pos) - np.float32(amp_neg))))
        self._pattern_params = dict(pkind=1, a_pos=ap, den_pos=dp, a_neg=an, den_neg=dn,
                                    threshold=float(limit) * span)
        return self._pattern("DoG", lambda d: ap * np.exp(-d / dp) - an * np.exp(-d / dn),
                             lambda v: np.abs(v) > float(limit) * span, delays,
                             allow_self_connections, storage_format, "Difference-of-Gaussian")

    connect_dog = dog

    def fixed_probability(self, probability, weights, delays=0.0, allow_self_connections=False,
                          force_multiple_weights=False, storage_format=None, storage_order=None):
        """Each (post, pre) pair is connected independently with the given
        probability (per-post Bernoulli masks, as in the reference's
        ANNarchy/cython_ext/Connector.pyx:306-345). Large projections (more
        than 2e7 expected synapses, or device_connectors=True) are generated
        on the device at compile() by geometric skipping
        (anb_connect_fixed_probability_rows)."""
        rng = self._rng()
        npost, npre = len(self.post_ranks_view), len(self.pre_ranks)
        if 0.0 < probability <= 1.0 and self._device_ok(int(npost * npre * probability)):
            self._device_conn = dict(kind="fixed_probability", probability=float(probability),
                                     **self._device_weights(weights, delays),
                                     seed=int(rng.integers(0, 2**63 - 1)),
                                     exclude_self=self._drops_self(allow_self_connections))
            self._nnz = int(round(npost * npre * probability))        # until compile()
            self.connector_name = "Random (device)"
            if storage_format is not None:
                self._storage_format = storage_format
            return self
        rows_l, cols_l = [], []
        for r0 in range(0, npost, 4096):
            r1 = min(npost, r0 + 4096)
            mask = rng.random((r1 - r0, npre)) < probability
            rr, cc = np.nonzero(mask)
            rows_l.append(rr + r0)
            cols_l.append(cc)
        rows = np.concatenate(rows_l) if rows_l else np.zeros(0, np.int64)
        cols = np.concatenate(cols_l) if cols_l else np.zeros(0, np.int64)
        if self._drops_self(allow_self_connections):
            keep = self._self_mask(rows, cols)
            rows, cols = rows[keep], cols[keep]
        w = self._weights(weights, rows.size)
        m = sp.csr_matrix((w, (rows, cols)), shape=(npost, npre))
        return self._store(m, "Random", storage_format, delays)

    def _device_ok(self, nnz: int) -> bool:
        mode = self.net._config.get("device_connectors", "auto") if self.net is not None else False
        contiguous = (np.all(np.diff(self.pre_ranks) == 1) and np.all(np.diff(self.post_ranks_view) == 1))
        if mode is True or mode == "always":
            if not contiguous:
                raise NotImplementedError("device connectors need contiguous pre and post ranks")
            return True
        return mode == "auto" and nnz > 20_000_000 and contiguous

    def _device_delays(self, delays):
        """Device connectors take no synaptic delays (one step at most)."""
        if not (np.ndim(delays) == 0 and not hasattr(delays, "get_values")
                and round(float(delays or 0.0) / self._dt()) <= 1):
            raise NotImplementedError("device connectors take no synaptic delays")

    def _device_weights(self, weights, delays) -> dict:
        """Weight law of a device connector: constant (wkind 0), Uniform (1)
        or unbounded Normal (2); no synaptic delays."""
        from .random import Normal, Uniform
        if np.ndim(weights) == 0 and not hasattr(weights, "get_values"):
            wk, a, b = 0, float(weights), 0.0
        elif isinstance(weights, Uniform):
            wk, a, b = 1, weights.min, weights.max
        elif isinstance(weights, Normal) and weights.min is None and weights.max is None:
            wk, a, b = 2, weights.mu, weights.sigma
        else:
            raise NotImplementedError("device connectors take constant, Uniform or Normal weights")
        if not (np.ndim(delays) == 0 and not hasattr(delays, "get_values")
                and round(float(delays or 0.0) / self._dt()) <= 1):
            raise NotImplementedError("device connectors take no synaptic delays")
        return dict(wkind=wk, a=a, b=b)

    def fixed_number_pre(self, number, weights, delays=0.0, allow_self_connections=False,
                         force_multiple_weights=False, storage_format=None, storage_order=None):
        """Every post neuron receives exactly `number` distinct pre neurons.

        Large projections (more than 2e7 synapses, or device_connectors=True)
        are generated on the device at compile(): one pre neuron per equal
        stratum of the pre range (anb_connect_fixed_number_pre)."""
        rng = self._rng()
        npost, npre = len(self.post_ranks_view), len(self.pre_ranks)
        if self._device_ok(npost * int(number)):
            self._device_conn = dict(kind="fixed_number_pre", number=int(number),
                                     **self._device_weights(weights, delays),
                                     seed=int(rng.integers(0, 2**63 - 1)),
                                     exclude_self=self._drops_self(allow_self_connections))
            self._nnz = npost * int(number)
            self.connector_name = "Random Convergent (device)"
            if storage_format is not None:
                self._storage_format = storage_format
            return self
        drop_self = self._drops_self(allow_self_connections)
        avail = npre - (1 if drop_self else 0)
        if number > avail:
            raise ValueError("fixed_number_pre: number exceeds the available pre-synaptic neurons")
        cols = np.empty((npost, number), dtype=np.int64)
        for r0 in range(0, npost, 2048):
            r1 = min(npost, r0 + 2048)
            keys = rng.random((r1 - r0, npre), dtype=np.float32)
            if drop_self:
                pos = {int(r): k for k, r in enumerate(self.pre_ranks)}
                for i in range(r0, r1):
                    k = pos.get(int(self.post_ranks_view[i]))
                    if k is not None:
                        keys[i - r0, k] = 2.0
            cols[r0:r1] = np.argpartition(keys, number - 1, axis=1)[:, :number]
        cols.sort(axis=1)
        indptr = np.arange(0, npost * number + 1, number, dtype=np.int64)
        w = self._weights(weights, npost * number)
        m = sp.csr_matrix((w, cols.ravel(), indptr), shape=(npost, npre))
        return self._store(m, "Random Convergent", storage_format, delays)

    def fixed_number_post(self, number, weights, delays=0.0, allow_self_connections=False,
                          force_multiple_weights=False, storage_format=None, storage_order=None):
        """Every pre neuron projects onto exactly `number` distinct post neurons."""
        rng = self._rng()
        npost, npre = len(self.post_ranks_view), len(self.pre_ranks)
        keys = rng.random((npre, npost))
        if self._drops_self(allow_self_connections):
            for c in range(npre):
                hit = np.nonzero(self.post_ranks_view == self.pre_ranks[c])[0]
                keys[c, hit] = 2.0
        posts = np.argpartition(keys, number - 1, axis=1)[:, :number]
        cols = np.repeat(np.arange(npre), number)
        rows = posts.ravel()
        w = self._weights(weights, rows.size)
        m = sp.csr_matrix((w, (rows, cols)), shape=(npost, npre))
        return self._store(m, "Random Divergent", storage_format, delays)

    # -- compiled connectivity (population ranks) ------------------------------------------
    def csr_population_ranks(self):
        """(post_ranks, row_ptr, pre_rank_per_synapse, w) with rows that have
        at least one synapse, like the reference's post_rank list."""
        m = self._csr
        lengths = np.diff(m.indptr)
        rows = np.nonzero(lengths > 0)[0]
        post_ranks = self.post_ranks_view[rows].astype(np.int32)
        row_ptr = np.zeros(rows.size + 1, dtype=np.int64)
        np.cumsum(lengths[rows], out=row_ptr[1:])
        cols = self.pre_ranks[m.indices].astype(np.int32)
        return post_ranks, row_ptr, cols, np.asarray(m.data, dtype=np.float64)

    # -- learning switches (ANNarchy/core/Projection.py:1440-1509) ----------------------
    def _write_flags(self):
        if self.net is not None and self.net._compiled:
            nat = self.net._backend.native
            if f"proj{self.id}__flags" in nat.arrays:
                nat.write(f"proj{self.id}__flags", np.array(self._learn_flags, dtype=np.int32))

    @property
    def plasticity(self) -> bool:
        """Whether the weights change (the other synaptic variables still update)."""
        return bool(self._learn_flags[0])

    @plasticity.setter
    def plasticity(self, value: bool):
        self._learn_flags[0] = 1 if value else 0
        self._write_flags()

    @property
    def update(self) -> bool:
        """Whether the continuous synaptic equations run."""
        return bool(self._learn_flags[1])

    @update.setter
    def update(self, value: bool):
        self._learn_flags[1] = 1 if value else 0
        self._write_flags()

    def enable_learning(self, period: float | None = None, offset: float | None = None):
        """Learning on: the synaptic equations run every `period` ms (default
        every step), at the steps t with (t - offset) % period == 0,
        integrating over the period; weights change again."""
        if period is not None and offset is not None and offset >= period:
            raise ValueError("enable_learning(): the offset must be smaller than the period")
        if period is None and offset is not None:
            raise ValueError("enable_learning(): if you define an offset, you have to define a "
                             "period")
        dt = self._dt()
        steps = int(period / dt) if period is not None else 1
        if period is None:
            period = dt
        if offset is not None:
            # the reference takes the time of its default network
            # (Global.get_time(), Projection.py:1481), which networks created
            # with Network() never advance: the offset counts from step 0
            rel = 0.0 % period + offset
            off = int(int(rel % period) / dt)
        else:
            off = 0
        self._learn_flags = [1, 1, max(1, steps), off]
        self._write_flags()

    def disable_learning(self, update=None):
        """Rate-coded: the synaptic equations stop (weights included);
        spiking: the weights stop changing, the other variables still
        update."""
        if self.synapse_type.type == "rate":
            self._learn_flags[1] = 0
        else:
            self._learn_flags[0] = 0
        self._write_flags()

    # -- attributes --------------------------------------------------------------------------
    def _attr_names(self):
        return ["w"] + list(self._host_attr)

    def get(self, name: str, flat: bool = False):
        if name in self._host_semi:                 # one value per dendrite
            if self.net is not None and self.net._compiled:
                return self.net._backend.read_projection_attribute(self, name)
            return self._host_semi[name].copy()
        glob = {p["name"]: p for p in self.desc["parameters"] + self.desc["variables"]
                if p["locality"] == "global"}
        if name not in self._attr_names() and name not in glob and \
                name not in {p["name"] for p in self.desc["parameters"]}:
            raise AttributeError(f"projection {self.name!r} has no attribute {name!r}")
        if name in glob:
            if self.net is not None and self.net._compiled:
                return float(self.net._backend.read_projection_attribute(self, name)[0])
            return float(self._global_values.get(name, glob[name]["init"]))
        if self.net is not None and self.net._compiled:
            flat_v = self.net._backend.read_projection_attribute(self, name)
        elif name == "w":
            flat_v = np.asarray(self._csr.data, dtype=np.float64).copy()
        else:
            flat_v = self._host_attr[name].copy()
        if flat:
            return flat_v
        if getattr(self, "_device_conn", None):
            lengths = getattr(self, "_device_lengths", None)
            if lengths is None:
                return np.split(flat_v, len(self.post_ranks_view))
            return np.split(flat_v, np.cumsum(lengths)[:-1])
        lengths = np.diff(self._csr.indptr)
        lengths = lengths[lengths > 0]
        return [a for a in np.split(flat_v, np.cumsum(lengths)[:-1])]

    def set(self, values: dict):
        glob = {p["name"] for p in self.desc["parameters"] + self.desc["variables"]
                if p["locality"] == "global"}
        for name, value in values.items():
            if name in glob:
                value = float(np.asarray(value).reshape(-1)[0])
                if self.net is not None and self.net._compiled:
                    self.net._backend.write_projection_attribute(self, name, np.array([value]))
                else:
                    self._global_values[name] = value
                continue
            if name in self._host_semi:
                arr = draw(value, self._host_semi[name].shape, self._rng())
                self._host_semi[name] = np.asarray(arr, dtype=np.float64)
                if self.net is not None and self.net._compiled:
                    self.net._backend.write_projection_attribute(self, name, self._host_semi[name])
                continue
            nnz = self.nb_synapses
            if isinstance(value, list):
                value = np.concatenate([np.atleast_1d(np.asarray(v, dtype=np.float64)) for v in value])
            arr = draw(value, (nnz,), self._rng())
            if name == "w":
                self._csr.data[:] = arr
            elif name in self._host_attr:
                self._host_attr[name] = arr
            else:
                raise AttributeError(f"projection {self.name!r} has no attribute {name!r}")
            if self.net is not None and self.net._compiled:
                self.net._backend.write_projection_attribute(self, name, arr)

    def __getattr__(self, name):
        if name.startswith("_") or name in ("pre", "post", "desc", "net", "synapse_type"):
            raise AttributeError(name)
        desc = self.__dict__.get("desc")
        if desc is not None and (name == "w" or name in self.__dict__.get("_host_attr", {}) or
                                 name in self.__dict__.get("_host_semi", {}) or
                                 name in {p["name"] for p in desc["parameters"] + desc["variables"]
                                          if p["locality"] == "global"}):
            return self.get(name)
        if desc is not None:
            from .population import _model_function
            fn = _model_function(desc, name)
            if fn is not None:
                return fn
        raise AttributeError(name)

    def __setattr__(self, name, value):
        desc = self.__dict__.get("desc")
        if desc is not None and (self.__dict__.get("_csr") is not None or
                                 self.__dict__.get("_device_conn")) and (
                name == "w" or name in self.__dict__.get("_host_attr", {}) or
                name in self.__dict__.get("_host_semi", {}) or
                name in {p["name"] for p in desc["parameters"] + desc["variables"]
                         if p["locality"] == "global"}):
            self.set({name: value})
            return
        object.__setattr__(self, name, value)

    # -- delays (ANNarchy/core/Projection.py:1283-1416) ------------------------------------
    @property
    def delay(self):
        """Uniform delay in ms, or per dendrite the delays (ms) of its synapses."""
        dt = self._dt()
        if self._delay_steps is None:
            return float(self.uniform_delay * dt)
        steps = self._delay_steps
        if self.net is not None and self.net._compiled:
            steps = self.net._backend.read_delays(self)
        return [[float(x) * dt for x in a] for a in np.split(steps, np.cumsum(self.dendrite_sizes())[:-1])]

    @delay.setter
    def delay(self, value):
        compiled = self.net is not None and self.net._compiled
        cap = self.net._backend.delay_capacity(self) if compiled else None
        if self._delay_steps is None:
            if np.ndim(value) > 0:
                raise ValueError("the projection was created with a uniform delay; "
                                 "non-uniform values cannot be loaded")
            d = int(self._steps([value])[0])
            if cap is not None and d > cap:
                raise ValueError(f"delay of {d} steps exceeds the {cap} steps of history kept since "
                                 f"compile(); give the largest delay before compile()")
            self.uniform_delay = d
            self.max_delay = max(self.max_delay, d) if not compiled else self.max_delay
            if compiled and self.max_delay > 1:      # without history the delay stays one step
                self.net._backend.write_delays(self, np.array([d], dtype=np.int32))
            return
        if not isinstance(value, (list, np.ndarray)):
            raise ValueError("non-uniform delays are set as one list of delays per dendrite")
        sizes = self.dendrite_sizes()
        if len(value) != sizes.size or any(len(v) != n for v, n in zip(value, sizes)):
            raise ValueError("the delays must match the synapses of every dendrite")
        steps = self._steps(np.concatenate([np.ravel(np.asarray(v, dtype=np.float64)) for v in value]))
        if int(steps.max()) > 63:
            raise ValueError("per-synapse delays are limited to 63 steps by this backend")
        if cap is not None and int(steps.max()) > cap:
            raise ValueError(f"delay of {int(steps.max())} steps exceeds the {cap} steps of history "
                             f"kept since compile(); give the largest delay before compile()")
        self._delay_steps = steps
        if not compiled:
            self.max_delay = int(steps.max())
        else:
            self.net._backend.write_delays(self, steps)

    # -- save / load (ANNarchy/core/Projection.py:1731-1950) ---------------------------
    def save(self, filename: str):
        """Connectivity, delays and synaptic attributes into a file (.npz,
        .gz, .mat or pickle), in the reference's layout."""
        from .io import projection_data, save_data
        save_data(filename, projection_data(self))

    def load(self, filename: str, pickle_encoding: str | None = None):
        """Before compile(): connectivity, weights and delays from a file
        saved by save() (or by the reference); after compile(): attributes
        and delays of the same connectivity."""
        from .io import load_data, load_projection_data
        load_projection_data(self, load_data(filename, pickle_encoding))
        return self

    def dendrite_sizes(self):
        if getattr(self, "_device_conn", None):
            lengths = getattr(self, "_device_lengths", None)
            return np.asarray(lengths if lengths is not None else [], dtype=np.int64)
        lengths = np.diff(self._csr.indptr)
        return lengths[lengths > 0]

    # -- dendrites and matrices (ANNarchy/core/Projection.py:841-1016, 1515-1730) --------
    def nb_synapses_per_dendrite(self) -> list:
        """Synapses of every dendrite (post neuron with synapses)."""
        return [int(x) for x in self.dendrite_sizes()]

    def _pre_ranks_of(self) -> list:
        """Pre-synaptic ranks of every dendrite."""
        m = self._csr
        rows = np.nonzero(np.diff(m.indptr) > 0)[0]
        return [self.pre_ranks[m.indices[m.indptr[r]:m.indptr[r + 1]]].tolist() for r in rows]

    @property
    def dendrites(self):
        """The dendrites in ascending post rank (an iterator, a property as in
        ANNarchy/core/Projection.py:954-970)."""
        return (Dendrite(self, n, idx) for idx, n in enumerate(self.post_ranks))

    def __iter__(self):
        return self.dendrites

    def dendrite(self, post):
        """The dendrite of a post-synaptic neuron (rank or coordinates)."""
        rank = int(post) if np.ndim(post) == 0 else self.post_pop.rank_from_coordinates(post)
        ranks = self.post_ranks
        if rank not in ranks:
            raise ValueError(f"the neuron of rank {rank} has no dendrite in this projection")
        return Dendrite(self, rank, ranks.index(rank))

    def __getitem__(self, *args):
        return self.dendrite(args[0] if len(args) == 1 else args)

    def synapse(self, pre: int, post: int):
        """The synapse between two neurons (an IndividualSynapse), or None."""
        if np.ndim(pre) != 0 or np.ndim(post) != 0:
            raise ValueError("Projection.synapse() only accepts ranks for the pre and post neurons")
        return self.dendrite(post).synapse(pre)

    def connectivity_matrix(self, fill: float = 0.0) -> np.ndarray:
        """Dense (post, pre) matrix of the weights over the whole populations,
        `fill` where there is no synapse."""
        res = np.ones((self.post_pop.size, self.pre_pop.size)) * fill
        w = self.get("w")
        for idx, (rank, pre) in enumerate(zip(self.post_ranks, self._pre_ranks_of())):
            res[rank, pre] = w[idx]
        return res

    def receptive_fields(self, variable: str = "w", in_post_geometry: bool = True) -> np.ndarray:
        """All receptive fields of a projection between 2-D populations, tiled
        in the post-synaptic geometry (or a square grid), with a zero first
        row as the reference builds it."""
        import math
        if in_post_geometry:
            x_size, y_size = self.post_pop.geometry[1], self.post_pop.geometry[0]
        else:
            x_size = int(math.floor(math.sqrt(self.post_pop.size)))
            y_size = int(math.ceil(math.sqrt(self.post_pop.size)))
        ranks = self.post_ranks
        pre = self._pre_ranks_of()
        vals = self.get(variable)
        geo = self.pre_pop.geometry

        def rf(post_rank):
            if post_rank not in ranks:
                return np.zeros(geo)
            i = ranks.index(post_rank)
            res = np.zeros(self.pre_pop.size)
            if len(res) == len(pre[i]):
                res[pre[i]] = vals[i]
            return res.reshape(geo)

        res = np.zeros((1, x_size * geo[1]))
        for y in range(y_size):
            row = np.concatenate([rf(self.post_pop.rank_from_coordinates((y, x))) for x in range(x_size)],
                                 axis=1)
            res = np.concatenate((res, row))
        return res

    def save_connectivity(self, filename: str):
        """Ranks, weights and delays in the reference's connectivity file
        layout (.npz, .gz, .mat or pickle), loadable with from_file()."""
        import os
        import pickle
        path = os.path.dirname(filename)
        if path and not os.path.isdir(path):
            os.makedirs(path)
        delay = self.delay
        data = {"name": self.name, "post_ranks": self.post_ranks,
                "pre_ranks": np.array(self._pre_ranks_of(), dtype=object),
                "w": np.array(self.get("w"), dtype=object),
                "delay": np.array(delay, dtype=object) if isinstance(delay, list) else delay,
                "max_delay": self.max_delay, "uniform_delay": self.uniform_delay,
                "size": self.size, "nb_synapses": self.nb_synapses}
        ext = os.path.splitext(filename)[1]
        if ext == ".gz":
            import gzip
            with gzip.open(filename, mode="wb") as f:
                pickle.dump(data, f, protocol=pickle.HIGHEST_PROTOCOL)
        elif ext == ".npz":
            np.savez_compressed(filename, **data)
        elif ext == ".mat":
            import scipy.io as sio
            sio.savemat(filename, {k: (0 if v is None else v) for k, v in data.items()})
        else:
            with open(filename, mode="wb") as f:
                pickle.dump(data, f, protocol=pickle.HIGHEST_PROTOCOL)

    def from_file(self, filename: str, pickle_encoding=None, storage_format=None,
                  storage_order=None):
        """Connectivity, weights and delays saved by save_connectivity()
        (ANNarchy/core/ConnectorMethods.py:799-890)."""
        import gzip
        import pickle
        if filename.endswith(".npz"):
            raw = np.load(filename, allow_pickle=True, **({} if pickle_encoding is None
                                                          else {"encoding": pickle_encoding}))
            data = {k: (raw[k].item() if raw[k].dtype == object and raw[k].ndim == 0 else raw[k])
                    for k in raw.files}
        else:
            opener = gzip.open if filename.endswith(".gz") else open
            with opener(filename, mode="rb") as f:
                data = pickle.load(f, **({} if pickle_encoding is None else {"encoding": pickle_encoding}))
        post = [int(r) for r in np.asarray(data["post_ranks"]).ravel()]
        pre = [list(map(int, r)) for r in data["pre_ranks"]]
        w_raw = data["w"]
        if np.ndim(w_raw) == 0 or (isinstance(w_raw, np.ndarray) and w_raw.size == 1
                                   and w_raw.dtype != object):
            w = [np.full(len(p), float(np.asarray(w_raw).ravel()[0])) for p in pre]
        else:
            w = [np.atleast_1d(np.asarray(x, dtype=np.float64)) for x in w_raw]
        pos_post = {int(r): i for i, r in enumerate(self.post_ranks_view)}
        pos_pre = {int(r): i for i, r in enumerate(self.pre_ranks)}
        rows = np.concatenate([np.full(len(p), pos_post[r]) for r, p in zip(post, pre)]) if pre else []
        cols = np.concatenate([[pos_pre[c] for c in p] for p in pre]).astype(np.int64) if pre else []
        m = sp.csr_matrix((np.concatenate(w) if w else [], (rows, cols)),
                          shape=(len(self.post_ranks_view), len(self.pre_ranks)))
        delay = data.get("delay")
        if isinstance(delay, np.ndarray) and delay.dtype == object and delay.ndim > 0:
            dm = sp.csr_matrix((np.concatenate([np.atleast_1d(np.asarray(x, dtype=np.float64))
                                                for x in delay]), (rows, cols)), shape=m.shape)
            return self._store(m, "From File", storage_format, None, dm)
        d = 0.0 if delay is None else float(np.asarray(delay).ravel()[0])
        return self._store(m, "From File", storage_format, d)

    connect_from_file = from_file

    def reset(self, attributes=-1, synapses: bool = False):
        """Synaptic variables (not the weights) back to their initial values
        (ANNarchy/core/Projection.py:841-880)."""
        if synapses:
            raise NotImplementedError("Projection.reset(synapses=True) is not supported by this "
                                      "backend")
        if self.net is not None and self.net._compiled:
            self.net._backend.reset_projection(self)
        for name in list(self._host_semi):
            init = next((v["init"] for v in self.desc["variables"] if v["name"] == name), 0.0)
            if not isinstance(init, str):
                self.set({name: float(init)})

    @property
    def post_ranks(self):
        return self.csr_population_ranks()[0].tolist()

    def __repr__(self):
        return (f"Projection({self.name!r}, {self.pre_pop.name}->{self.post_pop.name}, "
                f"target={self.target!r}, {self.nb_synapses} synapses, {self._storage_format})")


class LILConnectivity:
    """Connectivity built row by row by a user function (the reference's
    ANNarchy/cython_ext/Connector.pyx:93-170): add(post_rank, pre_ranks,
    weights, delays) with one weight for all the row's synapses or one per
    synapse, delays in ms (one or one per synapse) kept in steps."""

    def __init__(self, dt: float = 1.0):
        self.dt = float(dt)
        self.post_rank, self.pre_rank, self.w, self.delay = [], [], [], []
        self.max_delay = 0
        self.uniform_delay = -1
        self.size = 0
        self.nb_synapses = 0
        self.requires_sorting = False
        self._last = -1

    def add(self, rank, ranks, w, d):
        rank, ranks = int(rank), [int(r) for r in ranks]
        w = [float(x) for x in np.atleast_1d(w)]
        d = [float(x) for x in np.atleast_1d(d)]
        if rank < self._last:
            self.requires_sorting = True
        else:
            self._last = rank
        if not ranks:
            return
        self.post_rank.append(rank)
        self.pre_rank.append(ranks)
        self.w.append(w if (len(w) > 1 or len(ranks) == 1) else [w[0]] * len(ranks))
        steps = [int(round(x / self.dt)) for x in d]
        self.delay.append(steps)
        self.max_delay = max(self.max_delay, int(round(max(d) / self.dt)))
        if len(d) > 1:
            self.uniform_delay = -1
        else:
            u = int(round(d[0] / self.dt))
            self.uniform_delay = -1 if (self.uniform_delay != u and self.size > 0) else u
        self.size += 1
        self.nb_synapses += len(ranks)

    push_back = add

    def validate(self):
        """Each row's pre-synaptic ranks are distinct."""
        for rank, ranks in zip(self.post_rank, self.pre_rank):
            if len(set(ranks)) != len(ranks):
                raise ValueError(f"LILConnectivity: the dendrite of {rank} has duplicate synapses")


class IndividualSynapse:
    """One synapse of a dendrite: its attributes by name."""

    def __init__(self, dendrite, pre: int):
        object.__setattr__(self, "dendrite", dendrite)
        object.__setattr__(self, "pre", int(pre))
        object.__setattr__(self, "idx", dendrite.pre_ranks.index(int(pre)))

    def __getattr__(self, name):
        return self.dendrite.get(name)[self.idx]

    def __setattr__(self, name, value):
        vals = np.asarray(self.dendrite.get(name), dtype=np.float64).copy()
        vals[self.idx] = value
        self.dendrite.set({name: vals})


class Dendrite:
    """The synapses of one post-synaptic neuron (ANNarchy/core/Dendrite.py):
    `pre_ranks`, `size`, attributes by name."""

    def __init__(self, proj, post_rank: int, idx: int):
        object.__setattr__(self, "proj", proj)
        object.__setattr__(self, "post_rank", int(post_rank))
        object.__setattr__(self, "idx", int(idx))
        object.__setattr__(self, "pre_ranks", proj._pre_ranks_of()[idx])

    @property
    def size(self) -> int:
        return len(self.pre_ranks)

    def __len__(self):
        return self.size

    def get(self, name: str):
        if name in self.proj._host_semi:
            return self.proj.get(name)[self.idx]
        v = self.proj.get(name)
        return v[self.idx] if isinstance(v, list) else v

    def set(self, values: dict):
        for name, value in values.items():
            if name in self.proj._host_semi:
                allv = np.asarray(self.proj.get(name), dtype=np.float64).copy()
                allv[self.idx] = float(value)
                self.proj.set({name: allv})
                continue
            rows = self.proj.get(name)
            rows[self.idx] = np.broadcast_to(np.asarray(value, dtype=np.float64), (self.size,)).copy()
            self.proj.set({name: rows})

    def __getattr__(self, name):
        if name.startswith("_"):
            raise AttributeError(name)
        return self.get(name)

    def __setattr__(self, name, value):
        self.set({name: value})

    def synapse(self, pos):
        """The synapse from the pre-synaptic neuron of this rank or these
        coordinates (ANNarchy/core/Dendrite.py:69-87); None without one."""
        rank = int(pos) if isinstance(pos, (int, np.integer)) else \
            self.proj.pre_pop.rank_from_coordinates(tuple(pos))
        if rank not in self.pre_ranks:
            return None
        return IndividualSynapse(self, rank)

    def synapses(self):
        """The dendrite's synapses in ascending pre-synaptic rank."""
        return (IndividualSynapse(self, n) for n in self.pre_ranks)

    def __getitem__(self, *args):
        return self.synapse(args[0] if len(args) == 1 else args)

    def __iter__(self):
        return self.synapses()

    def receptive_field(self, variable: str = "w", fill: float = 0.0) -> np.ndarray:
        """The values over the pre-synaptic geometry (`fill` elsewhere)."""
        res = np.ones(self.proj.pre_pop.size) * fill
        res[self.pre_ranks] = self.get(variable)
        return res.reshape(self.proj.pre_pop.geometry)
