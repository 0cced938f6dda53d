"""Compiled state of a network on one GPU.

Creates the device arrays of every population, projection and monitor
through the C ABI, generates and loads the network's CUDA module, and runs
steps in chunks whose length is bounded by the monitors' device buffers;
after every chunk the buffers are copied to the host once.

Array names (the generated module binds a __constant__ pointer to each):
  pop<k>__<attr>            local attributes (size N) and globals (size 1)
  pop<k>___sum_<target>     rate-coded weighted sums
  pop<k>__spk               spike bitmap of the last step (N/32 words)
  pop<k>__refractory[_remaining], pop<k>__last_spike
  proj<k>__row_ptr/col/w/post_rank        CSR rows (post-major, pre ascending)
  proj<k>__col_ptr/post_idx/w_pre/inv_idx pre-major view for spike scatter
  proj<k>__<format arrays>                ELL/SELL/BSR/HYB (rate-coded)
  mon<k>__spk / mon<k>__<var>             recording buffers
"""
from __future__ import annotations

import numpy as np

from ..generator import formats as F
from ..generator.codegen import (CodeGenerator, compensated_vars, global_equations, grid_for, list_grid,
                                 trace_layout)
from ..runtime.lib import DryNative, NativeNet
from .monitor import array_name

BF16 = np.uint16
MAX_MONITOR_BYTES = 256 << 20
LOCAL_SMEM_LIMIT = 220 * 1024


def to_bf16(x: np.ndarray) -> np.ndarray:
    """float -> bfloat16 bits, round to nearest even."""
    f = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    rounding = ((f >> 16) & 1) + 0x7FFF
    return ((f + rounding) >> 16).astype(np.uint16)


def from_bf16(h: np.ndarray) -> np.ndarray:
    return (np.asarray(h, dtype=np.uint32) << 16).view(np.float32).astype(np.float64)


class CompiledNetwork:
    def __init__(self, net, dry: bool = False):
        self.net = net
        cfg = net._config
        self.exact = cfg["precision"] == "double"
        self.real = np.float64 if self.exact else np.float32
        wd = cfg.get("weight_dtype") or ("float64" if self.exact else "float32")
        if self.exact and wd != "float64":
            raise ValueError("double precision uses float64 weights")
        self.wdtype = {"float64": np.float64, "float32": np.float32, "bfloat16": BF16}[wd]
        self.wctype = {"float64": "double", "float32": "float", "bfloat16": "anb_bf16"}[wd]
        self.native = DryNative() if dry else NativeNet(cfg.get("device", 0))
        self.layout: dict[int, dict] = {}
        self.mon_layout: dict[int, dict] = {}
        self.local_layout = None
        self.spike_lists = False
        self._col_ptr: dict[int, np.ndarray] = {}
        self.engine = None
        self.module = None
        self.slots: dict[int, int] = {}    # history ring length (steps) per population
        # sharding by post neurons: (rank, world) and the owned slice per population
        self.shard = net._config.get("shard")
        self.owned: dict[int, tuple[int, int]] = {}
        self._exchange = None

    # --------------------------------------------------------------- helpers
    def _w(self, w: np.ndarray) -> np.ndarray:
        return to_bf16(w) if self.wdtype is BF16 else np.asarray(w, dtype=self.wdtype)

    def _dtype_of(self, pop, name):
        return np.int32 if pop._ctype.get(name) in ("int", "bool") else self.real

    # ------------------------------------------------------- packed traces
    def _trace_dtype(self, proj):
        lay = trace_layout(proj, self.exact)
        if lay is None:
            return None
        names, nbytes = lay
        return np.dtype({"names": names + ["_last_event"],
                         "formats": ["<f4"] * len(names) + ["<i4"],
                         "offsets": [4 * i for i in range(len(names) + 1)], "itemsize": nbytes})

    def _trace_init(self, proj, nnz, host=None):
        """Records of the packed traces: the initial values (or `host` arrays)
        and last event -10000, as uint32 words."""
        dt = self._trace_dtype(proj)
        rec = np.zeros(nnz if host is not None else 1, dtype=dt)
        for n in dt.names[:-1]:
            if host is not None and n in host:
                rec[n] = host[n]
            else:
                init = next((v["init"] for v in proj.desc["variables"] + proj.desc["parameters"]
                             if v["name"] == n), 0.0)
                rec[n] = float(init) if not isinstance(init, str) else 0.0
        rec["_last_event"] = -10000
        return rec.view(np.uint32).reshape(-1)

    # ----------------------------------------------------------------- build
    def build(self):
        net = self.net
        nat = self.native
        nat.initialize(net.dt)
        # key of the random draws in equations (drawn from the network's seed,
        # only when some equation draws)
        if any(p.desc.get("random_distributions") for p in net.populations + net.projections):
            key = net._rng.integers(0, 2**32, 2, dtype=np.uint64).astype(np.uint32)
        else:
            key = np.zeros(2, dtype=np.uint32)
        nat.set_seed(int(key[0]) | (int(key[1]) << 32))
        # history kept per population: its outgoing projections' largest delay
        for pop in net.populations:
            self.slots[pop.id] = max([1] + [int(p.max_delay) for p in net.projections
                                           if p.pre_pop is pop])
        self.engine = self._choose_engine()
        # fast grid engine: per-step spike lists drive the event kernels (a
        # sharded network transmits from the exchanged bitmaps instead)
        self.spike_lists = (not self.exact and self.engine == "grid" and not self.shard)
        if self.shard:
            self._setup_shard()
        for pop in net.populations:
            self._create_population(pop)
        for proj in net.projections:
            self._create_projection(proj)
        for mon in net.monitors:
            self._create_monitor(mon)
        for pop in net.populations:
            pop._init_state = {k: v.copy() for k, v in pop._host.items()}
        if self.engine == "local":
            self._build_cluster()
            return
        gen = CodeGenerator(self)
        if self.engine == "local":
            self._local_layout()
            mod = gen.local_module()
        else:
            nat.create("tickc", np.zeros(1, dtype=np.uint32))
            if any(getattr(p, "stop_condition", None) for p in net.populations):
                nat.create("stop_flags", np.full(len(net.populations), -1, dtype=np.int64))
            if self._persistent() and gen.persistent_ok():
                nat.create("gbar", np.zeros(2, dtype=np.uint32))
                mod = gen.persistent_module()
            else:
                mod = gen.grid_module()
        self.module = mod
        nat.load_module(mod.source, mod.options)
        self.write_constants()
        if mod.local is not None:
            nat.set_local_kernel(*mod.local)
        else:
            nat.plan(mod.plan)
            nat.set_graph_steps(int(net._config.get("graph_steps", 32)))
            nat.set_pdl(bool(net._config.get("pdl", True)))
            for pop_id, kernel, grid, block, mode_all in mod.stops:
                nat.set_stop_kernel(pop_id, kernel, grid, block, mode_all)

    def _persistent(self) -> bool:
        """Run the grid engine's step as one persistent cooperative launch
        (config persistent=True). Off by default: on the 1e9-synapse network
        it measured 26.9 us per step against 26.8 us for the graph of
        launches, and 17.4 against 16.1 us on its 200k-neuron version."""
        return bool(self.net._config.get("persistent", False))

    def _build_cluster(self):
        """Fast spiking engine on one thread-block cluster: the smallest
        cluster (up to 16 CTAs) whose shared memory holds the state and the
        synapses; otherwise 8 CTAs with the synapses read from global memory.
        A cluster the device cannot schedule falls back the same way."""
        from ..runtime.lib import BackendError
        want = self.net._config.get("cluster_size")
        total = max(p.size for p in self.net.populations)
        cands = [int(want)] if want else [c for c in (1, 2, 4, 8, 16) if (total + c - 1) // c <= 1024]
        # weights in shared memory with the smallest cluster that holds them,
        # else weights read from global memory
        plans = [(c, True) for c in cands] + [(c, False) for c in reversed(cands)]
        last_err = None
        for C, in_smem in plans:
            if self._cluster_layout(C, in_smem) > LOCAL_SMEM_LIMIT:
                continue
            for k, arrs in self._cl_arrays.items():
                for name, arr in arrs.items():
                    if name in ("cl_w", "cl_pal"):
                        arr = arr if self.exact else self._w(arr)
                    self.native.create(f"proj{k}__{name}", arr)
            gen = CodeGenerator(self)
            mod = gen.cluster_module()
            try:
                self.native.load_module(mod.source, mod.options)
                self.write_constants()
                self.native.set_local_kernel(*mod.local)
            except BackendError as exc:
                last_err = exc
                continue
            self.module = mod
            self.engine = "cluster"
            return
        raise RuntimeError(f"no cluster configuration fits this network ({last_err})")

    def _setup_shard(self):
        from .shard import Exchange, owned_range
        rank, world = (int(x) for x in self.shard)
        if not 0 <= rank < world:
            raise ValueError(f"shard {self.shard}: rank must lie in [0, world)")
        net = self.net
        if any(p.neuron_type.type != "spike" for p in net.populations):
            raise NotImplementedError("sharded networks are spiking networks")
        if any(p.max_delay > 1 for p in net.projections):
            raise NotImplementedError("sharded networks transmit without synaptic delays")
        for pop in net.populations:
            self.owned[pop.id] = owned_range(pop.size, rank, world)
        if not isinstance(self.native, DryNative):
            self._exchange = Exchange(rank, world, net._config.get("shard_group"))

    def _local_rows(self, proj, post_rank, row_ptr, cols, w):
        """The rows of the owned post neurons (sharded networks) and the mask
        of their synapses in CSR order."""
        keep_syn = np.ones(cols.size, dtype=bool)
        if not self.shard:
            return post_rank, row_ptr, cols, w, keep_syn
        lo, hi = self.owned[proj.post_pop.id]
        rows = (post_rank >= lo) & (post_rank < hi)
        lengths = np.diff(row_ptr)
        keep_syn = np.repeat(rows, lengths)
        new_ptr = np.zeros(int(rows.sum()) + 1, dtype=row_ptr.dtype)
        np.cumsum(lengths[rows], out=new_ptr[1:])
        return post_rank[rows], new_ptr, cols[keep_syn], w[keep_syn], keep_syn

    def _choose_engine(self) -> str:
        want = self.net._config.get("engine", "auto")
        if self.net._config.get("shard"):
            if want == "local":
                raise NotImplementedError("sharded networks run on the grid engine")
            return "grid"
        ok, why = self._local_possible()
        if any(getattr(p, "stop_condition", None) for p in self.net.populations):
            ok, why = False, "stop conditions"
        if want == "local":
            if not ok:
                raise NotImplementedError("local engine not possible: " + why)
            return "local"
        if want == "grid":
            return "grid"
        return "local" if ok else "grid"

    def _local_possible(self):
        net = self.net
        if any(p.max_delay > 1 for p in net.projections):
            return False, "synaptic delays"
        if any(p.neuron_type.type != "spike" for p in net.populations):
            return False, "rate-coded populations"
        if any(p.synapse_type.type != "spike" or p.plastic for p in net.projections):
            return False, "plastic or rate-coded projections"
        if any(getattr(p, "_device_conn", None) for p in net.projections):
            return False, "device-generated connectivity"
        if any(v != "spike" for m in net.monitors for v in m.variables):
            return False, "variable monitors"
        if any(global_equations(p) or p._globalops for p in net.populations):
            return False, "population-level variables with equations or global operations"
        smem = self._local_smem_bytes()
        if smem > LOCAL_SMEM_LIMIT:
            return False, f"state needs {smem} bytes of shared memory"
        return True, ""

    def _local_vars(self, pop):
        names = []
        for v in pop.desc["variables"]:
            if v.get("cpp"):
                names.append(v["name"])
        for r in pop.desc["spike"]["spike_reset"]:
            if r["name"] not in names:
                names.append(r["name"])
        for t in pop.targets:
            if "g_" + t not in names:
                names.append("g_" + t)
        return [n for n in names if pop._locality.get(n) == "local"]

    def _local_smem_bytes(self):
        total = 0
        rb = np.dtype(self.real).itemsize
        for pop in self.net.populations:
            n = pop.size
            total += len(self._local_vars(pop)) * ((n * rb + 15) // 16 * 16)
            total += (n * 4 + 15) // 16 * 16                     # refractory_remaining
            total += (((n + 31) // 32) * 4 + 15) // 16 * 16       # spike bitmap
        return total

    def _local_layout(self):
        off = 0
        pops = {}
        rb = np.dtype(self.real).itemsize
        rct = "double" if self.exact else "float"
        for pop in self.net.populations:
            d = {}
            n = pop.size
            for name in self._local_vars(pop):
                d[name] = (off, rct)
                off += (n * rb + 15) // 16 * 16
            d["refractory_remaining"] = (off, "int")
            off += (n * 4 + 15) // 16 * 16
            d["spk"] = (off, "anb_u32")
            off += (((n + 31) // 32) * 4 + 15) // 16 * 16
            pops[pop.id] = d
        self.local_layout = {"pops": pops, "smem": off, "block": 1024}

    def _cluster_size(self) -> int:
        """CTAs per cluster for the fast local engine: about 512 neurons per
        CTA, at most 8 (the portable cluster size); the double-precision mode
        keeps one CTA (its ordered delivery needs a single owner)."""
        if self.exact:
            return 1
        want = self.net._config.get("cluster_size")
        if want:
            return int(want)
        total = max(p.size for p in self.net.populations)
        return int(max(1, min(8, (total + 511) // 512)))

    def _cluster_layout(self, C: int, weights_in_smem: bool = True):
        """Shared-memory layout of one CTA of a C-CTA cluster and the
        per-CTA incoming-synapse arrays (see CodeGenerator.cluster_module).
        Returns the bytes of shared memory per CTA."""
        pops, projs = {}, {}
        off = 0
        rb = np.dtype(self.real).itemsize
        rct = "double" if self.exact else "float"
        a16 = lambda x: (x + 15) // 16 * 16
        for pop in self.net.populations:
            chunk = ((pop.size + C - 1) // C + 31) // 32 * 32
            words = (pop.size + 31) // 32
            d = {}
            for name in self._local_vars(pop):
                d[name] = (off, rct)
                off += a16(chunk * rb)
            d["refractory_remaining"] = (off, "int")
            off += a16(chunk * 4)
            if pop._has_refractory:
                d["refractory"] = (off, "int")
                off += a16(chunk * 4)
            for par in (0, 1):
                d[f"spk{par}"] = (off, "anb_u32")
                off += a16(words * 4)
            for name in compensated_vars(pop, self.exact, self.net._config):
                d["kc_" + name] = (off, rct)
                off += a16(chunk * rb)
            pops[pop.id] = {"chunk": chunk, "arrays": d}
        per_cta = np.zeros(C, dtype=np.int64)
        self._cl_arrays = {}
        for proj in self.net.projections:
            lay = self.layout[proj.id]
            span = (lay["w1"] - lay["w0"]) * 32
            arrs = self._incoming_slices(proj, C, pops[proj.post_pop.id]["chunk"], lay["w0"] * 32,
                                         span)
            self._cl_arrays[proj.id] = arrs
            per_cta += np.diff(arrs["cl_base"])
            projs[proj.id] = {"span": span, "w_smem": weights_in_smem}
            pops[proj.pre_pop.id]["arrays"][f"cp{proj.id}"] = (off, "int")
            off += a16((span + 1) * 4)
        pool = int(per_cta.max()) if per_cta.size else 0
        wb = 8 if self.exact else (2 if self.wdtype is BF16 else 4)
        wct = "double" if self.exact else ("anb_bf16" if self.wdtype is BF16 else "float")
        # weight palettes: every projection with at most 256 distinct weights
        # stores 1-byte indices into a per-projection table
        pal = {k: np.unique(a["cl_w"]) for k, a in self._cl_arrays.items()}
        use_pal = bool(pal) and all(v.size <= 256 for v in pal.values()) and wb > 1
        pool_l = {"post": (off, "unsigned short"), "w": (None, wct), "palette": use_pal,
                  "w_ct_real": wct}
        off += a16(pool * 2)
        if use_pal:
            for k, v in pal.items():
                arrs = self._cl_arrays[k]
                arrs["cl_wi"] = np.searchsorted(v, arrs["cl_w"]).astype(np.uint8)
                arrs["cl_pal"] = v
                projs[k]["pal"] = (off, int(v.size))
                off += a16(v.size * wb)
            pool_l["w"] = (off, "unsigned char")
            off += a16(pool)
            for k in projs:
                projs[k]["w_smem"] = True
        elif weights_in_smem:
            pool_l["w"] = (off, wct)
            off += a16(pool * wb)
        block = int(min(1024, max(128, max(l["chunk"] for l in pops.values()))))
        self.cluster_layout = {"C": C, "block": block, "pops": pops, "proj": projs, "smem": off,
                               "pool": pool_l}
        return off

    def _incoming_slices(self, proj, C, chunk_post, lo, span):
        """Per owner CTA r (post neurons [r*chunk_post, (r+1)*chunk_post)),
        the synapses of projection `proj` onto its neurons, sorted by pre rank
        then post rank: cl_base[r] = first synapse of CTA r, cl_ptr[r] = its
        local column pointers over pre ranks lo..lo+span, cl_post = post index
        relative to the CTA, cl_w = weights."""
        post_rank, row_ptr, cols, w = proj.csr_population_ranks()
        rows_of = np.repeat(np.arange(post_rank.size), np.diff(row_ptr))
        posts = post_rank[rows_of].astype(np.int64)
        owner = posts // chunk_post
        pre_rel = cols.astype(np.int64) - lo
        order = np.lexsort((posts, pre_rel, owner))
        counts = np.bincount(owner * span + pre_rel, minlength=C * span).reshape(C, span)
        cl_ptr = np.zeros((C, span + 1), dtype=np.int32)
        np.cumsum(counts, axis=1, out=cl_ptr[:, 1:])
        cl_base = np.zeros(C + 1, dtype=np.int32)
        np.cumsum(np.bincount(owner, minlength=C), out=cl_base[1:])
        return {"cl_ptr": cl_ptr.reshape(-1), "cl_base": cl_base,
                "cl_post": (posts - owner * chunk_post)[order].astype(np.uint16),
                "cl_w": w[order]}

    def _create_population(self, pop):
        nat = self.native
        for name, arr in pop._host.items():
            dt = np.int32 if arr.dtype == np.int32 else self.real
            nat.create(f"pop{pop.id}__{name}", np.asarray(arr, dtype=dt).reshape(-1))
        for name in compensated_vars(pop, self.exact, self.net._config):
            nat.create(f"pop{pop.id}__kc_{name}", np.zeros(pop.size, dtype=self.real))
        if pop.neuron_type.type == "rate":
            for t in pop.targets:         # the last step's weighted sums (Population.sum)
                nat.create(f"pop{pop.id}___last_sum_{t}", np.zeros(pop.size, dtype=self.real))
        if hasattr(pop, "_ta_schedule_ms"):
            self.write_timed_array(pop)
        R = self.slots.get(pop.id, 1)
        if pop.neuron_type.type == "rate" and R > 1:
            # rates of the last R steps (slot t % R holds step t), filled with
            # the current rates like the reference's queue at compile and reset
            nat.create(f"pop{pop.id}___delayed_r", self._ring_of(pop, pop._host["r"]))
        if pop.neuron_type.type == "spike":
            n = pop.size
            # spike bitmaps of the last R steps (slot t % R holds step t)
            words = (n + 31) // 32
            if self.shard:
                # room for every rank's chunk of words: the all-gather writes
                # world x chunk words in place
                from .shard import chunk_words
                words = max(words, chunk_words(n, int(self.shard[1])) * int(self.shard[1]))
            nat.create(f"pop{pop.id}__spk", np.zeros(R * words, dtype=np.uint32))
            if self.spike_lists:
                nat.create_empty(f"pop{pop.id}__spl", np.int32, (2 * n,))
                nat.create(f"pop{pop.id}__spn", np.zeros(2, dtype=np.int32))
            nat.create(f"pop{pop.id}__refractory", pop.refractory_steps.astype(np.int32))
            nat.create(f"pop{pop.id}__refractory_remaining", np.zeros(n, dtype=np.int32))
            nat.create(f"pop{pop.id}__last_spike", np.full(n, -10000, dtype=np.int64))
        if global_equations(pop):
            # ticket of the update kernel's last CTA, which stores the new
            # values of the population-level variables
            nat.create(f"pop{pop.id}__gtick", np.zeros(1, dtype=np.uint32))

    def _syn_local_names(self, proj):
        from ..generator.codegen import syn_local_names
        return syn_local_names(proj)[1:]

    def _create_device_projection(self, proj):
        """Fixed in-degree or fixed-probability projection generated on the
        device."""
        nat = self.native
        k = proj.id
        d = proj._device_conn
        if d["kind"] == "pattern":
            wdt0 = np.float64 if (self.exact or proj.synapse_type.type != "spike" or proj.plastic
                                  or self.shard) else self.wdtype
            nnz = nat.connect_distance_pattern(f"proj{k}", d["pkind"], d["post_c"], d["pre_c"],
                                               d["a_pos"], d["den_pos"], d["a_neg"], d["den_neg"],
                                               d["threshold"], d["exclude_self"], wdt0)
            if (proj.synapse_type.type != "spike" or proj.plastic or self.shard
                    or isinstance(nat, DryNative)):
                # the CSR comes back for the host path (storage formats, plastic
                # records, sharding)
                npost, npre = len(proj.post_ranks_view), len(proj.pre_ranks)
                if isinstance(nat, DryNative):
                    rp, col, w = np.zeros(npost + 1, np.int64), np.zeros(0, np.int64), np.zeros(0)
                else:
                    rp = nat.read(f"proj{k}__row_ptr").astype(np.int64)
                    col = nat.read(f"proj{k}__col").astype(np.int64)
                    w = nat.read(f"proj{k}__w").astype(np.float64)
                for suffix in ("__post_rank", "__row_ptr", "__col", "__w"):
                    nat.free(f"proj{k}{suffix}")
                proj._device_conn = None
                import scipy.sparse as sp
                proj._store(sp.csr_matrix((w, col, rp), shape=(npost, npre)), d["name"],
                            d["storage_format"], d["delays"])
                return self._create_projection(proj)
            return self._finish_device_projection(proj, nnz, np.diff(
                nat.read(f"proj{k}__row_ptr").astype(np.int64)))
        if proj.synapse_type.type != "spike":
            raise NotImplementedError("device connectors are implemented for spiking projections")
        npost = len(proj.post_ranks_view)
        post0, row0 = int(proj.post_ranks_view[0]), 0
        if self.shard:                    # the owned rows of this projection
            lo, hi = self.owned[proj.post_pop.id]
            a, b = max(lo, post0), min(hi, post0 + npost)
            if b <= a:
                raise NotImplementedError("every rank must own at least one row of each projection")
            row0, post0, npost = a - post0, a, b - a
        pre_lo, pre_hi = int(proj.pre_ranks[0]), int(proj.pre_ranks[-1]) + 1
        plastic = proj.plastic
        wdt = np.float64 if self.exact else (np.float32 if plastic else self.wdtype)
        if d["kind"] == "fixed_number_pre":
            nat.connect_fixed_number_pre(f"proj{k}", npost, post0, pre_lo, pre_hi,
                                         d["number"], d["seed"], d["wkind"], d["a"], d["b"], wdt,
                                         d["exclude_self"], row_offset=row0)
            nnz = npost * d["number"]
            lengths = np.full(npost, d["number"], dtype=np.int64)
        else:
            nnz = nat.connect_fixed_probability(f"proj{k}", npost, post0, pre_lo, pre_hi,
                                                d["probability"], d["seed"], d["wkind"], d["a"],
                                                d["b"], wdt, d["exclude_self"], row_offset=row0)
            if isinstance(nat, DryNative):          # the expected in-degree
                lengths = np.full(npost, -(-nnz // npost), dtype=np.int64)
            else:
                lengths = np.diff(nat.read(f"proj{k}__row_ptr").astype(np.int64))
        return self._finish_device_projection(proj, nnz, lengths)

    def _finish_device_projection(self, proj, nnz, lengths):
        """Layout of a projection whose CSR arrays the device built: the
        column view, the spike-list chunks and the launch sizes."""
        nat = self.native
        k = proj.id
        npost = len(proj.post_ranks_view)
        post0, row0 = int(proj.post_ranks_view[0]), 0
        if self.shard:
            lo, hi = self.owned[proj.post_pop.id]
            a, b = max(lo, post0), min(hi, post0 + npost)
            row0, post0, npost = a - post0, a, b - a
        pre_lo, pre_hi = int(proj.pre_ranks[0]), int(proj.pre_ranks[-1]) + 1
        plastic = proj.plastic
        proj._nnz = nnz
        proj._device_lengths = lengths
        lay = {"rows": npost, "nnz": nnz, "idx_t": "int", "format": "csr", "device": True,
               "w0": pre_lo // 32, "w1": (pre_hi - 1) // 32 + 1}
        for prm in proj.desc["parameters"] + proj.desc["variables"]:
            if prm["locality"] == "global":
                nat.create(f"proj{k}__{prm['name']}", np.array([prm["init"]], dtype=self.real))
        if not self.exact:
            nat.csr_to_csc(f"proj{k}", proj.pre_pop.size, with_weights=not plastic)
        mean_fan = nnz / max(1, pre_hi - pre_lo)
        lay["chunks"] = max(1, -(-int(1.25 * mean_fan) // 32))
        lay["post_chunks"] = max(1, -(-int(lengths.max() if lengths.size else 1) // 32))
        if plastic and self.spike_lists:
            row_of = np.full(proj.post_pop.size, -1, dtype=np.int32)
            row_of[post0:post0 + npost] = np.arange(npost, dtype=np.int32)
            nat.create(f"proj{k}__row_of", row_of)
        if self.spike_lists:
            lay["grid"] = list_grid(pre_hi - pre_lo, lay["chunks"])
        elif self.exact or plastic:
            lay["grid"] = grid_for(npost * 32)
        else:
            lay["grid"] = grid_for((lay["w1"] - lay["w0"]) * 32)
        if plastic:
            nat.create(f"proj{k}__flags", np.array(proj._learn_flags, dtype=np.int32))
            if self._trace_dtype(proj) is not None:
                dt = self._trace_dtype(proj)
                nat.create_empty(f"proj{k}__tr", np.uint32, (nnz * dt.itemsize // 4,))
                nat.fill(f"proj{k}__tr", self._trace_init(proj, nnz))
                # the generated weights into the records' first field
                nat.copy_strided(f"proj{k}__tr", 0, dt.itemsize, f"proj{k}__w", 0, 4, nnz)
                nat.free(f"proj{k}__w")
            else:
                for name in self._syn_local_names(proj):
                    init = next((v["init"] for v in proj.desc["variables"] + proj.desc["parameters"]
                                 if v["name"] == name), 0.0)
                    nat.create_empty(f"proj{k}__{name}", self.real, (nnz,))
                    nat.fill(f"proj{k}__{name}",
                             np.dtype(self.real).type(float(init) if not isinstance(init, str) else 0.0))
                nat.create_empty(f"proj{k}___last_event", np.int64, (nnz,))
                nat.fill(f"proj{k}___last_event", np.int64(-10000))
        self.layout[k] = lay

    def _create_delays(self, proj):
        k = proj.id
        if proj._delay_steps is not None:
            if proj.synapse_type.type == "rate" and proj._storage_format not in ("csr", "auto"):
                raise NotImplementedError("non-uniform delays of rate-coded projections use the csr "
                                          "format (the reference supports them in LIL only)")
            self.native.create(f"proj{k}__dly", np.asarray(proj._delay_steps, dtype=np.int32))
        elif proj.max_delay > 1:
            self.native.create(f"proj{k}__delay", np.array([proj.uniform_delay], dtype=np.int32))

    @staticmethod
    def ring_stride(pop) -> int:
        """Elements per slot of a rate history ring (a multiple of 4, so every
        slot starts 16-byte aligned)."""
        return -(-pop.size // 4) * 4

    def _ring_of(self, pop, r) -> np.ndarray:
        R, S = self.slots[pop.id], self.ring_stride(pop)
        ring = np.zeros((R, S), dtype=self.real)
        ring[:, :pop.size] = np.asarray(r, dtype=self.real).reshape(-1)
        return ring.reshape(-1)

    def write_timed_array(self, pop):
        """Buffer (blocks x N), schedule (steps) and [t0, period, blocks] of a
        TimedArray population."""
        nat, k = self.native, pop.id
        sched, per = pop.steps()
        rates = pop._ta_rates if pop._ta_rates is not None else np.zeros((0, pop.size))
        nb = len(sched)
        nat.create(f"pop{k}__ta_buf", np.asarray(rates[:nb], dtype=self.real).reshape(-1)
                   if nb else np.zeros(1, dtype=self.real))
        nat.create(f"pop{k}__ta_sched", np.asarray(sched if nb else [0], dtype=np.int32))
        nat.create(f"pop{k}__ta_meta", np.array([pop._ta_t0, per, nb], dtype=np.int64))

    def delay_capacity(self, proj) -> int:
        """Largest delay (steps) the pre-synaptic history kept since compile()
        can serve."""
        if proj.max_delay <= 1:
            return 1
        return self.slots[proj.pre_pop.id]

    def read_delays(self, proj) -> np.ndarray:
        return self.native.read(f"proj{proj.id}__dly").astype(np.int32)

    def write_delays(self, proj, steps: np.ndarray):
        name = f"proj{proj.id}__dly" if proj._delay_steps is not None else f"proj{proj.id}__delay"
        self.native.write(name, np.asarray(steps, dtype=np.int32))

    def _create_batched_tc(self, proj):
        """A projection shared by the copies of a RateBatch: the per-copy
        weights as 64 x 64 bfloat16 blocks in the layout of the tensor-core
        product (one set for all copies), and the packed-rate scratch."""
        from ..spmm import TILE, canonical_tiles
        from ..generator.formats import bsr_arrays
        nat = self.native
        k = proj.id
        batch, w = proj._batched
        n_post, n_pre = w.shape
        d = bsr_arrays(np.arange(n_post), w.indptr, w.indices, w.data, n_pre, TILE)
        vals = d["values"].reshape(-1, TILE, TILE).transpose(0, 2, 1)      # [block][row][k]
        n_bcols = -(-n_pre // TILE)
        nat.create(f"proj{k}__brow", d["block_row_ptr"].astype(np.int32))
        nat.create(f"proj{k}__bcol", d["block_col"].astype(np.int32))
        nat.create(f"proj{k}__tiles", to_bf16(canonical_tiles(vals)))
        nat.create_empty(f"proj{k}__xt", np.uint16, (n_bcols * batch * TILE,))
        self.layout[k] = {"format": "bsr_tc", "rows": n_post, "nnz": int(w.nnz),
                          "n_block_rows": int(d["n_block_rows"]), "n_blocks": int(d["n_blocks"]),
                          "batch": batch, "n_pre": n_pre, "n_post": n_post}

    def _create_projection(self, proj):
        nat = self.native
        k = proj.id
        if getattr(proj, "_batched", None) is not None:
            return self._create_batched_tc(proj)
        if getattr(proj, "_device_conn", None):
            return self._create_device_projection(proj)
        self._create_delays(proj)
        if proj._csr is None:
            raise RuntimeError(f"projection {proj.name} has no connectivity (call a connector)")
        post_rank, row_ptr, cols, w = proj.csr_population_ranks()
        post_rank, row_ptr, cols, w, keep_syn = self._local_rows(proj, post_rank, row_ptr, cols, w)
        rows = int(post_rank.size)
        nnz = int(cols.size)
        idx_t = "int" if nnz < 2**31 - 1 else "long long"
        lay = {"rows": rows, "nnz": nnz, "idx_t": idx_t, "format": "csr"}
        nat.create(f"proj{k}__post_rank", post_rank)
        nat.create(f"proj{k}__row_ptr", row_ptr.astype(np.int32 if idx_t == "int" else np.int64))
        nat.create(f"proj{k}__col", cols)
        nat.create(f"proj{k}__w", self._w(w))
        for prm in proj.desc["parameters"] + proj.desc["variables"]:
            if prm["locality"] == "global":
                value = proj._global_values.get(prm["name"], prm["init"])
                nat.create(f"proj{k}__{prm['name']}", np.array([value], dtype=self.real))
        if proj.synapse_type.type == "rate":
            learning = CodeGenerator.rate_learning(proj)
            custom = CodeGenerator.custom_psp(proj)
            if custom and not learning:
                # the psp kernel reads the synapse's own attributes, real weights
                if not self.exact:
                    nat.create(f"proj{k}__w", np.asarray(w, dtype=np.float32))
                for name, arr in proj._host_attr.items():
                    nat.create(f"proj{k}__{name}", np.asarray(arr, dtype=self.real)[keep_syn])
                for name, arr in proj._host_semi.items():
                    nat.create(f"proj{k}__{name}", np.asarray(arr, dtype=self.real))
            if learning:
                # the update kernel walks the CSR rows and writes the weights in place
                if proj._storage_format not in ("csr", "auto"):
                    raise NotImplementedError(f"{proj.name}: rate-coded projections with synaptic "
                                              "equations use the csr format in this backend")
                if proj.max_delay > 1:
                    raise NotImplementedError(f"{proj.name}: rate-coded learning with synaptic "
                                              "delays is not supported by this backend")
                if not self.exact:
                    nat.create(f"proj{k}__w", np.asarray(w, dtype=np.float32))
                for name, arr in proj._host_attr.items():
                    nat.create(f"proj{k}__{name}", np.asarray(arr, dtype=self.real)[keep_syn])
                for name, arr in proj._host_semi.items():
                    nat.create(f"proj{k}__{name}", np.asarray(arr, dtype=self.real))
                nat.create(f"proj{k}__flags", np.array(proj._learn_flags, dtype=np.int32))
            fmt = ("csr" if (proj._delay_steps is not None or learning or custom)
                   else self._rate_format(proj, lay))
            lay["format"] = fmt
            if fmt != "csr":
                F.create_format_arrays(self, proj, fmt, post_rank, row_ptr, cols, w, lay)
            lay["group"] = F.csr_group(nnz / max(rows, 1))
            lay["split"] = int(self.net._config.get("ell_split", 4))
            lay["kahan_min"] = 10000
            lay["grid"] = grid_for(rows * (lay["group"] if not self.exact and fmt == "csr" else 1))
            if fmt == "csr" and not self.exact:
                light, heavy = F.csr_bins(row_ptr)
                lay["heavy"] = int(heavy.size)
                lengths = np.diff(row_ptr)
                lay["vgroup"] = F.vec_group(float(lengths[light].mean()) if light.size else 1.0)
                if heavy.size:
                    nat.create(f"proj{k}__rows_light", light)
                    nat.create(f"proj{k}__rows_heavy", heavy)
                lay["light"] = int(light.size)
        else:
            # pre-major view (the reference's CSRC column view, CSRCMatrix.hpp:164-222)
            npre = proj.pre_pop.size
            rows_of = np.repeat(np.arange(rows, dtype=np.int64), np.diff(row_ptr))
            order = np.lexsort((rows_of, cols))
            col_ptr = np.zeros(npre + 1, dtype=np.int32)
            np.cumsum(np.bincount(cols, minlength=npre), out=col_ptr[1:])
            nat.create(f"proj{k}__col_ptr", col_ptr)
            self._col_ptr[k] = col_ptr
            nat.create(f"proj{k}__post_idx", post_rank[rows_of[order]].astype(np.int32))
            nat.create(f"proj{k}__inv_idx", order.astype(np.int32))
            if not proj.plastic:
                nat.create(f"proj{k}__w_pre", self._w(w[order]) if not self.exact else w[order])
            lay["w0"] = int(proj.pre_ranks.min()) // 32
            lay["w1"] = int(proj.pre_ranks.max()) // 32 + 1
            fan = np.diff(col_ptr)
            lay["chunks"] = max(1, -(-int(fan.max() if fan.size else 1) // 32))
            lay["post_chunks"] = max(1, -(-int(np.diff(row_ptr).max() if rows else 1) // 32))
            if proj.plastic and self.spike_lists:
                row_of = np.full(proj.post_pop.size, -1, dtype=np.int32)
                row_of[post_rank] = np.arange(rows, dtype=np.int32)
                nat.create(f"proj{k}__row_of", row_of)
            # warp per post row: exact order, per-synapse delays, and plastic
            # delayed projections (the spike lists hold only the last step)
            gather = self.exact or proj._delay_steps is not None or (
                proj.plastic and (proj.max_delay > 1 or not self.spike_lists))
            if gather:
                lay["grid"] = grid_for(rows * 32)
            elif self.spike_lists:
                lay["grid"] = list_grid(len(proj.pre_ranks), lay["chunks"])
            elif proj.plastic:
                lay["grid"] = grid_for(rows)
            else:
                lay["grid"] = grid_for((lay["w1"] - lay["w0"]) * 32)
            if proj.plastic:
                nat.create(f"proj{k}__flags", np.array(proj._learn_flags, dtype=np.int32))
                host = {name: np.asarray(arr)[keep_syn] for name, arr in proj._host_attr.items()}
                if self._trace_dtype(proj) is not None:
                    # w and the traces in one record per synapse (float32)
                    nat.free(f"proj{k}__w")
                    nat.create(f"proj{k}__tr", self._trace_init(proj, nnz, {**host, "w": w}))
                else:
                    if self.wdtype is not np.float64 and not self.exact:
                        # plastic weights stay float32 (they are updated every event)
                        nat.create(f"proj{k}__w", np.asarray(w, dtype=np.float32))
                    for name, arr in host.items():
                        nat.create(f"proj{k}__{name}", np.asarray(arr, dtype=self.real))
                    for name, arr in proj._host_semi.items():
                        nat.create(f"proj{k}__{name}", np.asarray(arr, dtype=self.real))
                    nat.create(f"proj{k}___last_event", np.full(nnz, -10000, dtype=np.int64))
        self.layout[k] = lay

    def _rate_format(self, proj, lay) -> str:
        fmt = proj._storage_format
        if fmt == "auto":
            fmt = F.select_format(proj, self)
        return fmt

    def _create_monitor(self, mon):
        nat = self.native
        m = mon.id
        pop = mon.population
        words = (pop.size + 31) // 32
        n = pop.size if mon.ranks is None else len(mon.ranks)
        nvars = sum(1 for v in mon.variables if v != "spike")
        per_step = (words * 4 if "spike" in mon.variables else 0) + nvars * n * 8 / mon.period_steps
        cap_steps = int(max(1, min(self.net._config.get("monitor_chunk", 100000),
                                   MAX_MONITOR_BYTES // max(per_step, 1))))
        lay = {"words": words, "n": n, "cap_steps": cap_steps,
               "cap_spike": cap_steps if "spike" in mon.variables else 0,
               "cap_var": cap_steps // mon.period_steps + 1}
        nat.create(f"mon{m}__on", np.array([1 if mon._recording else 0], dtype=np.int32))
        nat.create(f"mon{m}__t0", np.zeros(1, dtype=np.int64))
        nat.create(f"mon{m}__t0v", np.zeros(1, dtype=np.int64))
        nat.create(f"mon{m}__start", np.array([mon._start_step], dtype=np.int64))
        if "spike" in mon.variables:
            nat.create_empty(f"mon{m}__spk", np.uint32, (cap_steps, words))
            if self.shard:                # only the owned words are ever written
                nat.fill(f"mon{m}__spk", np.uint32(0))
        if mon.ranks is not None:
            nat.create(f"mon{m}__ranks", np.asarray(mon.ranks, dtype=np.int32))
        for v in mon.variables:
            if v != "spike":
                nat.create_empty(f"mon{m}__{array_name(v)}", np.float64, (lay["cap_var"], n))
                nat.record_declare(f"mon{m}__{array_name(v)}", n, 8, mon.period_steps)
        self.mon_layout[m] = lay

    # ------------------------------------------------------------------- run
    def chunk_steps(self) -> int:
        if not self.mon_layout:
            return 1 << 30
        return min(l["cap_steps"] for l in self.mon_layout.values())

    def write_constants(self):
        """The network constants' values into the loaded module."""
        for name, c in self.net._constants.items():
            self.native.set_constant(name, c.value)

    def run_until(self, nsteps: int, pops, or_and: bool) -> int:
        """At most nsteps steps, ending after the first step at which the
        stop conditions of `pops` hold (all of them, or any); monitors are
        drained per chunk as in run(). Returns the steps run."""
        if self.shard:
            raise NotImplementedError("simulate_until() is not supported for sharded networks")
        if self.engine == "local":
            if any(getattr(p, "stop_condition", None) for p in self.net.populations):
                raise NotImplementedError("stop conditions need the grid engine")
            self.run(nsteps)
            return int(nsteps)
        nat = self.native
        t = nat.get_time()
        left, total = int(nsteps), 0
        cap = self.chunk_steps()
        while left > 0:
            n = min(left, cap)
            starts = self.begin_chunk(t)
            done, stopped = nat.run_until(n, [p.id for p in pops], or_and)
            self.end_chunk(t, done, starts)
            t += done
            total += done
            left -= done
            if stopped or done < n:
                break
        return total

    def run(self, nsteps: int):
        nat = self.native
        t = nat.get_time()
        left = int(nsteps)
        cap = self.chunk_steps()
        while left > 0:
            n = min(left, cap)
            starts = self.begin_chunk(t)
            if self.shard:
                for s in range(n):            # one step, then the spike exchange
                    nat.run(1)
                    self._exchange_spikes(t + s)
            else:
                nat.run(n)
            nat.synchronize()
            self.end_chunk(t, n, starts)
            t += n
            left -= n

    def _exchange_spikes(self, t):
        """Every rank's bitmap words of step t into every rank's bitmap. Over
        NCCL the bitmap is gathered in place in device memory, ordered on the
        network's stream (no host copy); over gloo through the host."""
        from .shard import chunk_words
        rank, world = (int(x) for x in self.shard)
        if self._exchange.device == "cuda":
            for pop in self.net.populations:
                c = chunk_words(pop.size, world)
                self._exchange.all_gather_device(self.native, f"pop{pop.id}__spk", c)
            return
        for pop in self.net.populations:
            words = (pop.size + 31) // 32
            c = chunk_words(pop.size, world)
            slot = t % self.slots.get(pop.id, 1)
            name = f"pop{pop.id}__spk"
            first = min(words, c * rank)
            local = np.zeros(c, dtype=np.uint32)
            cnt = min(words, first + c) - first
            if cnt > 0:
                local[:cnt] = self.native.read(name, count=cnt, offset=slot * words + first)
            full = self._exchange.all_gather(local)[:words]
            self.native.write(name, full, offset_bytes=slot * words * 4)

    def begin_chunk(self, t):
        """Point every monitor's device ring at step t (a chunk of at most
        chunk_steps() steps starts there); returns the first variable-record
        step of each monitor."""
        starts = {}
        for mon in self.net.monitors:
            first = self._first_record(mon, t)
            starts[mon.id] = first
            self.native.write(f"mon{mon.id}__t0", np.array([t], dtype=np.int64))
            self.native.write(f"mon{mon.id}__t0v", np.array([first], dtype=np.int64))
            self.native.write(f"mon{mon.id}__start", np.array([mon._start_step], dtype=np.int64))
            self.native.write(f"mon{mon.id}__on", np.array([1 if mon._recording else 0],
                                                           dtype=np.int32))
        return starts

    def end_chunk(self, t, n, starts):
        """Copy the records of the n steps from t into the host monitors."""
        for mon in self.net.monitors:
            self._drain(mon, t, n, starts[mon.id])

    @staticmethod
    def _first_record(mon, t):
        """First step >= t at which the monitor's variables are recorded."""
        p, off = mon.period_steps, mon.period_offset_steps % mon.period_steps
        return t + ((off - (t - mon._start_step)) % p)

    def _drain(self, mon, t, n, first):
        if not mon._recording:
            return
        nat = self.native
        lay = self.mon_layout[mon.id]
        if "spike" in mon.variables:
            # decoded on the device: only the (step, rank) pairs are copied back
            steps, ranks = nat.monitor_decode(f"mon{mon.id}__spk", n, lay["words"],
                                              mon.population.size)
            mon._append_spikes(steps + t, ranks)
        nrec = 0 if first >= t + n else (t + n - 1 - first) // mon.period_steps + 1
        if nrec > 0:
            rec_steps = first + mon.period_steps * np.arange(nrec)
            for v in mon.variables:
                if v == "spike":
                    continue
                out = np.empty((nrec, lay["n"]), dtype=np.float64)
                nat.read_into(f"mon{mon.id}__{array_name(v)}", out)
                mon._append_values(v, out, rec_steps)

    # ------------------------------------------------------------ attributes
    def read_population_attribute(self, pop, name):
        arr = self.native.read(f"pop{pop.id}__{name}")
        return arr.astype(np.int32 if arr.dtype == np.int32 else np.float64)

    def write_population_attribute(self, pop, name, arr):
        dt = np.int32 if pop._host[name].dtype == np.int32 else self.real
        self.native.write(f"pop{pop.id}__{name}", np.asarray(arr, dtype=dt).reshape(-1))

    def write_refractory(self, pop):
        self.native.write(f"pop{pop.id}__refractory", pop.refractory_steps.astype(np.int32))

    def read_spiked(self, pop):
        bits = self.native.read(f"pop{pop.id}__spk")
        R = self.slots.get(pop.id, 1)
        if R > 1:                               # the slot of the last step
            words = (pop.size + 31) // 32
            slot = (self.native.get_time() - 1) % R
            bits = np.ascontiguousarray(bits[slot * words:(slot + 1) * words])
        return np.nonzero(np.unpackbits(bits.view(np.uint8), bitorder="little")[: pop.size])[0]

    # ----------------------------------------------------------------- reset
    def reset_population(self, pop, attributes=None):
        """Initial values back into the device arrays (all attributes, or
        the given ones) and the reference's PopStruct::reset(): no spikes
        emitted, refractory counters cleared, the delay queues refilled with
        the current rates (ANNarchy/generator/Population/
        SingleThreadTemplates.py:182-212)."""
        nat = self.native
        k = pop.id
        names = list(pop._init_state) if attributes is None else list(attributes)
        for name in names:
            if name.startswith("_sum_"):
                continue
            self.write_population_attribute(pop, name, pop._init_state[name])
        for name in compensated_vars(pop, self.exact, self.net._config):
            nat.fill(f"pop{k}__kc_{name}", self.real(0))
        for t in pop.targets if pop.neuron_type.type == "rate" else []:
            nat.fill(f"pop{k}___sum_{t}", self.real(0))
            nat.fill(f"pop{k}___last_sum_{t}", self.real(0))
        R = self.slots.get(k, 1)
        if pop.neuron_type.type == "rate" and R > 1:
            nat.write(f"pop{k}___delayed_r", self._ring_of(pop, self.read_population_attribute(pop, "r")))
        if pop.neuron_type.type == "spike":
            nat.fill(f"pop{k}__spk", np.uint32(0))
            nat.fill(f"pop{k}__refractory_remaining", np.int32(0))
            nat.fill(f"pop{k}__last_spike", np.int64(-10000))
            if f"pop{k}__spn" in nat.arrays:
                nat.fill(f"pop{k}__spn", np.int32(0))

    def reset_spike_state(self, pop):
        """The spike part of the reference's PopStruct::reset(): no spikes
        emitted, refractory counters cleared, no last spike."""
        nat = self.native
        k = pop.id
        if pop.neuron_type.type == "spike":
            nat.fill(f"pop{k}__spk", np.uint32(0))
            nat.fill(f"pop{k}__refractory_remaining", np.int32(0))
            nat.fill(f"pop{k}__last_spike", np.int64(-10000))
            if f"pop{k}__spn" in nat.arrays:
                nat.fill(f"pop{k}__spn", np.int32(0))

    def reset_projection(self, proj):
        """Synaptic variables (not the weights) back to their initial values."""
        nat = self.native
        k = proj.id
        if f"proj{k}__tr" in nat.arrays:
            # every field but the weights back to its initial value
            dt = self._trace_dtype(proj)
            init = self._trace_init(proj, 0).view(dt)[0]
            st, nnz = self._stage(proj), self.layout[k]["nnz"]
            for name in dt.names[1:]:
                nat.fill(st, np.asarray(init[name]).view(np.uint32))
                nat.copy_strided(f"proj{k}__tr", dt.fields[name][1], dt.itemsize, st, 0, 4, nnz)
            return
        for v in proj.desc["variables"]:
            if v["name"] == "w":
                continue
            name = f"proj{k}__{v['name']}"
            if name in nat.arrays and not isinstance(v["init"], str):
                dtype, _ = nat.arrays[name]
                nat.fill(name, np.dtype(dtype).type(v["init"]))
        if f"proj{k}___last_event" in nat.arrays:
            nat.fill(f"proj{k}___last_event", np.int64(-10000))

    def _stage(self, proj) -> str:
        """A float32 array of the projection's size for packing and
        unpacking one record field on the device."""
        name = f"proj{proj.id}__stage"
        if name not in self.native.arrays:
            self.native.create_empty(name, np.float32, (self.layout[proj.id]["nnz"],))
        return name

    def _field_io(self, proj, name, arr=None):
        """Read (arr None) or write one field of the packed records."""
        dt = self._trace_dtype(proj)
        k, nnz = proj.id, self.layout[proj.id]["nnz"]
        off = dt.fields[name][1]
        st = self._stage(proj)
        if arr is None:
            self.native.copy_strided(st, 0, 4, f"proj{k}__tr", off, dt.itemsize, nnz)
            return self.native.read(st).astype(np.float64)
        self.native.write(st, np.asarray(arr, dtype=dt.fields[name][0]).view(np.float32))
        self.native.copy_strided(f"proj{k}__tr", off, dt.itemsize, st, 0, 4, nnz)

    def _host_only(self, proj, name) -> bool:
        """A synaptic attribute no kernel uses (a parameter of a projection
        without learning or events) has no device array: the host copy is
        its value."""
        return (f"proj{proj.id}__{name}" not in self.native.arrays
                and not isinstance(self.native, DryNative))

    def read_projection_attribute(self, proj, name):
        dt = self._trace_dtype(proj)
        if dt is not None and name in dt.names[:-1]:
            return self._field_io(proj, name)
        if self._host_only(proj, name):
            if name in proj._host_semi:
                return proj._host_semi[name].copy()
            if name in proj._host_attr:
                return proj._host_attr[name].copy()
            glob = {p["name"]: p for p in proj.desc["parameters"] + proj.desc["variables"]}
            return np.array([float(proj._global_values.get(name, glob[name]["init"]))])
        arr = self.native.read(f"proj{proj.id}__{name}")
        if arr.dtype == np.uint16:
            return from_bf16(arr)
        return arr.astype(np.float64)

    def write_projection_attribute(self, proj, name, arr):
        k = proj.id
        tdt = self._trace_dtype(proj)
        if tdt is not None and name in tdt.names[:-1]:
            self._field_io(proj, name, arr)
            return
        if self._host_only(proj, name):
            if name not in proj._host_semi and name not in proj._host_attr:
                proj._global_values[name] = float(np.asarray(arr).reshape(-1)[0])
            return
        dtype, _ = self.native.arrays[f"proj{k}__{name}"]
        data = to_bf16(arr) if dtype == np.uint16 else np.asarray(arr, dtype=dtype)
        self.native.write(f"proj{k}__{name}", data)
        if name == "w" and f"proj{k}__w_pre" in self.native.arrays:
            order = self.native.read(f"proj{k}__inv_idx")
            dtype, _ = self.native.arrays[f"proj{k}__w_pre"]
            pre = arr[order]
            self.native.write(f"proj{k}__w_pre", to_bf16(pre) if dtype == np.uint16
                              else np.asarray(pre, dtype=dtype))
        if name == "w" and self.layout[k].get("format", "csr") != "csr":
            F.refresh_format_weights(self, proj, arr)


def bitmap_to_spikes(buf: np.ndarray, n: int):
    """(steps, words) uint32 bitmaps -> (step offsets, ranks), sorted by step
    then rank."""
    if buf.size == 0:
        return np.zeros(0, np.int64), np.zeros(0, np.int64)
    from ..runtime.lib import bitmap_decode
    return bitmap_decode(buf, n)


def bitmap_to_spikes_numpy(buf: np.ndarray, n: int):
    """Pure numpy version of bitmap_to_spikes (no native library needed)."""
    step, word = np.nonzero(buf)                   # only words holding a spike
    vals = np.ascontiguousarray(buf[step, word])
    bits = np.unpackbits(vals.view(np.uint8).reshape(-1, 4), axis=1, bitorder="little")
    k, b = np.nonzero(bits)
    ranks = word[k].astype(np.int64) * 32 + b
    keep = ranks < n
    return step[k][keep].astype(np.int64), ranks[keep]
