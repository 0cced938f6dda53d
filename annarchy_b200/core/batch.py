"""Batched instances: many independent spiking networks of one structure in
one persistent launch.

The reference runs parameter sweeps and seeds as separate processes, one
network copy each (Network.parallel_run, ANNarchy/core/Network.py:751-900).
Here the copies share one generated kernel: every CTA holds whole instances
in its shared memory and steps them together, so 256 networks of a few
thousand neurons fill the GPU where one of them alone would use a few SMs.

    nets = [build(i) for i in range(256)]      # ordinary Network objects
    batch = Batch(nets, precision="float", weight_dtype="bfloat16")
    batch.compile()
    batch.simulate(500.0)
    nets[3].monitors[0].get("spike")           # per-instance results

Each instance keeps its own Monitor objects and attribute access
(``pop.v``); simulation goes through the batch.
"""
from __future__ import annotations

import math
import re

import numpy as np

from ..runtime.lib import NativeNet, DryNative, bank_interleave, device_sm_count
from ..generator.codegen import compensated_vars, global_equations
from .backend import BF16, MAX_MONITOR_BYTES, to_bf16

# opt-in dynamic shared memory of one CTA on sm_100 (227 KB)
SMEM_LIMIT = 232448


def _neuron_signature(pop):
    d = pop.desc
    return (pop.neuron_type.type,
            tuple((v["name"], v["locality"], v.get("cpp"), v.get("switch"), v.get("method"),
                   tuple(sorted(v.get("bounds", {}).items())))
                  for v in d["variables"]),
            tuple((p["name"], p["locality"], p.get("ctype")) for p in d["parameters"]),
            repr(d.get("spike")), bool(pop._has_refractory), tuple(pop.targets))


def _structure(net):
    pops = net.populations
    pid = {p.id: i for i, p in enumerate(pops)}
    return (tuple(_neuron_signature(p) for p in pops),
            tuple((pid[pr.pre_pop.id], pid[pr.post_pop.id], pr.target, pr.synapse_type.type,
                   bool(pr.plastic)) for pr in net.projections),
            tuple((pid[m.population.id], tuple(m.variables)) for m in net.monitors))


class _Member:
    """Backend of one instance inside a Batch (attribute access and results;
    simulation goes through the batch)."""

    def __init__(self, batch, index):
        self.batch = batch
        self.index = index
        self.native = batch.native
        self.engine = "batch"

    def run(self, nsteps):
        raise RuntimeError("this network is an instance of a Batch: call Batch.simulate()")

    def _slice(self, pop, name):
        b = self.batch
        slot = b.slot_of[self.index]
        k = pop.id
        if pop._locality.get(name) == "local" or name in ("refractory", "refractory_remaining",
                                                          "last_spike"):
            off = int(b.goff[k][slot])
            return off, pop.size
        return slot, 1

    def read_population_attribute(self, pop, name):
        off, n = self._slice(pop, name)
        arr = self.native.read(f"pop{pop.id}__{name}", count=n, offset=off)
        return arr.astype(np.int32 if arr.dtype == np.int32 else np.float64)

    def write_population_attribute(self, pop, name, arr):
        off, n = self._slice(pop, name)
        dtype = self.native.arrays[f"pop{pop.id}__{name}"][0]
        data = np.asarray(arr, dtype=dtype).reshape(-1)
        if data.size != n:
            raise ValueError(f"{name}: expected {n} values, got {data.size}")
        self.native.write(f"pop{pop.id}__{name}", data, offset_bytes=off * np.dtype(dtype).itemsize)

    def write_refractory(self, pop):
        r = pop.refractory_steps.astype(np.int32)
        self.write_population_attribute(pop, "refractory", r)
        slot = int(self.batch.slot_of[self.index])
        u = int(r[0]) if r.size and np.all(r == r[0]) else -1
        self.native.write(f"pop{pop.id}__brefr", np.array([u], dtype=np.int32), offset_bytes=4 * slot)

    def read_spiked(self, pop):
        b = self.batch
        slot = b.slot_of[self.index]
        words = (pop.size + 31) // 32
        bits = self.native.read(f"pop{pop.id}__spk", count=words, offset=int(b.woff[pop.id][slot]))
        return np.nonzero(np.unpackbits(bits.view(np.uint8), bitorder="little")[: pop.size])[0]

    def read_projection_attribute(self, proj, name):
        if name != "w":
            raise AttributeError(f"batched projections expose only w, not {name!r}")
        return proj.csr_population_ranks()[3]

    def write_projection_attribute(self, proj, name, arr):
        raise RuntimeError("weights of a batched instance are fixed after Batch.compile()")


class Batch:
    """Independent spiking networks of one structure, simulated together.

    All networks must have the same populations (neuron equations), the same
    static spiking projections (pre, post, target) and the same monitors, and
    the same dt; sizes, parameter values, initial state, connectivity and
    weights are free. `precision` "double" reproduces every instance's
    single-network result bit for bit; "float" uses float state and float or
    bfloat16 weights (`weight_dtype`)."""

    def __init__(self, networks, precision: str = "float", weight_dtype: str | None = None,
                 device: int = 0, ctas: int | None = None, dry: bool = False,
                 compensate="auto"):
        self.networks = list(networks)
        if not self.networks:
            raise ValueError("Batch needs at least one network")
        self.net = self.networks[0]
        self.exact = precision == "double"
        if precision not in ("double", "float"):
            raise ValueError("precision must be 'double' or 'float'")
        self.real = np.float64 if self.exact else np.float32
        wd = weight_dtype or ("float64" if self.exact else "float32")
        if self.exact and wd != "float64":
            raise ValueError("double precision uses float64 weights")
        self.wdtype = {"float64": np.float64, "float32": np.float32, "bfloat16": BF16}[wd]
        self.device = device
        self.ctas = ctas
        # Kahan-compensated ODE variables in single precision: "auto" = those
        # that are not synaptic conductances (g_*), which keeps 4 bytes per
        # neuron and variable of shared memory for the conductances; True,
        # False or a list of names as for Network.config(compensate=...)
        self.compensate = compensate
        self.dry = dry
        self.native = DryNative() if dry else NativeNet(device)
        self.compiled = False
        self.module = None

    # -------------------------------------------------------------- checks
    def _check(self):
        ref = _structure(self.net)
        dt = self.net.dt
        for i, n in enumerate(self.networks):
            if n._compiled:
                raise RuntimeError(f"network {i} is already compiled on its own")
            if n.dt != dt:
                raise ValueError(f"network {i} has dt={n.dt}, the batch uses {dt}")
            if _structure(n) != ref:
                raise ValueError(f"network {i} does not have the structure of network 0")
        for pr in self.net.projections:
            if pr.synapse_type.type != "spike" or pr.plastic:
                raise NotImplementedError("batched instances support static spiking projections")
            if pr.max_delay > 1:
                raise NotImplementedError("batched instances transmit without synaptic delays")
            if any((v["name"], v.get("eq", "").replace(" ", "")) != ("g_target", "g_target+=w")
                   for v in pr.desc.get("pre_spike", [])) or pr.desc.get("post_spike"):
                raise NotImplementedError("batched projections add w to the target conductance only")
        for m in self.net.monitors:
            if any(v != "spike" for v in m.variables):
                raise NotImplementedError("batched monitors record spikes only")
        for p in self.net.populations:
            if p.desc.get("random_distributions"):
                raise NotImplementedError("batched instances draw no random numbers in equations")
            if global_equations(p) or p._globalops:
                raise NotImplementedError("batched instances evaluate no population-level "
                                          "equations or global operations")

    # -------------------------------------------------------------- layout
    def _smem_arrays(self, pop):
        """Shared-memory arrays of one population: the local attributes the
        update reads or writes, the refractory counter, the compensation
        terms and the spike bitmap (other attributes stay in global memory)."""
        d = pop.desc
        code = " ".join((v.get("cpp") or "") + " " + (v.get("switch") or "") for v in d["variables"])
        code += " " + d["spike"]["spike_cond"] + " " + " ".join(r["cpp"] for r in d["spike"]["spike_reset"])
        used = set(re.findall(r"[A-Za-z_]\w*", code))
        out = []
        for p in pop.desc["parameters"] + pop.desc["variables"]:
            if p["locality"] == "local" and p["name"] in used:
                ct = "int" if p.get("ctype") in ("int", "bool") else ("double" if self.exact else "float")
                out.append((p["name"], ct))
        # the refractory counter in 16 bits when every period fits
        j = self.net.populations.index(pop)
        rmax = max(int(np.max(n.populations[j].refractory_steps, initial=0)) for n in self.networks)
        out.append(("refractory_remaining", "short" if rmax < 32768 else "int"))
        for name in compensated_vars(pop, self.exact, self.comp_config(pop)):
            out.append(("kc_" + name, "float"))
        out.append(("spk", "anb_u32"))
        return out

    def comp_config(self, pop) -> dict:
        if self.compensate != "auto":
            return {"compensate": self.compensate}
        names = [v["name"] for v in pop.desc["variables"] if not v["name"].startswith("g_")]
        return {"compensate": names}

    def header_layout(self):
        """The per-slot quantities that a launch copies once into shared
        memory (so that no step reads them from global memory): 64-bit
        offsets, global parameter values and 32-bit entries, each a list of
        (key, global array, index within the slot's row of that array).
        Returns (longs, reals, ints, bytes per slot)."""
        longs, reals, ints = [], [], []
        for pop in self.net.populations:
            k = pop.id
            longs += [(f"goff{k}", f"pop{k}__bgoff", 1, 0), (f"woff{k}", f"pop{k}__bwoff", 1, 0)]
            ints += [(f"n{k}", f"pop{k}__bn", 1, 0), (f"refr{k}", f"pop{k}__brefr", 1, 0)]
            for p in pop.desc["parameters"] + pop.desc["variables"]:
                if p["locality"] == "global":
                    entry = (f"p{k}_{p['name']}", f"pop{k}__{p['name']}", 1, 0)
                    (ints if p.get("ctype") in ("int", "bool") else reals).append(entry)
        for proj in self.net.projections:
            k = proj.id
            longs.append((f"cp{k}", f"proj{k}__bcpoff", 1, 0))
            ints += [(f"wr{k}_0", f"proj{k}__bwr", 2, 0), (f"wr{k}_1", f"proj{k}__bwr", 2, 1)]
        ints += [(f"so{c}", "bt__soff", self.n_arrays, c) for c in range(self.n_arrays)]
        rs = 8 if self.exact else 4
        nbytes = -(-(8 * len(longs) + rs * len(reals) + 4 * len(ints)) // 16) * 16
        return longs, reals, ints, nbytes

    @staticmethod
    def _csize(ct):
        return {"double": 8, "float": 4, "int": 4, "short": 2, "anb_u32": 4}[ct]

    def _instance_bytes(self, net):
        """Shared-memory byte offsets of every array of one instance."""
        offs, total = [], 0
        for pop in net.populations:
            for name, ct in self.smem_arrays[pop.id]:
                n = (pop.size + 31) // 32 if name == "spk" else pop.size
                offs.append(total)
                total += -(-(n * self._csize(ct)) // 16) * 16
        return offs, total

    def _pack(self, costs, sizes, n_bins, limit):
        """Instances -> CTAs: longest-processing-time packing (the next
        costliest instance to the least loaded CTA where it fits) under the
        shared-memory limit. When that needs more CTAs than `n_bins` (more
        than one wave), the instances are placed by decreasing size instead,
        which fills the shared memory more tightly. Returns (CTA of every
        instance, number of CTAs)."""
        def place(order):
            load = [0.0] * n_bins
            used = [0] * n_bins
            where = np.empty(len(costs), dtype=np.int64)
            for i in order:
                cands = [b for b in range(len(load)) if used[b] + sizes[i] <= limit]
                if not cands:
                    load.append(0.0)
                    used.append(0)
                    cands = [len(load) - 1]
                b = min(cands, key=lambda x: (load[x], used[x]))
                load[b] += costs[i]
                used[b] += sizes[i]
                where[i] = b
            return where, len(load)
        where, n = place(np.argsort(-np.asarray(costs), kind="stable"))
        if n > n_bins:
            w2, n2 = place(np.argsort(-np.asarray(sizes), kind="stable"))
            if n2 < n:
                where, n = w2, n2
        return where, n

    # -------------------------------------------------------------- build
    def compile(self):
        from ..generator.batch import BatchGenerator
        self._check()
        nets = self.networks
        nat = self.native
        nat.initialize(self.net.dt)
        self.smem_arrays = {p.id: self._smem_arrays(p) for p in self.net.populations}
        self.array_index = {}
        for pop in self.net.populations:
            for name, _ in self.smem_arrays[pop.id]:
                self.array_index[(pop.id, name)] = len(self.array_index)
        self.n_arrays = len(self.array_index)
        inst = [self._instance_bytes(n) for n in nets]
        # every instance also takes one header slot at the start of its CTA's
        # shared memory
        self.header_bytes = self.header_layout()[3]
        sizes = [b + self.header_bytes for _, b in inst]
        # synapse indices in 32 bits while every projection's concatenation fits
        tot = max([sum(n.projections[j].nb_synapses for n in nets)
                   for j in range(len(self.net.projections))] or [0])
        self.idx_t = "int" if tot + 8 < 2**31 - 1 else "long long"
        # fast mode keeps room for the delivery scratch: 32 warp sums, the
        # list counter, then at least 512 list entries, each with its
        # synapse range in every projection
        isz = 4 if self.idx_t == "int" else 8
        self.entry_bytes = 4 + 2 * isz * len(self.net.projections)
        limit = SMEM_LIMIT - (0 if self.exact else 4 * 36 + 512 * self.entry_bytes + 16)
        if max(sizes) > limit:
            i = int(np.argmax(sizes))
            raise ValueError(f"instance {i} needs {sizes[i]} bytes of shared memory "
                             f"(at most {limit} per CTA in this precision)")
        nnz = [sum(pr.nb_synapses for pr in n.projections) for n in nets]
        neurons = [sum(p.size for p in n.populations) for n in nets]
        costs = [neurons[i] + 0.01 * nnz[i] for i in range(len(nets))]
        sms = self.ctas or (148 if self.dry else device_sm_count(self.device))
        where, n_cta = self._pack(costs, sizes, min(len(nets), sms), limit)
        # slots: instances in CTA order
        order = np.lexsort((np.arange(len(nets)), where))
        self.order = order                      # slot -> instance
        self.slot_of = np.empty(len(nets), dtype=np.int64)
        self.slot_of[order] = np.arange(len(nets))
        cta = np.zeros(n_cta + 1, dtype=np.int32)
        np.cumsum(np.bincount(where, minlength=n_cta), out=cta[1:])
        self.n_cta = n_cta
        self.cta_load = np.bincount(where, weights=costs, minlength=n_cta)
        nat.create("bt__cta", cta)
        # shared-memory offsets: the header slots of the CTA's instances, then
        # the instances' arrays one after the other
        soff = np.empty((len(nets), self.n_arrays), dtype=np.int64)
        for c in range(n_cta):
            base = (cta[c + 1] - cta[c]) * self.header_bytes
            for s in range(cta[c], cta[c + 1]):
                i = order[s]
                soff[s] = np.asarray(inst[i][0], dtype=np.int64) + base
                base += inst[i][1]
        assert soff.max() < SMEM_LIMIT
        nat.create("bt__soff", soff.astype(np.int32))
        self.native_soff, self.cta, self.inst_bytes = soff, cta, [b for _, b in inst]
        self.max_slots = int(np.diff(cta).max())
        # state of the CTA's instances, then (fast mode) the delivery scratch
        # with a list of list_cap entries (a multiple of 4)
        self.smem_state = -(-int(max(np.bincount(where, weights=sizes, minlength=n_cta))) // 16) * 16
        free = SMEM_LIMIT - self.smem_state - 4 * 36
        self.list_cap = 0 if self.exact else int(min(1024, free // self.entry_bytes) // 4 * 4)
        assert self.exact or self.list_cap >= 512
        self.smem = self.smem_state + (0 if self.exact else 4 * 36 + self.list_cap * self.entry_bytes)
        words = np.array([sum((p.size + 31) // 32 for p in n.populations) for n in nets])
        cta_words = np.bincount(where, weights=words, minlength=n_cta)
        if cta_words.max() > 1024:
            raise ValueError("a CTA holds more than 1024 bitmap words (32768 neurons)")
        self._create_populations(order)
        self._create_projections(order)
        self._create_monitors(order)
        gen = BatchGenerator(self)
        self.module = gen.module()
        nat.load_module(self.module.source, self.module.options)
        nat.set_local_kernel(*self.module.local)
        for i, n in enumerate(nets):
            n._backend = _Member(self, i)
            n._compiled = True
        self.compiled = True
        return self

    def _create_populations(self, order):
        nat = self.native
        nets = self.networks
        self.goff, self.woff, self.total_words = {}, {}, {}
        self._initial = {}
        for j, tpl in enumerate(self.net.populations):
            k = tpl.id
            pops = [nets[i].populations[j] for i in order]
            sizes = np.array([p.size for p in pops], dtype=np.int64)
            words = (sizes + 31) // 32
            goff = np.zeros(len(pops), dtype=np.int64)
            np.cumsum(sizes[:-1], out=goff[1:])
            woff = np.zeros(len(pops), dtype=np.int64)
            np.cumsum(words[:-1], out=woff[1:])
            self.goff[k], self.woff[k] = goff, woff
            self.total_words[k] = int(words.sum())
            nat.create(f"pop{k}__bn", sizes.astype(np.int32))
            nat.create(f"pop{k}__bgoff", goff)
            nat.create(f"pop{k}__bwoff", woff)
            for p in tpl.desc["parameters"] + tpl.desc["variables"]:
                name = p["name"]
                dt = np.int32 if p.get("ctype") in ("int", "bool") else self.real
                vals = [np.asarray(q._host[name], dtype=dt).reshape(-1) for q in pops]
                nat.create(f"pop{k}__{name}", np.concatenate(vals))
            for name, ct in self.smem_arrays[k]:
                if name.startswith("kc_"):
                    nat.create(f"pop{k}__{name}", np.zeros(int(sizes.sum()), dtype=np.float32))
            nat.create(f"pop{k}__spk", np.zeros(self.total_words[k], dtype=np.uint32))
            refr = [q.refractory_steps.astype(np.int32) for q in pops]
            nat.create(f"pop{k}__refractory", np.concatenate(refr))
            # per-slot refractory period when uniform over the instance, else -1
            nat.create(f"pop{k}__brefr", np.array(
                [int(r[0]) if r.size and np.all(r == r[0]) else -1 for r in refr], dtype=np.int32))
            nat.create(f"pop{k}__refractory_remaining", np.zeros(int(sizes.sum()), dtype=np.int32))
            nat.create(f"pop{k}__last_spike", np.full(int(sizes.sum()), -10000, dtype=np.int64))
            self._initial[k] = {p["name"]: np.concatenate(
                [np.asarray(q._host[p["name"]]).reshape(-1) for q in pops])
                for p in tpl.desc["parameters"] + tpl.desc["variables"]}

    def _create_projections(self, order):
        nat = self.native
        nets = self.networks
        self.packed = {}
        self.fan_out = {}
        for j, tpl in enumerate(self.net.projections):
            k = tpl.id
            projs = [nets[i].projections[j] for i in order]
            cps, posts, ws, cpoff, wr = [], [], [], [], []
            base, cbase = 0, 0
            fan = []
            for pr in projs:
                # pre-major view, ascending post rank per pre neuron (the
                # reference's CSRC column view, CSRCMatrix.hpp:164-222)
                csc = pr._csr.tocsc()
                csc.sort_indices()
                npre = pr.pre_pop.size
                counts = np.zeros(npre, dtype=np.int64)
                counts[pr.pre_ranks] = np.diff(csc.indptr)
                cp = np.zeros(npre + 1, dtype=np.int64)
                np.cumsum(counts, out=cp[1:])
                cps.append(cp + base)
                posts.append(np.asarray(pr.post_ranks_view, dtype=np.int64)[csc.indices])
                ws.append(np.asarray(csc.data, dtype=np.float64))
                cpoff.append(cbase)
                lo, hi = int(pr.pre_ranks.min()), int(pr.pre_ranks.max())
                wr.append((lo // 32, hi // 32 + 1))
                fan.append(counts)
                base += int(csc.nnz)
                cbase += npre + 1
            self.fan_out[k] = fan
            assert self.idx_t == "long long" or base + 8 < 2**31 - 1
            it = np.int32 if self.idx_t == "int" else np.int64
            nat.create(f"proj{k}__col_ptr", np.concatenate(cps).astype(it))
            nat.create(f"proj{k}__bcpoff", np.asarray(cpoff, dtype=np.int64))
            nat.create(f"proj{k}__bwr", np.asarray(wr, dtype=np.int32).reshape(-1))
            post = np.concatenate(posts) if posts else np.zeros(0, np.int64)
            w = np.concatenate(ws) if ws else np.zeros(0)
            if not self.exact and base:
                # fast mode adds a spike's synapses with shared-memory atomics
                # in any order: deal each row's synapses over the warp's atomic
                # instructions by bank
                row_ptr = np.concatenate([c[:-1] for c in cps] + [np.array([base])])
                perm = bank_interleave(row_ptr, post)
                post, w = post[perm], w[perm]
            # the fast delivery reads aligned groups of 4 synapses: pad the
            # arrays so that the last group stays inside them
            pad = (-post.size) % 4 + 4
            post = np.concatenate([post, np.zeros(pad, np.int64)])
            w = np.concatenate([w, np.zeros(pad)])
            max_post = max(pr.post_pop.size for pr in projs)
            if self.wdtype is BF16 and max_post < 65536:
                # one 32-bit word per synapse: post rank (high half), bfloat16 weight (low half)
                syn = (post.astype(np.uint32) << 16) | to_bf16(w).astype(np.uint32)
                nat.create(f"proj{k}__syn", syn.astype(np.uint32))
                self.packed[k] = True
            else:
                nat.create(f"proj{k}__post", post.astype(np.int32))
                wd = self.wdtype
                nat.create(f"proj{k}__w", to_bf16(w) if wd is BF16 else np.asarray(w, dtype=wd))
                self.packed[k] = False

    def _create_monitors(self, order):
        nat = self.native
        self.mon_cap = {}
        for tpl in self.net.monitors:
            m = tpl.id
            k = tpl.population.id
            per_step = self.total_words[k] * 4
            cap = int(max(1, min(self.net._config.get("monitor_chunk", 100000),
                                 MAX_MONITOR_BYTES // per_step)))
            self.mon_cap[m] = cap
            nat.create(f"mon{m}__on", np.array([1], dtype=np.int32))
            nat.create(f"mon{m}__t0", np.zeros(1, dtype=np.int64))
            nat.create_empty(f"mon{m}__spk", np.uint32, (cap, self.total_words[k]))

    # -------------------------------------------------------------- running
    @property
    def dt(self):
        return self.net.dt

    @property
    def current_step(self) -> int:
        return self.native.get_time()

    def chunk_steps(self) -> int:
        return min(self.mon_cap.values()) if self.mon_cap else 1 << 30

    def begin_chunk(self, t):
        for tpl in self.net.monitors:
            m = tpl.id
            on = any(n.monitors[self._mon_index(tpl)]._recording for n in self.networks)
            self.native.write(f"mon{m}__t0", np.array([t], dtype=np.int64))
            self.native.write(f"mon{m}__on", np.array([1 if on else 0], dtype=np.int32))

    def _mon_index(self, tpl):
        return self.net.monitors.index(tpl)

    def end_chunk(self, t, n):
        """Copy the spike records of the n steps from t into every instance's
        monitors."""
        for tpl in self.net.monitors:
            m = tpl.id
            k = tpl.population.id
            j = self._mon_index(tpl)
            if not any(net.monitors[j]._recording for net in self.networks):
                continue
            tw = self.total_words[k]
            steps, bits = self.native.monitor_decode(f"mon{m}__spk", n, tw, tw * 32)
            woff = self.woff[k]
            slot = np.searchsorted(woff * 32, bits, side="right") - 1
            rank = bits - woff[slot] * 32
            by_slot = np.argsort(slot, kind="stable")
            bounds = np.searchsorted(slot[by_slot], np.arange(len(self.networks) + 1))
            for s in range(len(self.networks)):
                i = int(self.order[s])
                mon = self.networks[i].monitors[j]
                if not mon._recording:
                    continue
                sel = by_slot[bounds[s]:bounds[s + 1]]
                mon._append_spikes(steps[sel].astype(np.int64) + t, rank[sel].astype(np.int64))

    def reset(self):
        """Every instance back to the state it was compiled with (attributes
        as set before compile(), no refractory counters, no spikes pending)
        and the time to step 0; monitors keep what they recorded."""
        nat = self.native
        for k, attrs in self._initial.items():
            for name, arr in attrs.items():
                dtype = nat.arrays[f"pop{k}__{name}"][0]
                nat.write(f"pop{k}__{name}", np.asarray(arr, dtype=dtype))
            for name, _ in self.smem_arrays[k]:
                if name.startswith("kc_"):
                    nat.zero(f"pop{k}__{name}")
            nat.zero(f"pop{k}__spk")
            nat.zero(f"pop{k}__refractory_remaining")
            n = nat.arrays[f"pop{k}__last_spike"][1][0]
            nat.write(f"pop{k}__last_spike", np.full(n, -10000, dtype=np.int64))
        nat.set_time(0)

    def simulate_steps(self, nsteps: int):
        if not self.compiled:
            raise RuntimeError("the batch is not compiled yet")
        nat = self.native
        t = nat.get_time()
        left = int(nsteps)
        cap = self.chunk_steps()
        while left > 0:
            n = min(left, cap)
            self.begin_chunk(t)
            nat.run(n)
            nat.synchronize()
            self.end_chunk(t, n)
            t += n
            left -= n

    def simulate(self, duration: float):
        self.simulate_steps(int(math.ceil(float(duration) / self.dt)))

    def delivered_events(self, spikes_per_instance) -> int:
        """Synaptic events of the given spikes: for instance i, a list of
        (pop position, ranks) pairs; every spike counts its out-degree in
        every projection leaving its population."""
        total = 0
        for i, per_pop in enumerate(spikes_per_instance):
            s = int(self.slot_of[i])
            for pos, ranks in per_pop:
                for j, tpl in enumerate(self.net.projections):
                    if self.net.populations.index(tpl.pre_pop) == pos:
                        total += int(self.fan_out[tpl.id][s][ranks].sum())
        return total

    def close(self):
        for n in self.networks:
            n._backend = None
            n._compiled = False
        self.native.close()
