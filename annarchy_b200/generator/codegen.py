"""CUDA source generation for one compiled network.

Lowers the parser's description dicts (C statements with index
placeholders) into the network's kernels and pairs them with the
hand-written templates of csrc/device/anb_device.cuh.

Step semantics follow the reference's generated core
(ANNarchy/generator/Template/OpenMPBaseTemplate.py:131-484):

    compute_psp of every projection (spikes of the previous step)
    -> update of every population (ODE block: all increments from the old
       state, then the switches, each followed by its min/max bound;
       refractory neurons keep v frozen: the switch of every non-g_
       variable is multiplied by in_ref; ANNarchy/generator/Utils.py:17-265)
    -> spike gather (threshold, reset, last_spike, refractory counter;
       Population/OpenMPGenerator.py:999-1237)
    -> post_event of plastic projections -> record -> t++

Two engines:

* grid  - one kernel per phase over the whole GPU, launched once per step;
          the runtime captures `graph_steps` steps into one CUDA graph.
* local - spiking networks whose state fits in one CTA's shared memory:
          a single kernel keeps the whole state on-chip and loops over the
          steps itself (no launch per step; barriers are __syncthreads).

Precision modes:

* exact (double) - reference operation order, no contraction
                   (--fmad=false): bit-identical to the reference's CPU build.
* fast  (float)  - float state, float or bfloat16 weights, float
                   accumulation with atomics; checked by tolerance.
"""
from __future__ import annotations

import os
import re
from dataclasses import dataclass, field

import numpy as np

from ..core.monitor import array_name, source_name

HERE = os.path.dirname(os.path.abspath(__file__))
DEVICE_HEADER = os.path.join(os.path.dirname(HERE), "csrc", "device", "anb_device.cuh")

BLOCK = 256
MAX_GRID = 148 * 16
PERSISTENT_BLOCK = 1024

CTYPE_OF = {np.dtype(np.float64): "double", np.dtype(np.float32): "float",
            np.dtype(np.int32): "int", np.dtype(np.int64): "long long",
            np.dtype(np.uint32): "anb_u32", np.dtype(np.uint16): "anb_bf16",
            np.dtype(np.uint8): "unsigned char"}


def compensated_vars(pop, exact: bool, config: dict) -> list:
    """ODE variables whose explicit-Euler switch is Kahan-compensated
    (single precision only): the rounding error of every `x += dt*_x` is
    carried in anb_kc_x and added back at the next step. config
    "compensate": True (every local ODE variable), False, "auto" (all but the
    conductances g_*, whose increments only decay them) or a list of
    variable names."""
    comp = config.get("compensate", True)
    if exact or not comp:
        return []
    names = [v["name"] for v in pop.desc["variables"]
             if v.get("switch") and v.get("method") != "event-driven"
             and v["name"] in pop.desc["local"]]
    if comp == "auto":
        return [n for n in names if not n.startswith("g_")]
    return names if comp is True else [n for n in names if n in comp]


def global_equations(pop) -> list:
    """The population-level (global) variables of a population's neuron that
    have an equation, in declaration order."""
    glob = set(pop.desc.get("global", []) or [])
    return [v for v in pop.desc["variables"]
            if v["name"] in glob and v.get("cpp") and v.get("method") != "event-driven"]


def syn_local_names(proj) -> list:
    """Per-synapse arrays of a plastic spiking projection: w, the other local
    variables, the local parameters (one value per synapse, as the
    reference stores them) and what the pre/post-spike statements assign."""
    names = ["w"] + [v["name"] for v in proj.desc["variables"] + proj.desc["parameters"]
                     if v["locality"] == "local" and v["name"] != "w"]
    for v in proj.desc.get("pre_spike", []) + proj.desc.get("post_spike", []):
        if v["name"] not in names and v["name"] not in ("w", "g_target"):
            names.append(v["name"])
    return names


def trace_layout(proj, exact: bool):
    """Fast-mode plastic spiking projections keep their per-synapse state
    (w, the other local variables, the last event step) packed in one record
    per synapse, so a synapse reached through the inverse index costs one
    scattered sector instead of one per variable. Returns (field names,
    record bytes) or None when the variables stay separate arrays."""
    if exact or not proj.plastic or proj.synapse_type.type != "spike":
        return None
    if CodeGenerator.continuous_update(proj):
        return None                 # the per-step update walks separate arrays
    names = syn_local_names(proj)
    nbytes = 4 * (len(names) + 1)
    nbytes = 8 if nbytes <= 8 else -(-nbytes // 16) * 16
    return names, nbytes


def grid_for(n: int, block: int = BLOCK) -> int:
    return max(1, min(MAX_GRID, (n + block - 1) // block))


def list_grid(n_pre: int, chunks: int, block: int = BLOCK) -> int:
    """CTAs of a kernel whose warps take (spike, chunk of 32 synapses) work
    items from a spike list: one warp per item while at most 1/64 of the
    n_pre neurons spike in a step, and never more than one resident wave
    (148 SMs x 8 CTAs); a busier step loops over the items."""
    return max(1, min(148 * 8, -(-(n_pre * chunks * 32) // (64 * block))))


def float_literals(code: str) -> str:
    """Suffix floating literals with f (single-precision modules), like the
    reference's float precision mode (ANNarchy/parser/Equation.py:172-197)."""
    return re.sub(r"(?<![\w.])(\d+\.\d+(?:[eE][-+]?\d+)?)(?![\w.])", r"\1f", code)


@dataclass
class Module:
    source: str
    options: list
    engine: str
    plan: list = field(default_factory=list)           # [(kernel, grid, block, smem)]
    local: tuple | None = None                         # (kernel, grid, block, smem)
    kernels: list = field(default_factory=list)
    stops: list = field(default_factory=list)          # [(pop id, kernel, grid, block, all)]


class CodeGenerator:
    def __init__(self, compiled):
        self.c = compiled                  # CompiledNetwork (arrays, precision, layout)
        self.net = compiled.net
        self.exact = compiled.exact
        self.real = "double" if self.exact else "float"
        self.decls: dict[str, str] = {}
        self.types: dict[str, str] = {}

    # ------------------------------------------------------------------ utils
    def ptr(self, name: str) -> str:
        """C expression of the device pointer of array `name` (declares it)."""
        dtype = self.c.native.arrays[name][0]
        self.decls[name] = CTYPE_OF[np.dtype(dtype)]
        return "anb_p_" + name

    # history rings (synaptic delays)
    def slots(self, pop) -> int:
        return self.c.slots.get(pop.id, 1)

    def spk_at(self, pop, step: str) -> str:
        """Spike bitmap of the population at time step `step` (a C
        expression); the slot of that step when the population keeps a ring."""
        spk = self.ptr(f"pop{pop.id}__spk")
        R = self.slots(pop)
        if R == 1:
            return spk
        return f"({spk} + (size_t)anb_ring_slot({step}, {R}) * {(pop.size + 31) // 32})"

    def delayed(self, proj) -> bool:
        """The projection reads its pre-synaptic output through a delay ring."""
        return proj.max_delay > 1

    def atomic_psp(self, proj) -> bool:
        """The projection's transmission kernel only adds into g with atomics
        (and touches its own synapses): fast mode, spike lists or the bitmap
        scatter; not the warp-per-row gathers."""
        if self.exact or proj.synapse_type.type != "spike":
            return False
        if proj._delay_steps is not None:
            return False
        if proj.plastic:
            return self.c.spike_lists and not self.delayed(proj)
        return True

    def pre_spk(self, proj) -> str:
        if self.delayed(proj) and proj._delay_steps is None:
            return self.spk_at(proj.pre_pop, f"t - {self.ptr(f'proj{proj.id}__delay')}[0]")
        return self.spk_at(proj.pre_pop, "t - 1")

    def pre_rate(self, proj) -> str:
        k = proj.pre_pop.id
        if self.delayed(proj) and proj._delay_steps is None:
            R, S = self.slots(proj.pre_pop), self.c.ring_stride(proj.pre_pop)
            return (f"({self.ptr(f'pop{k}___delayed_r')} + (size_t)anb_ring_slot(t - "
                    f"{self.ptr(f'proj{proj.id}__delay')}[0], {R}) * {S})")
        return self.ptr(f"pop{k}__r")

    def typed(self, code: str) -> str:
        code = code.replace("double ", self.real + " ")
        return code if self.exact else float_literals(code)

    @staticmethod
    def fill(code: str, local="", glob="", semi="", pre_prefix="", pre_index="", post_prefix="",
             post_index="") -> str:
        return code % {"local_index": local, "global_index": glob, "semiglobal_index": semi,
                       "pre_prefix": pre_prefix, "pre_index": pre_index,
                       "post_prefix": post_prefix, "post_index": post_index}

    # --------------------------------------------------------------- neurons
    def compensated(self, pop) -> list:
        return compensated_vars(pop, self.exact, self.c.net._config)

    def _neuron_body(self, pop, src_of, masked: bool) -> tuple[str, list]:
        """Statements updating one neuron; locals are C variables named after
        the attributes. Returns (code, names of modified attributes)."""
        comp = set(self.compensated(pop))
        desc = pop.desc
        local = set(desc["local"])
        blocks = []
        is_ode = False
        for v in desc["variables"]:
            if v.get("cpp", "") == "" or v.get("method") == "event-driven":
                continue
            if v["name"] not in local:
                continue            # population-level: _global_update
            if v.get("switch"):
                if is_ode:
                    blocks[-1][1].append(v)
                else:
                    blocks.append(("ode", [v]))
                    is_ode = True
            else:
                if is_ode or not blocks:
                    blocks.append(("non-ode", [v]))
                    is_ode = False
                else:
                    blocks[-1][1].append(v)
        lines, modified = [], []

        def bounds(v):
            out = []
            for b, val in v.get("bounds", {}).items():
                if b in ("min", "max"):
                    op = "<" if b == "min" else ">"
                    val = self.fill(str(val))
                    out.append(f"if ({v['name']} {op} {val}) {v['name']} = {val};")
            return out

        for kind, vs in blocks:
            if kind == "ode":
                for v in vs:
                    lines.append(self.typed(self.fill(v["cpp"])))
                for v in vs:
                    sw = self.fill(v["switch"])
                    if masked and not v["name"].startswith("g_"):
                        sw = sw.replace(";", "* in_ref;")
                    if v["name"] in comp:
                        x = v["name"]
                        inc = sw.split("+=", 1)[1].strip().rstrip(";")
                        sw = (f"{{ const {self.real} anb_y = ({inc}) - anb_kc_{x}; "
                              f"const {self.real} anb_tx = {x} + anb_y; "
                              f"anb_kc_{x} = (anb_tx - {x}) - anb_y; {x} = anb_tx; }}")
                    lines.append(sw)
                    lines += [self.typed(b) for b in bounds(v)]
                    modified.append(v["name"])
            else:
                for v in vs:
                    code = self.typed(self.fill(v["cpp"]))
                    if masked and not v["name"].startswith("g_"):
                        code = "if (in_ref) { " + code + " }"
                    lines.append(code)
                    lines += [self.typed(b) for b in bounds(v)]
                    modified.append(v["name"])
        return "\n".join(lines), modified

    def _reciprocals(self, pop):
        """Global real parameters used as divisors: in fast mode their
        reciprocal is computed once and the division becomes a multiply."""
        if self.exact:
            return []
        names = [p["name"] for p in pop.desc["parameters"]
                 if p["locality"] == "global" and p.get("ctype") not in ("int", "bool")]
        code = " ".join(v.get("cpp", "") or "" for v in pop.desc["variables"])
        return [n for n in names if re.search(r"/" + re.escape(n) + r"(?![\w\[])", code)]

    def _use_reciprocals(self, pop, code: str) -> str:
        for n in self._reciprocals(pop):
            code = re.sub(r"/" + re.escape(n) + r"(?![\w\[])", "*anb_inv_" + n, code)
        return code

    def _globals_preamble(self, pop, src) -> str:
        out = []
        evolving = {v["name"] for v in global_equations(pop)}
        for p in pop.desc["parameters"] + pop.desc["variables"]:
            if p["locality"] == "global":
                ct = "int" if p.get("ctype") in ("int", "bool") else self.real
                const = "" if p["name"] in evolving else "const "
                out.append(f"{const}{ct} {p['name']} = {src(p['name'])}[0];")
        for op in pop._globalops:
            name = "_" + op["function"] + "_" + op["variable"]
            out.append(f"const {self.real} {name} = {src(name)}[0];")
        for n in self._reciprocals(pop):
            out.append(f"const {self.real} anb_inv_{n} = ({self.real})1 / {n};")
        for v in pop.desc["variables"]:
            pl = v.get("pre_loop") or {}
            if pl:
                out.append(self.typed(f"const double {pl['name']} = {self.fill(pl['value'])};"))
        return "\n    ".join(out)

    _DRAW_FN = {"Uniform": "anb_draw_uniform", "Normal": "anb_draw_normal",
                "LogNormal": "anb_draw_lognormal", "Exponential": "anb_draw_exponential",
                "DiscreteUniform": "anb_draw_discrete_uniform"}

    def _random_draws(self, pop, which: str = "all") -> str:
        """This step's draws of the random distributions in the neuron's
        equations: Philox4x32-10 keyed by the network's seed, counter (neuron,
        step, population and distribution); one draw per neuron, or one per
        population (same counter in every thread) for a global variable.
        `which`: "all", "local" or "global" draws."""
        out = []
        for k, rd in enumerate(pop.desc.get("random_distributions", [])):
            if which != "all" and (rd["locality"] == "local") != (which == "local"):
                continue
            idx = "(unsigned)anb_i" if rd["locality"] == "local" else "0xFFFFFFFFu"
            args = ", ".join(f"({self.real})({self.typed(a)})" for a in rd["args"])
            out.append(f"const {self.real} {rd['name']} = {self._DRAW_FN[rd['dist']]}<{self.real}>("
                       f"{self.ptr('rng_seed')}, {(pop.id << 8) | k}u, t, {idx}, {args});")
        return "\n".join(out)

    def _locals(self, pop):
        return [p["name"] for p in pop.desc["parameters"] + pop.desc["variables"]
                if p["locality"] == "local"]

    def _fused_spike_records(self, pop) -> str:
        """Grid engine: lane 0 of every warp also writes its bitmap word into
        the ring of each spike monitor of the population (no record kernel)."""
        out = ""
        for mon in self.net.monitors:
            if mon.population is not pop or "spike" not in mon.variables:
                continue
            ml = self.c.mon_layout[mon.id]
            m = mon.id
            out += f"""
          if (anb_mon_on{m}) {{
            const long long anb_slot = t - anb_mon_t0{m};
            if (anb_slot >= 0 && anb_slot < {ml['cap_spike']})
              {self.ptr(f'mon{m}__spk')}[anb_slot * {ml['words']} + (anb_i >> 5)] = anb_m;
            else
              anb_report({self.ptr('err')}, ANB_DEVERR_MONITOR_OVERFLOW);
          }}"""
        return out

    def _fused_record_preamble(self, pop) -> str:
        out = []
        for mon in self.net.monitors:
            if mon.population is pop and "spike" in mon.variables:
                m = mon.id
                out.append(f"const int anb_mon_on{m} = {self.ptr(f'mon{m}__on')}[0];")
                out.append(f"const long long anb_mon_t0{m} = {self.ptr(f'mon{m}__t0')}[0];")
        return "\n    ".join(out)

    def _global_update(self, pop) -> str:
        """The population-level equations of step t, evaluated before the
        neurons' (the reference's global step, ANNarchy/generator/Population/
        CUDAGenerator.py: the global kernel launched before the local one) by
        every thread on the same loaded values, so each has this step's
        values without a grid barrier; consecutive ODEs form one block (all
        increments, then the switches and bounds)."""
        lines, group = [], []

        def flush():
            for v in group:
                lines.append(self.typed(self.fill(v["cpp"])))
            for v in group:
                lines.append(self.typed(self.fill(v["switch"])))
                lines.extend(self._bound_lines(v))
            group.clear()

        for v in global_equations(pop):
            if v.get("switch"):
                group.append(v)
                continue
            flush()
            lines.append(self.typed(self.fill(v["cpp"])))
            lines.extend(self._bound_lines(v))
        flush()
        draws = self._random_draws(pop, "global")
        return "\n    ".join(([draws] if draws else []) + lines)

    def _bound_lines(self, v) -> list:
        out = []
        for b, val in v.get("bounds", {}).items():
            if b in ("min", "max"):
                op = "<" if b == "min" else ">"
                val = self.fill(str(val))
                out.append(self.typed(f"if ({v['name']} {op} {val}) {v['name']} = {val};"))
        return out

    def neuron_update(self, pop, *, local_engine=False, smem=None, cluster=None,
                      ballot_hook=None, size=None, gsrc=None, refractory=None) -> str:
        """Update (+ spike gather) of one population for step t.

        grid: grid-stride over all neurons, state in global memory; local:
        one CTA over all neurons, state in shared memory (`smem`); cluster:
        this CTA's slice [anb_base, anb_base + anb_cnt), shared-memory state
        indexed by the local index anb_q and the conductance increments of
        the step (`cluster` = {target: increment buffer}) added first.
        `size` (a C expression) and `gsrc` (attribute name -> C pointer
        expression) override the population's size and global arrays; a
        `ballot_hook` replaces the bitmap store of the local engine;
        `refractory` is a C expression of the refractory period (in steps)
        that replaces the per-neuron array."""
        spiking = pop.neuron_type.type == "spike"
        masked = spiking and pop._has_refractory
        geq = bool(global_equations(pop))
        if geq and (smem or cluster is not None or local_engine or size is not None):
            raise NotImplementedError(f"{pop.name}: population-level variables with equations run "
                                      "on the grid engine only")
        body, modified = self._neuron_body(pop, None, masked)
        body = self._use_reciprocals(pop, body)
        draws = self._random_draws(pop, "local" if geq else "all")
        if draws:
            body = draws + "\n" + body
        # only the local attributes the update reads or writes are loaded
        used = body
        if spiking:
            used += " " + pop.desc["spike"]["spike_cond"] + " " + " ".join(
                r["cpp"] for r in pop.desc["spike"]["spike_reset"])
        names = [n for n in self._locals(pop) if re.search(rf"\b{re.escape(n)}\b", used)]
        k = pop.id

        if gsrc is None:
            def gsrc(name):
                return self.ptr(f"pop{k}__{name}")

        grid_path = not smem and cluster is None and not local_engine
        loads, stores = [], []
        hoist = []          # grid path: (ctype, variable, array) loaded for K neurons at once
        sidx = "anb_q" if cluster is not None else "anb_i"
        for name in names:
            ct = "int" if pop._ctype.get(name) in ("int", "bool") else self.real
            on_chip = bool(smem and name in smem)
            src = smem[name] if on_chip else gsrc(name)
            idx = sidx if on_chip else "anb_i"
            loads.append(f"{ct} {name} = {src}[{idx}];")
            hoist.append((ct, name, src))
            if name in modified or (spiking and any(r["name"] == name for r in
                                                    pop.desc["spike"]["spike_reset"])):
                stores.append(f"{src}[{idx}] = {name};")
        if cluster is not None:
            for target, dg in cluster.items():
                loads.append(f"g_{target} += {dg}[anb_q]; {dg}[anb_q] = 0.f;")
        comp = self.compensated(pop)
        for x in comp:
            on_chip = bool(smem and ("kc_" + x) in smem)
            src = smem["kc_" + x] if on_chip else gsrc("kc_" + x)
            idx = sidx if on_chip else "anb_i"
            loads.append(f"{self.real} anb_kc_{x} = {src}[{idx}];")
            hoist.append((self.real, f"anb_kc_{x}", src))
            stores.append(f"{src}[{idx}] = anb_kc_{x};")
        if pop.neuron_type.type == "rate":
            for t in pop.targets:
                src = gsrc("_sum_" + t)
                loads.append(f"const {self.real} _sum_{t} = {src}[anb_i];")
                hoist.append((f"const {self.real}", f"_sum_{t}", src))
                stores.append(f"{src}[anb_i] = ({self.real})0;")
                if grid_path:
                    # kept for Population.sum(target) (the sums are consumed here)
                    stores.append(f"{gsrc('_last_sum_' + t)}[anb_i] = _sum_{t};")
        spike_code = ""
        if spiking:
            rr_src = smem["refractory_remaining"] if smem else gsrc("refractory_remaining")
            rr_idx = sidx if smem else "anb_i"
            cond = self.typed(self.fill(pop.desc["spike"]["spike_cond"]))
            resets = "\n          ".join(self.typed(self.fill(r["cpp"]))
                                         for r in pop.desc["spike"]["spike_reset"])
            for r in pop.desc["spike"]["spike_reset"]:
                if r["name"] in comp:
                    resets += f"\n          anb_kc_{r['name']} = ({self.real})0;"
            if masked:
                loads.append(f"int refractory_remaining = {rr_src}[{rr_idx}];")
                hoist.append(("int", "refractory_remaining", rr_src))
                loads.append("const int in_ref = (refractory_remaining > 0) ? 0 : 1;")
                refr_dec = "refractory_remaining -= (1 - in_ref);"
                guard = f"(in_ref != 0) && ({cond})"
                if refractory is not None:
                    refr_set = f"refractory_remaining = {refractory};"
                elif smem and "refractory" in smem:
                    refr_set = f"refractory_remaining = {smem['refractory']}[{rr_idx}];"
                else:
                    refr_set = f"refractory_remaining = {gsrc('refractory')}[anb_i];"
                stores.append(f"{rr_src}[{rr_idx}] = refractory_remaining;")
            else:
                refr_dec, guard, refr_set = "", f"({cond})", ""
            spike_code = f"""{refr_dec}
        if ({guard}) {{
          {resets}
          anb_spiked = true;
          {gsrc('last_spike')}[anb_i] = t;
          {refr_set}
        }}"""
        if spiking and ballot_hook is None:
            spk_dst = smem.get("spk") if smem else (self.spk_at(pop, "t") if grid_path else gsrc("spk"))
        else:
            spk_dst = None
        if grid_path and pop.neuron_type.type == "rate" and self.slots(pop) > 1:
            # this step's rate into the history ring (the reference's update_delay)
            rv = "r" if "r" in names else f"{gsrc('r')}[anb_i]"
            stores.append(f"{self.ptr(f'pop{k}___delayed_r')}[(size_t)anb_ring_slot(t, {self.slots(pop)}) * "
                          f"{self.c.ring_stride(pop)} + anb_i] = {rv};")
        ballot = ""
        listed = (spiking and cluster is None and not local_engine and not self.exact
                  and self.c.spike_lists)
        recs = "" if (local_engine or cluster is not None) else self._fused_spike_records(pop)
        if recs:
            recs = f"""
        if ((threadIdx.x & 31) == 0 && anb_i < anb_n) {{{recs}
        }}"""
        if listed:
            spl, spn = gsrc("spl"), gsrc("spn")
            ballot = f"""
      {{
        const anb_u32 anb_m = __ballot_sync(0xffffffffu, anb_spiked);
        if ((threadIdx.x & 31) == 0 && anb_i < anb_n) {spk_dst}[anb_i >> 5] = anb_m;{recs}
        if (anb_m) {{   // append to this step's spike list (warp-aggregated)
          int anb_pos = 0;
          if ((threadIdx.x & 31) == 0) anb_pos = atomicAdd(&{spn}[t & 1], __popc(anb_m));
          anb_pos = __shfl_sync(0xffffffffu, anb_pos, 0);
          if (anb_spiked)
            {spl}[(t & 1) * (long long)anb_n + anb_pos + __popc(anb_m & ((1u << (threadIdx.x & 31)) - 1u))] = anb_i;
        }}
      }}"""
        elif spiking and ballot_hook is not None:
            ballot = ballot_hook
        elif spiking:
            widx, lim = ("anb_q", "anb_cnt") if cluster is not None else ("anb_i", "anb_n")
            ballot = f"""
      {{
        const anb_u32 anb_m = __ballot_sync(0xffffffffu, anb_spiked);
        if ((threadIdx.x & 31) == 0 && {widx} < {lim}) {spk_dst}[{widx} >> 5] = anb_m;{recs}
      }}"""
        nl = "\n        "
        if cluster is not None:
            k = pop.id
            return f"""
    {{  // population {pop.name}: this CTA's slice
      const int anb_n = {pop.size};
      const int anb_base = anb_base{k}, anb_cnt = anb_cnt{k};
      for (int anb_q0 = 0; anb_q0 < anb_cnt; anb_q0 += blockDim.x) {{
        const int anb_q = anb_q0 + threadIdx.x;
        const int anb_i = anb_base + anb_q;
        bool anb_spiked = false;
        if (anb_q < anb_cnt) {{
        {nl.join(loads)}
        {body.replace(chr(10), nl)}
        {spike_code}
        {nl.join(stores)}
        }}{ballot}
      }}
    }}"""
        first = 0
        K = self.neurons_per_thread(pop) if grid_path else 1
        if grid_path and K > 1:
            if pop.id in getattr(self.c, "owned", {}):
                first, size = self.c.owned[pop.id]
            derived = [ln for ln in loads if not any(ln == f"{ct} {nm} = {src}[anb_i];"
                                                     for ct, nm, src in hoist)]
            arrays = nl.join(f"{ct.replace('const ', '')} anb_h_{nm}[{K}];" for ct, nm, _ in hoist)
            fetch = nl.join(f"  anb_h_{nm}[anb_k] = {src}[anb_j];" for _, nm, src in hoist)
            unpack = nl.join(f"{ct} {nm} = anb_h_{nm}[anb_k];" for ct, nm, _ in hoist)
            return f"""
    {{  // population {pop.name}: update{' and spike gather' if spiking else ''}, {K} neurons per
        // thread and pass with all their loads issued first
      const int anb_n = {size if size is not None else pop.size};
      for (int anb_base0 = {first} + blockIdx.x * blockDim.x * {K}; anb_base0 < anb_n;
           anb_base0 += gridDim.x * blockDim.x * {K}) {{
        {arrays}
#pragma unroll
        for (int anb_k = 0; anb_k < {K}; ++anb_k) {{
          const int anb_j = anb_base0 + anb_k * blockDim.x + threadIdx.x;
          if (anb_j < anb_n) {{
          {fetch}
          }}
        }}
#pragma unroll
        for (int anb_k = 0; anb_k < {K}; ++anb_k) {{
        const int anb_base = anb_base0 + anb_k * blockDim.x;
        const int anb_i = anb_base + threadIdx.x;
        bool anb_spiked = false;
        if (anb_i < anb_n) {{
        {unpack}
        {nl.join(derived)}
        {body.replace(chr(10), nl)}
        {spike_code}
        {nl.join(stores)}
        }}{ballot}
        }}
      }}
    }}"""
        if local_engine:
            loop = "for (int anb_base = 0; anb_base < anb_n; anb_base += blockDim.x)"
        else:
            # a sharded network updates the owned slice [first, anb_n) only
            if grid_path and pop.id in getattr(self.c, "owned", {}):
                first, size = self.c.owned[pop.id]
            loop = (f"for (int anb_base = {first} + blockIdx.x * blockDim.x; anb_base < anb_n; "
                    "anb_base += gridDim.x * blockDim.x)")
        return f"""
    {{  // population {pop.name}: update{' and spike gather' if spiking else ''}
      const int anb_n = {size if size is not None else pop.size};
      {loop} {{
        const int anb_i = anb_base + threadIdx.x;
        bool anb_spiked = false;
        if (anb_i < anb_n) {{
        {nl.join(loads)}
        {body.replace(chr(10), nl)}
        {spike_code}
        {nl.join(stores)}
        }}{ballot}
      }}
    }}"""

    @staticmethod
    def neurons_per_thread(pop) -> int:
        """Neurons one thread updates per pass of the grid engine's update
        kernel: large populations issue the loads of several neurons before
        computing any, so that enough bytes are in flight per thread."""
        return 4 if pop.size >= (1 << 18) else (2 if pop.size >= (1 << 16) else 1)

    def pop_kernel(self, pop) -> str:
        k = pop.id
        preamble = self._globals_preamble(pop, lambda n: self.ptr(f"pop{k}__{n}"))
        rp = self._fused_record_preamble(pop)
        if rp:
            preamble += "\n    " + rp
        geq = global_equations(pop)
        store = ""
        if geq:
            preamble += "\n    " + self._global_update(pop)
            # the last CTA to finish (every other one has read the old values)
            # stores the new ones
            writes = " ".join(f"{self.ptr(f'pop{k}__{v['name']}')}[0] = {v['name']};" for v in geq)
            store = f"""
    __syncthreads();
    if (threadIdx.x == 0) {{
      __threadfence();
      if (atomicAdd({self.ptr(f'pop{k}__gtick')}, 1u) == gridDim.x - 1) {{
        *{self.ptr(f'pop{k}__gtick')} = 0u;
        {writes}
      }}
    }}"""
        dt_t = "double" if self.exact else "float"
        return f"""
extern "C" __global__ void __launch_bounds__({BLOCK}) pop{k}_step() {{
    const long long t = *{self.ptr('t')};
    const {dt_t} dt = ({dt_t})(*{self.ptr('dt')});
    {preamble}
{self.neuron_update(pop)}{store}
}}
"""

    def globalops_kernel(self, pop) -> str:
        """The population's reductions after this step's update
        (ANNarchy/generator/Template/GlobalOperationTemplate.py): in double
        precision one thread in index order as the reference (the sum starts
        from element 0; mean = sum / n, norm2 = sqrt of the sum of squares);
        in single precision one CTA's tree reduction."""
        k = pop.id
        n = pop.size
        R = self.real
        outs = []
        for op in pop._globalops:
            f, v = op["function"], op["variable"]
            outs.append((f, self.ptr(f"pop{k}__{v}"), self.ptr(f"pop{k}___{f}_{v}")))
        if self.exact:
            body = []
            for f, src, dst in outs:
                first = {"norm1": f"fabs({src}[0])", "norm2": f"{src}[0] * {src}[0]"}.get(f, f"{src}[0]")
                step = {"max": f"if ({src}[i] > s) s = {src}[i];",
                        "min": f"if ({src}[i] < s) s = {src}[i];",
                        "mean": f"s += {src}[i];",
                        "norm1": f"s += fabs({src}[i]);",
                        "norm2": f"s += {src}[i] * {src}[i];"}[f]
                fin = {"mean": f"s / ({R}){n}", "norm2": "sqrt(s)"}.get(f, "s")
                body.append(f"{{ {R} s = {first}; for (int i = 1; i < {n}; ++i) {{ {step} }} {dst}[0] = {fin}; }}")
            code = "\n      ".join(body)
            return f"""
extern "C" __global__ void __launch_bounds__(32) pop{k}_globalops() {{
    if (blockIdx.x == 0 && threadIdx.x == 0) {{
      {code}
    }}
}}
"""
        parts = []
        for idx, (f, src, dst) in enumerate(outs):
            init = {"max": "__int_as_float(0xff800000)",
                    "min": "__int_as_float(0x7f800000)"}.get(f, "0.f")
            acc = {"max": "fmaxf(s, x)", "min": "fminf(s, x)", "mean": "s + x",
                   "norm1": "s + fabsf(x)", "norm2": "s + x * x"}[f]
            comb = {"max": "fmaxf(s, o)", "min": "fminf(s, o)"}.get(f, "s + o")
            fin = {"mean": f"s / (float){n}", "norm2": "sqrtf(s)"}.get(f, "s")
            parts.append(f"""
    {{
      float s = {init};
      for (int i = threadIdx.x; i < {n}; i += blockDim.x) {{ const float x = (float){src}[i]; s = {acc}; }}
      for (int d = 16; d > 0; d >>= 1) {{ const float o = __shfl_xor_sync(0xffffffffu, s, d); s = {comb}; }}
      if ((threadIdx.x & 31) == 0) anb_red[threadIdx.x >> 5] = s;
      __syncthreads();
      if (threadIdx.x < 32) {{
        s = threadIdx.x < (blockDim.x >> 5) ? anb_red[threadIdx.x] : {init};
        for (int d = 16; d > 0; d >>= 1) {{ const float o = __shfl_xor_sync(0xffffffffu, s, d); s = {comb}; }}
        if (threadIdx.x == 0) {dst}[0] = {fin};
      }}
      __syncthreads();
    }}""")
        return f"""
extern "C" __global__ void __launch_bounds__(1024) pop{k}_globalops() {{
    __shared__ float anb_red[32];
    if (blockIdx.x != 0) return;{''.join(parts)}
}}
"""

    def stop_kernel(self, pop) -> tuple[str, bool]:
        """Stop condition of a population for simulate_until (the reference
        compiles it as PopStruct::stop_condition(),
        ANNarchy/generator/Population/CUDAGenerator.py:836-917, parsed by
        ANNarchy/parser/Extraction.py:927-947): "<condition> : any" (the
        default) holds when a neuron satisfies it, ": all" when every neuron
        does; "spiked" tests the spikes of the step just finished. The kernel
        writes the device step into stop_flags[pop] when a neuron satisfies
        the condition (any) or fails it (all). Returns (source, all)."""
        from ..parser.equation import Statement
        eq, _, flags = pop.stop_condition.partition(":")
        mode_all = "all" in flags.split()
        k = pop.id
        eq = eq.strip()
        if eq.replace(" ", "") == "spiked":
            loads = ""
            cond = f"(({self.spk_at(pop, '(t - 1)')}[anb_i >> 5] >> (anb_i & 31)) & 1u) != 0u"
        else:
            code = self.typed(self.fill(Statement("stop_cond", eq, pop.desc).parse()))
            names = [n for n in self._locals(pop) if re.search(rf"\b{re.escape(n)}\b", code)]
            loads = " ".join(
                f"const {'int' if pop._ctype.get(n) in ('int', 'bool') else self.real} {n} = "
                f"{self.ptr(f'pop{k}__{n}')}[anb_i];" for n in names)
            cond = code
        test = f"!({cond})" if mode_all else f"({cond})"
        dt_t = "double" if self.exact else "float"
        preamble = self._globals_preamble(pop, lambda n: self.ptr(f"pop{k}__{n}"))
        src = f"""
extern "C" __global__ void __launch_bounds__({BLOCK}) pop{k}_stop() {{
    const long long t = *{self.ptr('t')};
    const {dt_t} dt = ({dt_t})(*{self.ptr('dt')});
    (void)dt;
    {preamble}
    bool anb_hit = false;
    for (int anb_i = blockIdx.x * blockDim.x + threadIdx.x; anb_i < {pop.size};
         anb_i += gridDim.x * blockDim.x) {{
      {loads}
      if ({test}) anb_hit = true;
    }}
    if (__ballot_sync(0xffffffffu, anb_hit) != 0u && (threadIdx.x & 31) == 0)
      atomicMax({self.ptr('stop_flags')} + {k}, t);
}}
"""
        return src, mode_all

    # ------------------------------------------------- rate-coded learning
    @staticmethod
    def custom_psp(proj) -> bool:
        """A rate-coded synapse whose psp is not w * pre.r, or whose
        operation over the synapses is not a sum."""
        if proj.synapse_type.type != "rate":
            return False
        if getattr(proj.synapse_type, "operation", "sum") != "sum":
            return True
        eq = proj.desc.get("psp", {}).get("eq", "w*pre.r").replace(" ", "")
        return eq not in ("w*pre.r", "pre.r*w")

    def custom_psp_kernel(self, proj) -> str:
        """Weighted sum with the synapse's own psp expression and operation
        (ANNarchy/generator/Projection/OpenMP/CSR.py:177-253): thread per
        post row over its synapses in stored (ascending pre rank) order -
        the terms added (sum), their largest or smallest starting from the
        first synapse's (max, min), or their sum over the row's synapse
        count (mean) - then added to the target's sum."""
        k = proj.id
        lay = self.c.layout[k]
        a, b = proj.pre_pop, proj.post_pop
        desc = proj.desc
        p = lambda n: self.ptr(f"proj{k}__{n}")
        code = self.typed(self.fill(desc["psp"]["cpp"], local="[j]", semi="[anb_row]",
                                    pre_prefix="anb_pre_", pre_index="[anb_col[j]]",
                                    post_prefix="anb_post_", post_index="[anb_post]"))
        expr = code.strip().rstrip(";")
        decl = [f"const {self.real} {q['name']} = {p(q['name'])}[0];"
                for q in desc["parameters"] + desc["variables"] if q["locality"] == "global"]
        for q in desc["parameters"] + desc["variables"]:
            if q["locality"] in ("local", "semiglobal") and q["name"] != "w":
                decl.append(f"const {self.real}* __restrict__ {q['name']} = {p(q['name'])};")
        decl.append(f"const {self.real}* __restrict__ w = {p('w')};")
        for prefix, pop in (("anb_pre_", a), ("anb_post_", b)):
            for n in sorted(set(re.findall(prefix + r"(\w+)\[", expr))):
                if n not in pop._host:
                    raise NotImplementedError(f"{proj.name}: {prefix[4:-1]}.{n} is not an attribute "
                                              f"of {pop.name}")
                ct = "int" if pop._ctype.get(n) in ("int", "bool") else self.real
                decl.append(f"const {ct}* __restrict__ {prefix}{n} = {self.ptr(f'pop{pop.id}__{n}')};")
        decl += self._globalop_refs(proj, expr)
        dt_t = "double" if self.exact else "float"
        sum_ = self.ptr(f"pop{b.id}___sum_{proj.target}")
        rp_t = lay["idx_t"]
        nl = "\n    "
        op = getattr(proj.synapse_type, "operation", "sum")
        beg, end = "anb_rp[anb_row]", "anb_rp[anb_row + 1]"
        if op in ("max", "min"):
            cmp = ">" if op == "max" else "<"
            reduce = (f"{self.real} anb_s = ({self.real})0;\n      if ({beg} < {end}) {{\n"
                      f"        {{ const {rp_t} j = {beg}; anb_s = {expr}; }}\n"
                      f"        for ({rp_t} j = {beg} + 1; j < {end}; ++j) {{\n"
                      f"          const {self.real} anb_v = {expr};\n"
                      f"          if (anb_v {cmp} anb_s) anb_s = anb_v;\n        }}\n      }}")
        else:
            reduce = (f"{self.real} anb_s = ({self.real})0;\n"
                      f"      for ({rp_t} j = {beg}; j < {end}; ++j) anb_s += {expr};")
            if op == "mean":
                reduce += f"\n      if ({end} > {beg}) anb_s /= ({self.real})({end} - {beg});"
        return f"""
extern "C" __global__ void __launch_bounds__({BLOCK}) proj{k}_psp() {{
    const long long t = *{self.ptr('t')};
    const {dt_t} dt = ({dt_t})(*{self.ptr('dt')});
    (void)t; (void)dt;
    {nl.join(decl)}
    const int* __restrict__ anb_col = {p('col')};
    const {rp_t}* __restrict__ anb_rp = {p('row_ptr')};
    for (int anb_row = blockIdx.x * blockDim.x + threadIdx.x; anb_row < {lay['rows']};
         anb_row += gridDim.x * blockDim.x) {{
      const int anb_post = {p('post_rank')}[anb_row];
      {reduce}
      {sum_}[anb_post] += anb_s;
    }}
}}
"""

    @staticmethod
    def continuous_update(proj) -> bool:
        """Synaptic variables with equations evaluated every step (the
        reference's update_synapse), rate-coded or spiking."""
        return any(v.get("cpp") and v.get("method") != "event-driven"
                   for v in proj.desc["variables"])

    @staticmethod
    def rate_learning(proj) -> bool:
        """A rate-coded projection whose synapse has continuous equations
        (the reference's update_synapse)."""
        if proj.synapse_type.type != "rate":
            return False
        return any(v.get("cpp") and v.get("method") != "event-driven"
                   for v in proj.desc["variables"])

    def _syn_block(self, proj, locality: str) -> str:
        """The equations of one locality in the reference's order
        (ANNarchy/generator/Utils.py:17-210): consecutive ODEs as one block
        (all increments, then the switches with their bounds), other
        statements with their bounds; the weight's update only while
        plasticity is on."""
        desc = proj.desc
        blocks, is_ode = [], False
        for v in desc["variables"]:
            if not v.get("cpp") or v.get("method") == "event-driven" or v["name"] not in desc[locality]:
                continue
            if v.get("switch"):
                if is_ode and blocks:
                    blocks[-1][1].append(v)
                else:
                    blocks.append(("ode", [v]))
                is_ode = True
            else:
                if not is_ode and blocks:
                    blocks[-1][1].append(v)
                else:
                    blocks.append(("non-ode", [v]))
                is_ode = False
        idx = {"local": "%(local_index)s", "semiglobal": "%(semiglobal_index)s", "global": ""}[locality]

        def bounds(v):
            out = ""
            for b, val in v.get("bounds", {}).items():
                if b in ("min", "max"):
                    op = "<" if b == "min" else ">"
                    out += f"if({v['name']}{idx} {op} {val}) {v['name']}{idx} = {val};\n"
            return out

        code = []
        for kind, vs in blocks:
            if kind == "ode":
                for v in vs:
                    cpp = v["cpp"] if isinstance(v["cpp"], str) else "\n".join(v["cpp"])
                    code.append(cpp)
                for v in vs:
                    body = v["switch"] + "\n" + bounds(v)
                    code.append(f"if (anb_plastic) {{ {body} }}" if v["name"] == "w" else body)
            else:
                for v in vs:
                    body = v["cpp"] + "\n" + bounds(v)
                    code.append(f"if (anb_plastic) {{ {body} }}" if v["name"] == "w" else body)
        text = "\n".join(code)
        # updates every `period` steps integrate over period * dt (as the reference's _dt)
        return re.sub(r"(?<![\w.])dt(?!\w)", "anb_dt", text)

    def rate_update_kernels(self, proj) -> list:
        """Continuous update of the synaptic variables of a rate-coded
        projection after the neuron updates of the step
        (ANNarchy/generator/Projection/SingleThreadGenerator.py:1575-1700,
        OpenMP/CSR.py:833-865): when learning is on and (t - offset) is a
        multiple of the period, the global equations once, then per dendrite
        (a warp) its semiglobal equations (lane 0) followed by the local
        equations of its synapses (one lane each). Returns [(source, plan
        entry)]."""
        k = proj.id
        a, b = proj.pre_pop, proj.post_pop
        lay = self.c.layout[k]
        desc = proj.desc
        if getattr(proj, "_device_conn", None) or lay.get("device"):
            raise NotImplementedError(f"{proj.name}: synaptic equations evaluated every step need "
                                      "connectivity built on the host in this backend")
        for v in desc["variables"]:
            if v.get("cpp") and v.get("method") not in ("explicit", "exponential", "event-driven",
                                                        None) and v.get("switch"):
                raise NotImplementedError(f"{proj.name}: synaptic variable {v['name']!r} uses the "
                                          f"{v['method']!r} method; rate-coded synapses support "
                                          "explicit and exponential Euler in this backend")
        # constants of the exponential method (the step's decay factor over
        # the update period, the reference's __stepsize_<x>)
        pre_loop = "\n    ".join(
            self.typed("const double " + v["pre_loop"]["name"] + " = " + re.sub(
                r"(?<![\w.])dt(?!\w)", "anb_dt", self.fill(v["pre_loop"]["value"])) + ";")
            for v in desc["variables"] if v.get("pre_loop"))
        p = lambda n: self.ptr(f"proj{k}__{n}")
        dt_t = "double" if self.exact else "float"
        # no early return: the step counter's epilogue may follow these kernels
        head = f"""    const long long t = *{self.ptr('t')};
    const int* anb_fl = {p('flags')};
    const int anb_plastic = anb_fl[0];
    const bool anb_go = anb_fl[1] && (t - anb_fl[3]) % anb_fl[2] == 0;
    const {dt_t} anb_dt = ({dt_t})(*{self.ptr('dt')}) * anb_fl[2];
"""
        glob_all = [q for q in desc["parameters"] + desc["variables"] if q["locality"] == "global"]
        glob_eq = self._syn_block(proj, "global")
        out = []

        def draws(locality, index):
            """This step's draws of the synapse's random distributions of one
            locality: Philox keyed by the network's seed, stream (projection,
            distribution), step and index (synapse, dendrite or 0)."""
            lines = []
            for kk, rd in enumerate(desc.get("random_distributions", [])):
                if rd["locality"] != locality:
                    continue
                args = ", ".join(f"({self.real})({self.typed(a)})" for a in rd["args"])
                lines.append(f"const {self.real} {rd['name']} = {self._DRAW_FN[rd['dist']]}<{self.real}>("
                             f"{self.ptr('rng_seed')}, {0x40000000 | (k << 8) | kk}u, t, "
                             f"(unsigned)({index}), {args});")
            return "\n        ".join(lines)

        def refs(code):
            decl = []
            for prefix, pop in (("anb_pre_", a), ("anb_post_", b)):
                for n in sorted(set(re.findall(prefix + r"(\w+)\[", code))):
                    if n not in pop._host:
                        raise NotImplementedError(f"{proj.name}: {prefix[4:-1]}.{n} is not an attribute "
                                                  f"of {pop.name}")
                    ct = "int" if pop._ctype.get(n) in ("int", "bool") else self.real
                    decl.append(f"const {ct}* __restrict__ {prefix}{n} = "
                                f"{self.ptr(f'pop{pop.id}__{n}')};")
            return "\n    ".join(decl + self._globalop_refs(proj, code))

        if glob_eq.strip():
            code = self.typed(self.fill(glob_eq, post_prefix="anb_post_", post_index="[0]"))
            code = draws("global", "0") + "\n    " + code
            names = {q["name"] for q in desc["variables"] if q["locality"] == "global" and q.get("cpp")}
            loads = "\n    ".join(f"{self.real} {q['name']} = {p(q['name'])}[0];" for q in glob_all)
            stores = "\n    ".join(f"{p(n)}[0] = {n};" for n in sorted(names))
            src = f"""
extern "C" __global__ void __launch_bounds__(32) proj{k}_update_global() {{
{head}    if (anb_go && threadIdx.x == 0) {{
    {loads}
    {pre_loop}
    {refs(code)}
    {code}
    {stores}
    }}
}}
"""
            out.append((src, (f"proj{k}_update_global", 1, 32, 0)))
        semi_eq = self.typed(self.fill(self._syn_block(proj, "semiglobal"), semi="[anb_row]",
                                       post_prefix="anb_post_", post_index="[anb_post]"))
        loc_eq = self.typed(self.fill(self._syn_block(proj, "local"), local="[j]", semi="[anb_row]",
                                      pre_prefix="anb_pre_", pre_index="[anb_col[j]]",
                                      post_prefix="anb_post_", post_index="[anb_post]"))
        if not (semi_eq.strip() or loc_eq.strip()):
            return out
        if semi_eq.strip():
            semi_eq = draws("semiglobal", "anb_row") + "\n        " + semi_eq
        if loc_eq.strip():
            loc_eq = draws("local", "j") + "\n        " + loc_eq
        gvals = "\n    ".join(f"const {self.real} {q['name']} = {p(q['name'])}[0];" for q in glob_all)
        if pre_loop:
            gvals += "\n    " + pre_loop
        arrays = []
        for q in desc["variables"] + desc["parameters"]:
            if q["locality"] in ("local", "semiglobal"):
                arrays.append(f"{self.real}* __restrict__ {q['name']} = {p(q['name'])};")
        if "w" not in {q["name"] for q in desc["variables"] + desc["parameters"]}:
            arrays.append(f"{self.real}* __restrict__ w = {p('w')};")
        rp_t = lay["idx_t"]
        src = f"""
extern "C" __global__ void __launch_bounds__({BLOCK}) proj{k}_update() {{
{head}    {gvals}
    {chr(10).join('    ' + x for x in arrays).strip()}
    {refs(semi_eq + loc_eq)}
    const int* __restrict__ anb_col = {p('col')};
    const {rp_t}* __restrict__ anb_rp = {p('row_ptr')};
    const int anb_lane = threadIdx.x & 31;
    for (int anb_row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; anb_go && anb_row < {lay['rows']};
         anb_row += (gridDim.x * blockDim.x) >> 5) {{
      const int anb_post = {p('post_rank')}[anb_row];
      if (anb_lane == 0) {{
        {semi_eq}
      }}
      __syncwarp();
      for ({rp_t} j = anb_rp[anb_row] + anb_lane; j < anb_rp[anb_row + 1]; j += 32) {{
        {loc_eq}
      }}
      __syncwarp();
    }}
}}
"""
        out.append((src, (f"proj{k}_update", grid_for(lay["rows"] * 32), BLOCK, 0)))
        return out

    def timed_array_kernel(self, pop) -> str:
        """TimedArray update (ANNarchy/inputs/TimedArray.py, update_variables):
        internal time tau = t - t0 (modulo the period when positive); when tau
        equals schedule[b], r = buffer[b]; otherwise r keeps its value. The
        schedule is increasing, so b is found by bisection."""
        k = pop.id
        return f"""
extern "C" __global__ void __launch_bounds__({BLOCK}) pop{k}_timed() {{
    const long long t = *{self.ptr('t')};
    const long long* anb_meta = {self.ptr(f'pop{k}__ta_meta')};
    long long tau = t - anb_meta[0];
    const long long period = anb_meta[1];
    const int nb = (int)anb_meta[2];
    if (tau < 0 || nb == 0) return;
    if (period > 0) tau %= period;
    const int* __restrict__ sched = {self.ptr(f'pop{k}__ta_sched')};
    int lo = 0, hi = nb - 1, b = -1;
    while (lo <= hi) {{
      const int mid = (lo + hi) >> 1;
      const long long s = sched[mid];
      if (s == tau) {{ b = mid; break; }}
      if (s < tau) lo = mid + 1; else hi = mid - 1;
    }}
    if (b < 0) return;
    const {self.real}* __restrict__ buf = {self.ptr(f'pop{k}__ta_buf')} + (size_t)b * {pop.size};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < {pop.size}; i += gridDim.x * blockDim.x)
      {self.ptr(f'pop{k}__r')}[i] = buf[i];
}}
"""

    def delay_kernel(self, pop) -> str:
        """This step's rates into the history ring of a population without
        an update of its own (the reference's update_delay)."""
        k = pop.id
        return f"""
extern "C" __global__ void __launch_bounds__({BLOCK}) pop{k}_delay() {{
    const long long t = *{self.ptr('t')};
    for (int anb_i = blockIdx.x * blockDim.x + threadIdx.x; anb_i < {pop.size};
         anb_i += gridDim.x * blockDim.x)
      {self.ptr(f'pop{k}___delayed_r')}[(size_t)anb_ring_slot(t, {self.slots(pop)}) * {self.c.ring_stride(pop)} + anb_i] =
          {self.ptr(f'pop{k}__r')}[anb_i];
}}
"""

    def has_update(self, pop) -> bool:
        if pop.neuron_type.type == "spike":
            return True
        return any(v.get("cpp") for v in pop.desc["variables"])

    # ------------------------------------------------------------ projections
    def rate_kernel(self, proj):
        """Weighted-sum kernel(s) of a rate-coded projection in its storage
        format. Returns (source, [(kernel, grid, block, smem)])."""
        k = proj.id
        lay = self.c.layout[proj.id]
        pre_r = self.pre_rate(proj)
        sum_ = self.ptr(f"pop{proj.post_pop.id}___sum_{proj.target}")
        fmt = lay["format"]
        p = lambda n: self.ptr(f"proj{k}__{n}")
        # learning and custom-psp projections keep float32 weights
        W = ("float" if ((self.rate_learning(proj) or self.custom_psp(proj)) and not self.exact)
             else self.c.wctype)
        name = f"proj{k}_psp"
        tdecl = f"const long long t = *{self.ptr('t')};\n    " if self.delayed(proj) else ""

        def kern(nm, body, block=BLOCK, min_blocks=None):
            bounds = f"{block}, {min_blocks}" if min_blocks else f"{block}"
            return f"""
extern "C" __global__ void __launch_bounds__({bounds}) {nm}() {{
    {tdecl}{body}
}}
"""
        if self.custom_psp(proj):
            if self.delayed(proj):
                raise NotImplementedError(f"{proj.name}: a custom psp with synaptic delays is not "
                                          "supported by this backend")
            return self.custom_psp_kernel(proj), [(name, grid_for(lay["rows"]), BLOCK, 0)]
        if fmt == "bsr_tc":
            # copies of the network sharing the weights: one tensor-core
            # product for all of them (a library operation of the plan)
            op = {"prefix": f"proj{k}", "x": f"pop{proj.pre_pop.id}__r",
                  "y": f"pop{proj.post_pop.id}___sum_{proj.target}",
                  "n_block_rows": lay["n_block_rows"], "batch": lay["batch"],
                  "n_pre": lay["n_pre"], "n_post": lay["n_post"]}
            return "", [(op, 0, 0, 0)]
        if proj._delay_steps is not None:
            # one delay per synapse: CSR rows read the rate ring per synapse
            a = proj.pre_pop
            call = (f"anb_rate_csr_delayed_ordered<{self.real}, {W}, {lay['idx_t']}>({lay['rows']}, "
                    f"{p('row_ptr')}, {p('col')}, {p('w')}, {p('dly')}, "
                    f"{self.ptr(f'pop{a.id}___delayed_r')}, {self.c.ring_stride(a)}, {self.slots(a)}, t, "
                    f"{p('post_rank')}, {sum_});")
            return kern(name, call), [(name, grid_for(lay["rows"] * 32), BLOCK, 0)]
        if fmt == "pcsr" and not self.exact:
            pw = lay["panel_width"]
            call = (f"anb_rate_pcsr<{W}, {lay['pc_unroll']}>({p('pc_cta')}, {p('pc_warp')}, "
                    f"{p('pc_col')}, {p('pc_w')}, {pre_r}, "
                    f"{proj.pre_pop.size}, {pw}, {sum_}, {self.ptr('err')});")
            B = lay["pc_block"]
            return (kern(name, call, B, lay["pc_resident"]),
                    [(name, lay["pc_ctas"], B, 4 * pw)])
        if fmt in ("csr", "pcsr"):       # pcsr in double precision: CSR order
            if self.exact:
                # warp per row, additions in stored order
                call = (f"anb_rate_csr_ordered<double, double, {lay['idx_t']}>({lay['rows']}, "
                        f"{p('row_ptr')}, {p('col')}, {p('w')}, {pre_r}, {p('post_rank')}, {sum_});")
                return kern(name, call), [(name, grid_for(lay["rows"] * 32), BLOCK, 0)]
            G = lay["vgroup"]
            if lay.get("heavy", 0):
                light = (f"anb_rate_csr_vec<{G}, {W}>({lay['light']}, {p('rows_light')}, {p('row_ptr')}, "
                         f"{p('col')}, {p('w')}, {pre_r}, {p('post_rank')}, {sum_});")
                heavy = (f"anb_rate_csr_cta<{W}>({lay['heavy']}, {p('rows_heavy')}, {p('row_ptr')}, "
                         f"{p('col')}, {p('w')}, {pre_r}, {p('post_rank')}, {sum_});")
                return (kern(name, light) + kern(name + "_heavy", heavy),
                        [(name, grid_for(lay["light"] * G), BLOCK, 0),
                         (name + "_heavy", min(lay["heavy"], MAX_GRID), BLOCK, 0)])
            call = (f"anb_rate_csr_vec<{G}, {W}>({lay['rows']}, nullptr, {p('row_ptr')}, {p('col')}, "
                    f"{p('w')}, {pre_r}, {p('post_rank')}, {sum_});")
            return kern(name, call), [(name, grid_for(lay["rows"] * G), BLOCK, 0)]
        if fmt in ("ell", "ellr", "hyb"):
            rl = p("rl") if fmt in ("ellr", "hyb") else "nullptr"
            if self.exact:
                call = (f"anb_rate_ell<{self.real}, {W}>({lay['rows']}, {lay['width']}, {p('ell_col')}, "
                        f"{p('ell_w')}, {rl}, {pre_r}, {p('post_rank')}, {sum_});")
                src, plan = kern(name, call), [(name, lay["grid"], BLOCK, 0)]
            else:
                G = lay["split"]
                call = (f"anb_rate_slots_split<{G}, 1, {W}>({lay['rows']}, {lay['width']}, nullptr, "
                        f"{p('ell_col')}, {p('ell_w')}, {rl}, nullptr, {pre_r}, {p('post_rank')}, {sum_});")
                src = kern(name, call)
                plan = [(name, grid_for(lay["rows"] * G), BLOCK, 0)]
            if fmt == "hyb" and lay["coo_nnz"] > 0:
                src += self._hyb_tail(proj, lay, pre_r, sum_)
                plan.append((name + "_tail", lay["tail_grid"], BLOCK, 0))
            return src, plan
        if fmt == "sell":
            if self.exact:
                call = (f"anb_rate_sell<{lay['C']}, {self.real}, {W}>({lay['rows']}, {p('slice_ptr')}, "
                        f"{p('slice_len')}, {p('sell_col')}, {p('sell_w')}, {p('sell_rl')}, "
                        f"{p('perm')}, {pre_r}, {p('post_rank')}, {sum_});")
                return kern(name, call), [(name, lay["grid"], BLOCK, 0)]
            G = lay["split"]
            call = (f"anb_rate_slots_split<{G}, {lay['C']}, {W}>({lay['rows']}, 0, {p('slice_ptr')}, "
                    f"{p('sell_col')}, {p('sell_w')}, {p('sell_rl')}, {p('perm')}, {pre_r}, "
                    f"{p('post_rank')}, {sum_});")
            return kern(name, call), [(name, grid_for(lay["rows"] * G), BLOCK, 0)]
        if fmt == "bsr":
            T = lay["tile"]
            parts = 1 if self.exact else max(1, min(T, 256 // T))
            block = T * parts
            call = (f"anb_rate_bsr_rows<{T}, {parts}, {self.real}, {W}>({lay['block_rows']}, "
                    f"{p('bsr_row_ptr')}, {p('bsr_col')}, {p('bsr_val')}, {pre_r}, "
                    f"{proj.pre_pop.size}, {proj.post_pop.size}, {sum_});")
            return kern(name, call, block), [(name, min(lay["block_rows"], MAX_GRID * 4), block, 0)]
        raise NotImplementedError(fmt)

    def _hyb_tail(self, proj, lay, pre_r, sum_):
        k = proj.id
        p = lambda n: self.ptr(f"proj{k}__{n}")
        if self.exact:
            body = (f"anb_rate_csr_scalar<double, double, int>({lay['coo_rows']}, {p('coo_row_ptr')}, "
                    f"{p('coo_col')}, {p('coo_w')}, {pre_r}, {p('coo_post')}, {sum_});")
        else:
            body = (f"anb_rate_coo_atomic<{self.c.wctype}>({lay['coo_nnz']}, {p('coo_row')}, "
                    f"{p('coo_col')}, {p('coo_w')}, {pre_r}, {p('post_rank')}, {sum_});")
        tdecl = f"const long long t = *{self.ptr('t')};\n    " if self.delayed(proj) else ""
        return f"""
extern "C" __global__ void __launch_bounds__({BLOCK}) proj{k}_psp_tail() {{
    {tdecl}{body}
}}
"""

    def spike_kernel(self, proj) -> str:
        k = proj.id
        lay = self.c.layout[proj.id]
        pre_spk = self.pre_spk(proj)
        g = self.ptr(f"pop{proj.post_pop.id}__g_{proj.target}")
        p = lambda n: self.ptr(f"proj{k}__{n}")
        if proj.plastic:
            return self.plastic_psp_kernel(proj, lay, pre_spk, g)
        tdecl = f"const long long t = *{self.ptr('t')};"
        if proj._delay_steps is not None:
            a = proj.pre_pop
            call = (f"anb_spike_gather_delayed<{self.real}, {self.c.wctype if not self.exact else 'double'}, "
                    f"{'true' if self.exact else 'false'}>("
                    f"{lay['rows']}, {p('row_ptr')}, {p('col')}, {p('w')}, {p('dly')}, "
                    f"{self.ptr(f'pop{a.id}__spk')}, {(a.size + 31) // 32}, {self.slots(a)}, t, "
                    f"{p('post_rank')}, {g});")
            return f"""
extern "C" __global__ void __launch_bounds__({BLOCK}) proj{k}_psp() {{
    {tdecl}
    {call}
}}
"""
        if self.exact:
            call = (f"anb_spike_gather_warp<double, double>({lay['rows']}, {p('row_ptr')}, {p('col')}, "
                    f"{p('w')}, {pre_spk}, {p('post_rank')}, {g});")
        elif self.c.spike_lists and not self.delayed(proj):
            a = proj.pre_pop.id
            call = (f"anb_spike_scatter_list<float, {self.c.wctype}>({lay['w0'] * 32}, {lay['w1'] * 32}, "
                    f"{self.ptr(f'pop{a}__spl')} + ((t - 1) & 1) * (long long){proj.pre_pop.size}, "
                    f"{self.ptr(f'pop{a}__spn')}[(t - 1) & 1], {lay['chunks']}, {p('col_ptr')}, "
                    f"{p('post_idx')}, {p('w_pre')}, {g});")
            return f"""
extern "C" __global__ void __launch_bounds__({BLOCK}) proj{k}_psp() {{
    const long long t = *{self.ptr('t')};
    {call}
}}
"""
        else:
            call = (f"anb_spike_scatter<float, {self.c.wctype}>({lay['w0']}, {lay['w1']}, {pre_spk}, "
                    f"{p('col_ptr')}, {p('post_idx')}, {p('w_pre')}, {g});")
        return f"""
extern "C" __global__ void __launch_bounds__({BLOCK}) proj{k}_psp() {{
    {tdecl}
    {call}
}}
"""

    # plastic synapses: pre_spike statements inlined in the transmission
    def _syn_globals(self, proj):
        out = []
        for prm in proj.desc["parameters"] + proj.desc["variables"]:
            if prm["locality"] == "global":
                out.append(f"const {self.real} {prm['name']} = {self.ptr(f'proj{proj.id}__{prm['name']}')}[0];")
        return "\n    ".join(out)

    def _packed(self, proj):
        return trace_layout(proj, self.exact)

    def _pack_fields(self, proj, body: str, idx: str = "j") -> str:
        """Per-synapse statements rewritten onto the fields of the packed
        record `anb_s` (unchanged when the projection keeps separate arrays)."""
        lay = self._packed(proj)
        if lay is None:
            return body
        names, _ = lay
        body = body.replace(f"_last_event[{idx}] = t;", "anb_s._last_event = (int)t;")
        for n in names + ["_last_event"]:
            body = re.sub(rf"\b{re.escape(n)}\[{idx}\]", f"anb_s.{n}", body)
        return body

    def _pack_body(self, proj, body: str, idx: str = "j") -> str:
        """Per-synapse statements on the packed record: load it once, use
        its fields, store it back."""
        if self._packed(proj) is None:
            return body
        return (f"anb_tr{proj.id} anb_s = anb_tr[{idx}];\n          {self._pack_fields(proj, body, idx)}\n"
                f"          anb_tr[{idx}] = anb_s;")

    def _stdp_statements(self, proj):
        """(pre-spike statements, post-spike statements) of a plastic spiking
        projection, per synapse j: the event-driven decays (to t - 1 on the
        pre side, as the reference's transmission of the previous step's
        spikes; to t on the post side), then the synapse's own statements."""
        pre = self._event_driven(proj, "j", "t-1") + self.syn_spike_statements(proj, "pre_spike")
        post = self._event_driven(proj, "j", "t") + self.syn_spike_statements(proj, "post_spike")
        return "\n          ".join(pre), "\n          ".join(post)

    def fused_stdp_functions(self, proj) -> str:
        """Device functions of the persistent engine for a plastic projection
        with post-spike statements, which let the post events of step t - 1
        run in the same phase as the transmission of step t's spikes (one
        grid barrier less per step):

        * proj<k>_psp_fused_body(t, fused): the transmission of the spikes of
          t - 1 (pre-spike statements, g += w); with `fused`, a synapse whose
          post neuron also spiked at t - 1 first gets its post event of t - 1
          (the reference's order: post events end step t - 1, transmissions
          open step t), in the same thread, on the same loaded record;
        * proj<k>_post_prev_body(t): the post events of the spikes of t - 1
          (at time t - 1), skipping the synapses whose pre neuron spiked at
          t - 1 (done by the transmission above)."""
        k = proj.id
        lay = self.c.layout[proj.id]
        p = lambda n: self.ptr(f"proj{k}__{n}")
        a, b = proj.pre_pop.id, proj.post_pop.id
        pre_stmts, post_stmts = self._stdp_statements(proj)
        packed = self._packed(proj) is not None
        load = f"anb_tr{k} anb_s = anb_tr[j];" if packed else ""
        store = "anb_tr[j] = anb_s;" if packed else ""
        g = self.ptr(f"pop{b}__g_{proj.target}")
        pre_bits, post_bits = self.ptr(f"pop{a}__spk"), self.ptr(f"pop{b}__spk")
        ch, pch = lay["chunks"], lay["post_chunks"]
        head = f"""
    const float dt = (float)(*{self.ptr('dt')});
    const int anb_plastic = {p('flags')}[0];
    {self._syn_globals(proj)}
    {self._syn_arrays(proj)}"""
        return f"""
__device__ __forceinline__ void proj{k}_psp_fused_body(const long long anb_pt, const int anb_fused) {{
    const long long t = anb_pt;{head}
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int* __restrict__ anb_list = {self.ptr(f'pop{a}__spl')} + ((t - 1) & 1) * (long long){proj.pre_pop.size};
    const long long anb_items = (long long){self.ptr(f'pop{a}__spn')}[(t - 1) & 1] * {ch};
    for (long long anb_it = warp; anb_it < anb_items; anb_it += nwarps) {{
      const int anb_pre = anb_list[anb_it / {ch}];
      if (anb_pre < {lay['w0'] * 32} || anb_pre >= {lay['w1'] * 32}) continue;
      const int anb_c = (int)(anb_it % {ch});
      const int anb_end = {p('col_ptr')}[anb_pre + 1];
      for (int anb_k = {p('col_ptr')}[anb_pre] + anb_c * 32 + lane; anb_k < anb_end;
           anb_k += 32 * {ch}) {{
        const int j = {p('inv_idx')}[anb_k];
        const int anb_post = {p('post_idx')}[anb_k];
        float sum = 0.f;
        {self.syn_index_defs(pre_stmts + post_stmts, "anb_pre", "anb_post")}{load}
        if (anb_fused && anb_bit({post_bits}, anb_post)) {{
          const long long t = anb_pt - 1;
          {self._pack_fields(proj, post_stmts)}
        }}
        {self._pack_fields(proj, pre_stmts)}
        {store}
        atomicAdd(&{g}[anb_post], sum);
      }}
    }}
}}

__device__ __forceinline__ void proj{k}_post_prev_body(const long long anb_pt) {{
    const long long t = anb_pt - 1;{head}
    const int anb_lane = threadIdx.x & 31;
    const int* __restrict__ anb_list = {self.ptr(f'pop{b}__spl')} + (t & 1) * (long long){proj.post_pop.size};
    const long long anb_items = (long long){self.ptr(f'pop{b}__spn')}[t & 1] * {pch};
    for (long long anb_it = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; anb_it < anb_items;
         anb_it += (gridDim.x * blockDim.x) >> 5) {{
      const int anb_spiker = anb_list[anb_it / {pch}];
      const int anb_row = {p('row_of')}[anb_spiker];
      if (anb_row < 0) continue;
      const int anb_c = (int)(anb_it % {pch});
      const int anb_end = {p('row_ptr')}[anb_row + 1];
      for (int j = {p('row_ptr')}[anb_row] + anb_c * 32 + anb_lane; j < anb_end; j += 32 * {pch}) {{
        if (anb_bit({pre_bits}, {p('col')}[j])) continue;   // done with the transmission
        {self.syn_index_defs(post_stmts, f"{p('col')}[j]", "anb_spiker")}{self._pack_body(proj, post_stmts)}
      }}
    }}
}}
"""

    def _syn_arrays(self, proj):
        lay = self._packed(proj)
        if lay is not None:
            names, nbytes = lay
            fields = " ".join(f"float {n};" for n in names) + " int _last_event;"
            pad = nbytes // 4 - len(names) - 1
            fields += "".join(f" int anb_pad{i};" for i in range(pad))
            self.types[f"anb_tr{proj.id}"] = (f"struct __align__({min(nbytes, 16)}) anb_tr{proj.id} "
                                              f"{{ {fields} }};\n")
            return "\n    ".join(
                [f"anb_tr{proj.id}* __restrict__ anb_tr = "
                 f"reinterpret_cast<anb_tr{proj.id}*>({self.ptr(f'proj{proj.id}__tr')});"]
                + self._syn_neuron_refs(proj))
        decl = []
        for n in syn_local_names(proj):
            decl.append(f"{self.real}* __restrict__ {n} = {self.ptr(f'proj{proj.id}__{n}')};")
        decl.append(f"long long* __restrict__ _last_event = {self.ptr(f'proj{proj.id}___last_event')};")
        return "\n    ".join(decl + self._syn_neuron_refs(proj))

    def syn_fill(self, code: str, idx: str = "j") -> str:
        """A per-synapse statement: synapse arrays at [idx], the pre- and
        post-synaptic neurons' attributes (pre.x, post.x, t_pre, t_post) at
        [anb_pi] and [anb_qi], which every kernel running these statements
        defines for its synapse (syn_index_defs)."""
        return self.fill(code, local=f"[{idx}]", pre_prefix="anb_pre_", pre_index="[anb_pi]",
                         post_prefix="anb_post_", post_index="[anb_qi]")

    def syn_spike_statements(self, proj, which: str) -> list:
        """The pre_spike or post_spike statements of a spiking projection for
        synapse j, each followed by its bounds (`w -= 1.0 : min=0.0`), the
        weight's only while plasticity is on."""
        out = []
        for v in proj.desc[which]:
            code = self.syn_fill(v["cpp"])
            if v["name"] != "g_target":
                idx = "[j]" if v["locality"] == "local" else "[0]"
                for b, val in v.get("bounds", {}).items():
                    if b in ("min", "max"):
                        op = "<" if b == "min" else ">"
                        val = self.syn_fill(str(val))
                        code += f" if ({v['name']}{idx} {op} {val}) {v['name']}{idx} = {val};"
            if v["name"] == "w" and (which == "post_spike" or proj.desc["plasticity"]):
                code = f"if (anb_plastic) {{ {code} }}"
            out.append(self.typed(code))
        return out

    def _syn_neuron_refs(self, proj) -> list:
        """Pointers to the pre/post population arrays the projection's
        per-synapse statements read (last_spike for t_pre / t_post)."""
        code = " ".join(v.get("cpp", "") or "" for v in
                        proj.desc.get("pre_spike", []) + proj.desc.get("post_spike", [])
                        + [v for v in proj.desc["variables"] if v.get("method") == "event-driven"])
        code = self.syn_fill(code) if code.strip() else ""
        decl = []
        for prefix, pop in (("anb_pre_", proj.pre_pop), ("anb_post_", proj.post_pop)):
            for n in sorted(set(re.findall(prefix + r"(\w+)\[", code))):
                if n == "last_spike":
                    ct = "long long"
                elif n in pop._host:
                    ct = "int" if pop._ctype.get(n) in ("int", "bool") else self.real
                else:
                    raise NotImplementedError(f"{proj.name}: {prefix[4:-1]}.{n} is not an attribute "
                                              f"of {pop.name}")
                decl.append(f"const {ct}* __restrict__ {prefix}{n} = {self.ptr(f'pop{pop.id}__{n}')};")
        return decl + self._globalop_refs(proj, code)

    def _globalop_refs(self, proj, code: str) -> list:
        """Scalars of the pre/post populations' reductions a synaptic
        statement reads (`anb_pre__mean_r`: the value after the previous
        step)."""
        decl = []
        for prefix, pop in (("anb_pre_", proj.pre_pop), ("anb_post_", proj.post_pop)):
            for n in sorted(set(re.findall(prefix + r"_(\w+)\b(?!\s*\[)", code))):
                if "_" + n in pop._host and pop._locality.get("_" + n) == "global":
                    decl.append(f"const {self.real} {prefix}_{n} = {self.ptr(f'pop{pop.id}___{n}')}[0];")
        return decl

    @staticmethod
    def syn_index_defs(body: str, pre: str, post: str) -> str:
        """Definitions of anb_pi / anb_qi (pre and post neuron of the synapse)
        for a body that uses them."""
        out = ""
        if "anb_pi]" in body:
            out += f"const int anb_pi = {pre};\n          "
        if "anb_qi]" in body:
            out += f"const int anb_qi = {post};\n          "
        return out

    def _event_driven(self, proj, idx, t_expr):
        out = []
        for v in proj.desc["variables"]:
            if v.get("method") == "event-driven":
                code = self.syn_fill(v["cpp"], idx)
                out.append(self.typed(code.replace("(t))", f"({t_expr}))")))
        out.append(f"_last_event[{idx}] = t;")
        return out

    def plastic_psp_kernel(self, proj, lay, pre_spk, g) -> str:
        k = proj.id
        p = lambda n: self.ptr(f"proj{k}__{n}")
        stmts = self._event_driven(proj, "j", "t-1") + self.syn_spike_statements(proj, "pre_spike")
        body = self._pack_body(proj, "\n          ".join(stmts))
        if self.exact or self.delayed(proj) or not self.c.spike_lists:
            # warp per post row; the spiking synapses of a row are processed in
            # ascending pre rank, one at a time, by the lane that holds them
            # (the running conductance `sum` is passed along with a shuffle);
            # also the fast form of a delayed projection (spike lists hold
            # only the previous step)
            return f"""
extern "C" __global__ void __launch_bounds__({BLOCK}) proj{k}_psp() {{
    const long long t = *{self.ptr('t')};
    const {self.real} dt = ({self.real})(*{self.ptr('dt')});
    const int anb_plastic = {p('flags')}[0];
    {self._syn_globals(proj)}
    {self._syn_arrays(proj)}
    const int anb_lane = threadIdx.x & 31;
    for (int anb_row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; anb_row < {lay['rows']};
         anb_row += (gridDim.x * blockDim.x) >> 5) {{
      const int anb_post = {p('post_rank')}[anb_row];
      const int anb_beg = {p('row_ptr')}[anb_row], anb_end = {p('row_ptr')}[anb_row + 1];
      {self.real} sum = {g}[anb_post];
      bool anb_any = false;
      for (int anb_b0 = anb_beg; anb_b0 < anb_end; anb_b0 += 32) {{
        const int j = anb_b0 + anb_lane;
        const bool anb_sp = j < anb_end && anb_bit({pre_spk}, {p('col')}[j]);
        anb_u32 anb_m = __ballot_sync(0xffffffffu, anb_sp);
        anb_any |= anb_m != 0u;
        while (anb_m) {{
          const int anb_b = __ffs(anb_m) - 1;
          anb_m &= anb_m - 1;
          if (anb_lane == anb_b) {{
            {self.syn_index_defs(body, f"{p('col')}[j]", "anb_post")}{body}
          }}
          sum = __shfl_sync(0xffffffffu, sum, anb_b);
        }}
      }}
      if (anb_any && anb_lane == 0) {g}[anb_post] = sum;
    }}
}}
"""
        # fast: work items (spike of the previous step, 32-synapse chunk of its
        # fan-out); the synapse state is reached through inv_idx
        a = proj.pre_pop.id
        return f"""
extern "C" __global__ void __launch_bounds__({BLOCK}) proj{k}_psp() {{
    const long long t = *{self.ptr('t')};
    const float dt = (float)(*{self.ptr('dt')});
    const int anb_plastic = {p('flags')}[0];
    {self._syn_globals(proj)}
    {self._syn_arrays(proj)}
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int* __restrict__ anb_list = {self.ptr(f'pop{a}__spl')} + ((t - 1) & 1) * (long long){proj.pre_pop.size};
    const long long anb_items = (long long){self.ptr(f'pop{a}__spn')}[(t - 1) & 1] * {lay['chunks']};
    for (long long anb_it = warp; anb_it < anb_items; anb_it += nwarps) {{
      const int anb_pre = anb_list[anb_it / {lay['chunks']}];
      if (anb_pre < {lay['w0'] * 32} || anb_pre >= {lay['w1'] * 32}) continue;
      const int anb_c = (int)(anb_it % {lay['chunks']});
      const int anb_end = {p('col_ptr')}[anb_pre + 1];
      for (int anb_k = {p('col_ptr')}[anb_pre] + anb_c * 32 + lane; anb_k < anb_end;
           anb_k += 32 * {lay['chunks']}) {{
        const int j = {p('inv_idx')}[anb_k];
        float sum = 0.f;
        {self.syn_index_defs(body, "anb_pre", f"{p('post_idx')}[anb_k]")}{body}
        atomicAdd(&{g}[{p('post_idx')}[anb_k]], sum);
      }}
    }}
}}
"""

    def post_event_kernel(self, proj) -> str:
        k = proj.id
        lay = self.c.layout[proj.id]
        p = lambda n: self.ptr(f"proj{k}__{n}")
        post_spk = self.spk_at(proj.post_pop, "t")
        stmts = self._event_driven(proj, "j", "t") + self.syn_spike_statements(proj, "post_spike")
        body = self._pack_body(proj, "\n        ".join(stmts))
        dt_t = "double" if self.exact else "float"
        if not self.exact and self.c.spike_lists:
            b = proj.post_pop.id
            ch = lay["post_chunks"]
            return f"""
extern "C" __global__ void __launch_bounds__({BLOCK}) proj{k}_post_event() {{
    const long long t = *{self.ptr('t')};
    const float dt = (float)(*{self.ptr('dt')});
    const int anb_plastic = {p('flags')}[0];
    {self._syn_globals(proj)}
    {self._syn_arrays(proj)}
    const int anb_lane = threadIdx.x & 31;
    const int* __restrict__ anb_list = {self.ptr(f'pop{b}__spl')} + (t & 1) * (long long){proj.post_pop.size};
    const long long anb_items = (long long){self.ptr(f'pop{b}__spn')}[t & 1] * {ch};
    for (long long anb_it = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; anb_it < anb_items;
         anb_it += (gridDim.x * blockDim.x) >> 5) {{
      const int anb_spiker = anb_list[anb_it / {ch}];
      const int anb_row = {p('row_of')}[anb_spiker];
      if (anb_row < 0) continue;
      const int anb_c = (int)(anb_it % {ch});
      const int anb_end = {p('row_ptr')}[anb_row + 1];
      for (int j = {p('row_ptr')}[anb_row] + anb_c * 32 + anb_lane; j < anb_end; j += 32 * {ch}) {{
        {self.syn_index_defs(body, f"{p('col')}[j]", "anb_spiker")}{body}
      }}
    }}
}}
"""
        return f"""
extern "C" __global__ void __launch_bounds__({BLOCK}) proj{k}_post_event() {{
    const long long t = *{self.ptr('t')};
    const {dt_t} dt = ({dt_t})(*{self.ptr('dt')});
    const int anb_plastic = {p('flags')}[0];
    {self._syn_globals(proj)}
    {self._syn_arrays(proj)}
    const int anb_lane = threadIdx.x & 31;
    for (int anb_row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; anb_row < {lay['rows']};
         anb_row += (gridDim.x * blockDim.x) >> 5) {{
      const int anb_post = {p('post_rank')}[anb_row];
      if (!anb_bit({post_spk}, anb_post)) continue;           // warp-uniform
      for (int j = {p('row_ptr')}[anb_row] + anb_lane; j < {p('row_ptr')}[anb_row + 1]; j += 32) {{
        {self.syn_index_defs(body, f"{p('col')}[j]", "anb_post")}{body}
      }}
    }}
}}
"""

    # --------------------------------------------------------------- monitors
    @staticmethod
    def target_variables(mon) -> list:
        """The conductances g_<target> a monitor of a spiking population
        records: the reference records them right after the step's
        transmissions, before the neurons' update (record_targets,
        ANNarchy/generator/Template/OpenMPBaseTemplate.py:236-242 and
        Monitor/MonitorGenerator.py:112-156); every other variable after the
        update."""
        pop = mon.population
        if pop.neuron_type.type != "spike":
            return []
        names = {"g_" + t for t in pop.targets}
        return [v for v in mon.variables if v in names]

    def monitor_kernel(self, mon, targets: bool = False) -> str:
        """Variable recording of one monitor (grid engine): the conductances
        of the step's transmissions (`targets`, kernel mon<m>_record_targets,
        launched before the updates) or the other variables (mon<m>_record,
        after them). Spike bitmaps are written by the update kernel of the
        population."""
        m = mon.id
        lay = self.c.mon_layout[m]
        tv = self.target_variables(mon)
        parts = []
        for var in mon.variables:
            if var == "spike" or (var in tv) != targets:
                continue
            src = self.ptr(f"pop{mon.population.id}__{source_name(var)}")
            ranks = self.ptr(f"mon{m}__ranks") if mon.ranks is not None else "nullptr"
            parts.append(f"""
    if (anb_on && ((t - {self.ptr(f'mon{m}__start')}[0]) % {mon.period_steps} == {mon.period_offset_steps % mon.period_steps})) {{
      const long long anb_slot = (t - {self.ptr(f'mon{m}__t0v')}[0]) / {mon.period_steps};
      if (anb_slot >= 0 && anb_slot < {lay['cap_var']})
        anb_record({src}, {ranks}, {lay['n']}, {self.ptr(f'mon{m}__{array_name(var)}')}, anb_slot);
      else if (blockIdx.x == 0 && threadIdx.x == 0)
        anb_report({self.ptr('err')}, ANB_DEVERR_MONITOR_OVERFLOW);
    }}""")
        return f"""
extern "C" __global__ void __launch_bounds__({BLOCK}) mon{m}_record{'_targets' if targets else ''}() {{
    const long long t = *{self.ptr('t')};
    const int anb_on = {self.ptr(f'mon{m}__on')}[0];
    {''.join(parts)}
}}
"""

    # ------------------------------------------------------------------ engines
    def persistent_ok(self) -> bool:
        """The grid engine's per-step kernels can run as phases of one
        persistent launch: fast spiking networks whose kernels all walk their
        work grid-stride (spike-list transmissions, updates, post events,
        variable records) - no rate-coded projections (some formats need
        their own grid), delays, timed arrays or stop conditions."""
        net = self.net
        if self.exact or not self.c.spike_lists or getattr(self.c, "shard", None):
            return False
        if any(p.synapse_type.type != "spike" for p in net.projections):
            return False
        if any(getattr(p, "stop_condition", None) or hasattr(p, "_ta_schedule_ms")
               or p.neuron_type.type != "spike" or self.slots(p) > 1 or global_equations(p)
               or p._globalops for p in net.populations):
            return False
        return True

    def persistent_module(self) -> Module:
        """The grid engine's step as one cooperative persistent kernel
        anb_grid_run(t0, nsteps): every kernel of the step plan becomes a
        device function; per step the functions run in plan order, the
        concurrent group of atomic transmissions as one phase, with a
        grid-wide barrier after every phase (bounded: a CTA that waits about
        a second reports ANB_DEVERR_BARRIER_TIMEOUT and every CTA leaves).
        The reference launches each of these kernels every step and copies
        the spike count to the host between them
        (ANNarchy/generator/Template/CUDABaseTemplate.py:328-630)."""
        kernels, plan = self._grid_parts()
        t_ptr = self.ptr("t")
        # plastic projections with post events: those run with the next
        # step's transmissions (fused_stdp_functions), the last step's after
        # the loop
        fused = [p for p in self.net.projections
                 if p.synapse_type.type == "spike" and p.desc.get("post_spike")]
        fused_ids = {p.id for p in fused}
        plan = [e for e in plan if not (e[0].endswith("_post_event") and
                                       int(e[0][4:e[0].index("_")]) in fused_ids)]
        bodies = []
        for src in kernels:
            if not src.strip():
                continue
            src = re.sub(r'extern "C" __global__ void (?:__launch_bounds__\([^)]*\) )?(\w+)\(\) \{',
                         r"__device__ __forceinline__ void \1_body(const long long anb_pt) {", src)
            bodies.append(src.replace("*" + t_ptr, "anb_pt"))
        phases, i = [], 0
        while i < len(plan):
            j = i + 1
            if len(plan[i]) > 4 and plan[i][4]:
                while j < len(plan) and len(plan[j]) > 4 and plan[j][4] == plan[i][4]:
                    j += 1
            phases.append([e[0] for e in plan[i:j]])
            i = j
        resets = "".join(f"\n        {self.ptr(f'pop{p.id}__spn')}[t & 1] = 0;"
                         for p in self.net.populations if p.neuron_type.type == "spike")
        def call(name):
            if name.endswith("_psp") and int(name[4:name.index("_")]) in fused_ids:
                k = name[4:name.index("_")]
                return (f"\n      proj{k}_psp_fused_body(t, anb_s > 0);"
                        f"\n      if (anb_s > 0) proj{k}_post_prev_body(t);")
            return f"\n      {name}_body(t);"
        steps = []
        for ph in phases:
            calls = "".join(call(name) for name in ph)
            steps.append(f"""{calls}
      if (!anb_grid_sync({self.ptr('gbar')}, {self.ptr('err')})) break;""")
        bodies += [self.fused_stdp_functions(p) for p in fused]
        # the post events of the last step (the next launch starts unfused):
        # proj<k>_post_event_body, converted with the plan's other kernels
        tail = "".join(f"\n      proj{p.id}_post_event_body(t0 + nsteps - 1);" for p in fused)
        # one CTA of PERSISTENT_BLOCK threads per SM: few CTAs arrive at each
        # grid barrier (the arrivals serialise on one counter)
        src = f"""
extern "C" __global__ void __launch_bounds__({PERSISTENT_BLOCK}, 1) anb_grid_run(long long t0, int nsteps) {{
    int anb_s = 0;
    for (; anb_s < nsteps; ++anb_s) {{
      const long long t = t0 + anb_s;
      // this step's spike lists start empty (their parity was last read by
      // the transmissions of step t - 1 and the post events of step t - 2)
      if (blockIdx.x == 0 && threadIdx.x == 0) {{{resets}
      }}{''.join(steps)}
    }}
    if (anb_s == nsteps && nsteps > 0) {{{tail}
    }}
    if (blockIdx.x == 0 && threadIdx.x == 0 && anb_s == nsteps) *{t_ptr} = t0 + nsteps;
}}
"""
        return Module(self.assemble(bodies + [src]), self.options(), "grid",
                      local=("anb_grid_run", 0, PERSISTENT_BLOCK, 0, -1), kernels=["anb_grid_run"])

    def grid_module(self) -> Module:
        kernels, plan = self._grid_parts()
        return self._grid_finish(kernels, plan)

    def _grid_parts(self):
        """Kernels and step plan of the grid engine (without the step
        counter's epilogue)."""
        net = self.net
        kernels, plan = [], []
        for proj in net.projections:
            lay = self.c.layout[proj.id]
            if proj.synapse_type.type == "rate":
                src, launches = self.rate_kernel(proj)
                kernels.append(src)
                plan.extend(launches)
            else:
                kernels.append(self.spike_kernel(proj))
                # fast transmissions that add with atomics run concurrently
                # (one graph branch each); the gathers write g[post] in place
                group = 1 if self.atomic_psp(proj) else 0
                plan.append((f"proj{proj.id}_psp", lay["grid"], BLOCK, 0, group))
        for mon in net.monitors:
            if self.target_variables(mon):
                # the conductances after the transmissions, before the updates
                kernels.append(self.monitor_kernel(mon, targets=True))
                n = self.c.mon_layout[mon.id]["n"]
                plan.append((f"mon{mon.id}_record_targets", grid_for(max(n, 32)), BLOCK, 0))
        for pop in net.populations:
            if hasattr(pop, "_ta_schedule_ms"):
                kernels.append(self.timed_array_kernel(pop))
                plan.append((f"pop{pop.id}_timed", grid_for(pop.size), BLOCK, 0))
                if self.slots(pop) > 1:
                    kernels.append(self.delay_kernel(pop))
                    plan.append((f"pop{pop.id}_delay", grid_for(pop.size), BLOCK, 0))
            elif self.has_update(pop):
                kernels.append(self.pop_kernel(pop))
                lo, hi = getattr(self.c, "owned", {}).get(pop.id, (0, pop.size))
                K = self.neurons_per_thread(pop)
                plan.append((f"pop{pop.id}_step", grid_for(max(1, -(-(hi - lo) // K))), BLOCK, 0))
            if pop._globalops:
                kernels.append(self.globalops_kernel(pop))
                plan.append((f"pop{pop.id}_globalops", 1, 32 if self.exact else 1024, 0))
            elif pop.neuron_type.type == "rate" and self.slots(pop) > 1:
                kernels.append(self.delay_kernel(pop))
                plan.append((f"pop{pop.id}_delay", grid_for(pop.size), BLOCK, 0))
        for proj in net.projections:
            if self.continuous_update(proj):
                for src, entry in self.rate_update_kernels(proj):
                    kernels.append(src)
                    plan.append(entry)
        for proj in net.projections:
            if proj.synapse_type.type == "spike" and proj.desc.get("post_spike"):
                kernels.append(self.post_event_kernel(proj))
                lay = self.c.layout[proj.id]
                grid = (list_grid(proj.post_pop.size, lay["post_chunks"])
                        if (self.c.spike_lists and not self.exact) else grid_for(lay["rows"] * 32))
                plan.append((f"proj{proj.id}_post_event", grid, BLOCK, 0))
        for mon in net.monitors:
            tv = self.target_variables(mon)
            if any(v != "spike" and v not in tv for v in mon.variables):
                # spikes are written by the update kernel of the population
                kernels.append(self.monitor_kernel(mon))
                n = self.c.mon_layout[mon.id]["n"]
                plan.append((f"mon{mon.id}_record", grid_for(max(n, 32)), BLOCK, 0))
        return kernels, plan

    def _grid_finish(self, kernels, plan) -> Module:
        net = self.net
        resets = ""
        if self.c.spike_lists:
            for pop in net.populations:
                if pop.neuron_type.type == "spike":
                    resets += f" {self.ptr(f'pop{pop.id}__spn')}[(anb_tt + 1) & 1] = 0;"
        # the step counter advances at the end of the step's last kernel, by the
        # last of its CTAs to finish (every CTA has read t by then)
        epilogue = f"""
    __syncthreads();
    if (threadIdx.x == 0) {{
      __threadfence();
      const unsigned anb_prev = atomicAdd({self.ptr('tickc')}, 1u);
      if (anb_prev == gridDim.x - 1) {{
        *{self.ptr('tickc')} = 0u;
        const long long anb_tt = *{self.ptr('t')};{resets}
        *{self.ptr('t')} = anb_tt + 1;
      }}
    }}
"""
        last_src = next((kk for kk in kernels if f" {plan[-1][0]}()" in kk), "") if plan else ""
        if not plan or [p[0] for p in plan].count(plan[-1][0]) > 1 or (len(plan[-1]) > 4 and plan[-1][4]) \
                or re.search(r"\breturn\b", last_src):
            # (a kernel that may return early cannot carry the step counter's epilogue)
            kernels.append("""
extern "C" __global__ void anb_tick() {
}
""")
            plan.append(("anb_tick", 1, 32, 0))
        kernels = self._append_epilogue(kernels, plan[-1][0], epilogue)
        stops = []
        for pop in net.populations:
            if getattr(pop, "stop_condition", None):
                code, mode_all = self.stop_kernel(pop)
                kernels.append(code)
                stops.append((pop.id, f"pop{pop.id}_stop", grid_for(pop.size), BLOCK, mode_all))
        # every kernel first waits for its predecessor on the stream (the plan
        # is launched with programmatic dependent launch)
        kernels = [re.sub(r'(extern "C" __global__ void (?:__launch_bounds__\([^)]*\) )?\w+\(\) \{)',
                          r"\1\n    anb_pdl_enter();", src) for src in kernels]
        return Module(self.assemble(kernels), self.options(), "grid", plan=plan,
                      kernels=[p[0] for p in plan], stops=stops)

    @staticmethod
    def _append_epilogue(kernels: list, name: str, code: str) -> list:
        """Insert `code` before the closing brace of kernel `name`."""
        out = []
        found = False
        for src in kernels:
            i = src.find(f" {name}(")
            if i >= 0 and not found:
                j = src.index("{", i)
                depth = 0
                for k in range(j, len(src)):
                    if src[k] == "{":
                        depth += 1
                    elif src[k] == "}":
                        depth -= 1
                        if depth == 0:
                            src = src[:k] + code + src[k:]
                            found = True
                            break
            out.append(src)
        if not found:
            raise RuntimeError(f"kernel {name} not found for the step epilogue")
        return out

    def local_module(self) -> Module:
        """One CTA holds every population's state in shared memory and runs
        many steps per launch."""
        net = self.net
        layout = self.c.local_layout
        block = layout["block"]
        smem_ptrs: dict[int, dict] = {}
        carve = []
        for pop in net.populations:
            d = {}
            for name, (off, ct) in layout["pops"][pop.id].items():
                carve.append(f"{ct}* __restrict__ anb_s_pop{pop.id}_{name} = "
                             f"reinterpret_cast<{ct}*>(anb_smem + {off});")
                d[name] = f"anb_s_pop{pop.id}_{name}"
            smem_ptrs[pop.id] = d
        load, store = [], []
        for pop in net.populations:
            for name, (off, ct) in layout["pops"][pop.id].items():
                n = (pop.size + 31) // 32 if name == "spk" else pop.size
                g = self.ptr(f"pop{pop.id}__{name}")
                s = smem_ptrs[pop.id][name]
                load.append(f"for (int q = threadIdx.x; q < {n}; q += blockDim.x) {s}[q] = {g}[q];")
                store.append(f"for (int q = threadIdx.x; q < {n}; q += blockDim.x) {g}[q] = {s}[q];")
        # propagation
        prop = []
        for proj in net.projections:
            lay = self.c.layout[proj.id]
            spk = smem_ptrs[proj.pre_pop.id]["spk"]
            gname = "g_" + proj.target
            g = smem_ptrs[proj.post_pop.id][gname]
            p = lambda n, k=proj.id: self.ptr(f"proj{k}__{n}")
            W = "double" if self.exact else self.c.wctype
            if self.exact:
                prop.append(f"""
      // {proj.name}: spikes in ascending pre rank; one barrier per spike keeps
      // the per-post accumulation order of the reference
      for (int word = {lay['w0']}; word < {lay['w1']}; ++word) {{
        anb_u32 m = {spk}[word];
        while (m) {{
          const int b = __ffs(m) - 1;
          m &= m - 1;
          const int pre = (word << 5) + b;
          const int beg = {p('col_ptr')}[pre], end = {p('col_ptr')}[pre + 1];
          if (end > beg) {{
            for (int q = beg + threadIdx.x; q < end; q += blockDim.x)
              {g}[{p('post_idx')}[q]] += {p('w_pre')}[q];
            __syncthreads();
          }}
        }}
      }}""")
            else:
                prop.append(f"""
      // {proj.name}: warp per 32-neuron word, shared-memory atomics
      for (int word = {lay['w0']} + anb_warp; word < {lay['w1']}; word += anb_nwarps) {{
        anb_u32 m = {spk}[word];
        while (m) {{
          const int b = __ffs(m) - 1;
          m &= m - 1;
          const int pre = (word << 5) + b;
          const int beg = {p('col_ptr')}[pre], end = {p('col_ptr')}[pre + 1];
          for (int q = beg + anb_lane; q < end; q += 32)
            atomicAdd(&{g}[{p('post_idx')}[q]], anb_wf({p('w_pre')}[q]));
        }}
      }}""")
        updates = []
        globals_ = []
        for pop in net.populations:
            globals_.append(self._globals_preamble(pop, lambda n, k=pop.id: self.ptr(f"pop{k}__{n}")))
            updates.append(self.neuron_update(pop, local_engine=True, smem=smem_ptrs[pop.id]))
        recs = []
        for mon in net.monitors:
            lay = self.c.mon_layout[mon.id]
            m = mon.id
            spk = smem_ptrs[mon.population.id]["spk"]
            recs.append(f"""
      if (anb_mon_on{m}) {{
        const long long anb_slot = t - anb_mon_t0{m};
        if (anb_slot >= 0 && anb_slot < {lay['cap_spike']}) {{
          anb_u32* anb_dst = {self.ptr(f'mon{m}__spk')} + anb_slot * {lay['words']};
          for (int q = threadIdx.x; q < {lay['words']}; q += blockDim.x) anb_dst[q] = {spk}[q];
        }} else if (threadIdx.x == 0) {{
          anb_report({self.ptr('err')}, ANB_DEVERR_MONITOR_OVERFLOW);
        }}
      }}""")
        mon_pre = "\n    ".join(
            f"const int anb_mon_on{mon.id} = {self.ptr(f'mon{mon.id}__on')}[0];\n    "
            f"const long long anb_mon_t0{mon.id} = {self.ptr(f'mon{mon.id}__t0')}[0];"
            for mon in net.monitors)
        dt_t = "double" if self.exact else "float"
        nl = "\n    "
        src = f"""
extern "C" __global__ void __launch_bounds__({block}, 1) anb_local_run(long long t0, int nsteps) {{
    extern __shared__ __align__(16) unsigned char anb_smem[];
    const {dt_t} dt = ({dt_t})(*{self.ptr('dt')});
    const int anb_lane = threadIdx.x & 31;
    const int anb_warp = threadIdx.x >> 5;
    const int anb_nwarps = blockDim.x >> 5;
    (void)anb_lane; (void)anb_warp; (void)anb_nwarps;
    {nl.join(carve)}
    {nl.join(g for g in globals_ if g)}
    {mon_pre}
    {nl.join(load)}
    __syncthreads();
    for (int anb_s = 0; anb_s < nsteps; ++anb_s) {{
      const long long t = t0 + anb_s;
      {''.join(prop)}
      __syncthreads();
      {''.join(updates)}
      __syncthreads();
      {''.join(recs)}
    }}
    __syncthreads();
    {nl.join(store)}
    if (threadIdx.x == 0) *{self.ptr('t')} = t0 + nsteps;
}}
"""
        return Module(self.assemble([src]), self.options(), "local",
                      local=("anb_local_run", 1, block, layout["smem"]), kernels=["anb_local_run"])

    def cluster_module(self) -> Module:
        """Spiking networks on the CTAs of one thread-block cluster.

        CTA r owns the neurons [r*chunk, (r+1)*chunk) of every population
        (chunk a multiple of 32) with their state in its shared memory, and
        the incoming synapses of those neurons (pre-major, per projection).
        Every CTA keeps a replica of each population's spike bitmap, double
        buffered by step parity. A step s:

          1. deliver the spikes of step s-1 (replica of parity (s-1)&1) into
             the own neurons' conductances: fast mode with shared-memory
             atomics, exact mode by one warp per conductance array, its
             projections in order and their spikes in ascending pre rank (a
             warp barrier after each spike), which is the reference's
             per-post order;
          2. update the own neurons and write the own bitmap words into the
             local replica of parity s&1 and into every other CTA's (DSMEM
             stores);
          3. one cluster barrier.

        Step s+1 writes the other replica, so the barrier of step s is the
        only one: nobody still reads a replica when it is overwritten."""
        net = self.net
        lay = self.c.cluster_layout
        C, block = lay["C"], lay["block"]
        carve, load, store = [], [], []
        smem_ptrs: dict[int, dict] = {}
        ranges = []
        for pop in net.populations:
            pl = lay["pops"][pop.id]
            chunk = pl["chunk"]
            k = pop.id
            d = {}
            for name, (off, ct) in pl["arrays"].items():
                carve.append(f"{ct}* __restrict__ anb_s_pop{k}_{name} = "
                             f"reinterpret_cast<{ct}*>(anb_smem + {off});")
                d[name] = f"anb_s_pop{k}_{name}"
            smem_ptrs[k] = d
            words = (pop.size + 31) // 32
            ranges.append(f"const int anb_base{k} = (int)anb_rank * {chunk};")
            ranges.append(f"const int anb_cnt{k} = max(0, min({pop.size}, anb_base{k} + {chunk}) - anb_base{k});")
            ranges.append(f"const int anb_words{k} = (anb_cnt{k} + 31) >> 5;")
            for name in pl["arrays"]:
                s_ = d[name]
                if name.startswith(("spk", "cp", "spl", "spn")):
                    continue
                if name.startswith("kc_"):
                    load.append(f"for (int q = threadIdx.x; q < anb_cnt{k}; q += blockDim.x) {s_}[q] = 0.f;")
                    continue
                g = self.ptr(f"pop{k}__{name}")
                load.append(f"for (int q = threadIdx.x; q < anb_cnt{k}; q += blockDim.x) {s_}[q] = {g}[anb_base{k} + q];")
                if name != "refractory":
                    store.append(f"for (int q = threadIdx.x; q < anb_cnt{k}; q += blockDim.x) {g}[anb_base{k} + q] = {s_}[q];")
            gspk = self.ptr(f"pop{k}__spk")
            # spikes of the step before the launch go to the replica of parity 1
            load.append(f"for (int q = threadIdx.x; q < {words}; q += blockDim.x) {{ {d['spk1']}[q] = {gspk}[q]; {d['spk0']}[q] = 0u; }}")
            store.append(f"for (int q = threadIdx.x; q < anb_words{k}; q += blockDim.x) "
                         f"{gspk}[(anb_base{k} >> 5) + q] = (nsteps & 1 ? {d['spk0']} : {d['spk1']})[(anb_base{k} >> 5) + q];")
        prop = []
        fast_groups: dict[int, list] = {}
        exact_groups: dict[tuple, list] = {}
        for proj in net.projections:
            a, b = proj.pre_pop.id, proj.post_pop.id
            play = self.c.layout[proj.id]
            cl = lay["proj"][proj.id]
            k = proj.id
            p = lambda n, kk=k: self.ptr(f"proj{kk}__{n}")
            lo, hi = play["w0"] * 32, play["w1"] * 32
            cp = smem_ptrs[a][f"cp{k}"]
            g = smem_ptrs[b]["g_" + proj.target]
            # this CTA's incoming synapses of projection k, appended to the pool
            palette = lay["pool"].get("palette")
            w_src = "anb_s_pool_w" if cl["w_smem"] else p("cl_w")
            w_idx = "q" if cl["w_smem"] else "anb_gbase{k} + q - anb_poff{k}".format(k=k)
            pool_w_src = p("cl_wi") if palette else p("cl_w")
            if palette:
                poff, npal = cl["pal"]
                wct = lay["pool"]["w_ct_real"]
                carve.append(f"{wct}* __restrict__ anb_s_pal{k} = reinterpret_cast<{wct}*>(anb_smem + {poff});")
                load.append(f"for (int q = threadIdx.x; q < {npal}; q += blockDim.x) anb_s_pal{k}[q] = {p('cl_pal')}[q];")
                w_src, w_idx = f"anb_s_pal{k}", "anb_s_pool_w[q]"
            load.append(f"""const int anb_gbase{k} = {p('cl_base')}[anb_rank];
    const int anb_poff{k} = anb_pool_off;
    {{
      const int anb_n = {p('cl_base')}[anb_rank + 1] - anb_gbase{k};
      for (int q = threadIdx.x; q <= {cl['span']}; q += blockDim.x)
        {cp}[q] = anb_pool_off + {p('cl_ptr')}[anb_rank * {cl['span'] + 1} + q];
      for (int q = threadIdx.x; q < anb_n; q += blockDim.x) {{
        anb_s_pool_post[anb_pool_off + q] = {p('cl_post')}[anb_gbase{k} + q];
        {"anb_s_pool_w[anb_pool_off + q] = " + pool_w_src + "[anb_gbase" + str(k) + " + q];" if cl["w_smem"] else ""}
      }}
      anb_pool_off += anb_n;
    }}""")
            deliver = (f"const int beg = {cp}[pre - {lo}], end = {cp}[pre - {lo} + 1];")
            spk = f"(anb_par ? {smem_ptrs[a]['spk0']} : {smem_ptrs[a]['spk1']})"
            if self.exact:
                # one warp per conductance array walks the nonzero words of the
                # projection's range in ascending order; the lanes add one
                # spike's synapses (distinct posts), then __syncwarp orders
                # them before the next spike: per post, ascending pre rank
                exact_groups.setdefault((b, proj.target), []).append(f"""
        {{  // {proj.name}: spikes in ascending pre rank
          const anb_u32* __restrict__ anb_spk = {spk};
          for (int c = {play['w0']}; c < {play['w1']}; c += 32) {{
            const anb_u32 anb_wv = (c + anb_lane < {play['w1']}) ? anb_spk[c + anb_lane] : 0u;
            anb_u32 anb_nz = __ballot_sync(0xffffffffu, anb_wv != 0u);
            while (anb_nz) {{
              const int j = __ffs(anb_nz) - 1;
              anb_nz &= anb_nz - 1;
              anb_u32 m = __shfl_sync(0xffffffffu, anb_wv, j);
              while (m) {{
                const int b = __ffs(m) - 1;
                m &= m - 1;
                const int pre = ((c + j) << 5) + b;
                {deliver}
                for (int q = beg + anb_lane; q < end; q += 32)
                  {g}[anb_s_pool_post[q]] += {w_src}[{w_idx}];
                __syncwarp();
              }}
            }}
          }}
        }}""")
            else:
                fast_groups.setdefault(a, []).append(f"""
          if (pre >= {lo} && pre < {hi}) {{  // {proj.name}
            {deliver}
            for (int q = beg + anb_lane; q < end; q += 32)
              atomicAdd(&{g}[anb_s_pool_post[q]], anb_wf({w_src}[{w_idx}]));
          }}""")
        if len(exact_groups) > lay["block"] // 32:
            raise ValueError("more conductance arrays than warps in the cluster engine")
        for gi, ((b, target), blocks) in enumerate(exact_groups.items()):
            prop.append(f"""
      if (anb_warp == {gi}) {{  // population {b}, g_{target}: projections in order{''.join(blocks)}
      }}""")
        for a, blocks in fast_groups.items():
            pop_a = next(pp for pp in net.populations if pp.id == a)
            W = (pop_a.size + 31) // 32
            ch = max(1, min(32, -(-W // (lay["block"] // 32))))
            spk = f"(anb_par ? {smem_ptrs[a]['spk0']} : {smem_ptrs[a]['spk1']})"
            prop.append(f"""
      {{  // population {a}: warp w scans its own {ch} bitmap words and delivers their
          // spikes with shared-memory atomics (lanes over the synapses)
        const anb_u32* __restrict__ anb_spk = {spk};
        for (int c0 = anb_warp * {ch}; c0 < {W}; c0 += anb_nwarps * {ch}) {{
          const anb_u32 anb_wv = (anb_lane < {ch} && c0 + anb_lane < {W}) ? anb_spk[c0 + anb_lane] : 0u;
          anb_u32 anb_nz = __ballot_sync(0xffffffffu, anb_wv != 0u);
          while (anb_nz) {{
            const int j = __ffs(anb_nz) - 1;
            anb_nz &= anb_nz - 1;
            anb_u32 m = __shfl_sync(0xffffffffu, anb_wv, j);
            while (m) {{
              const int b = __ffs(m) - 1;
              m &= m - 1;
              const int pre = ((c0 + j) << 5) + b;{''.join(blocks)}
            }}
          }}
        }}
      }}""")
        updates, globals_, bcast, recs = [], [], [], []
        for pop in net.populations:
            k = pop.id
            globals_.append(self._globals_preamble(pop, lambda n, kk=k: self.ptr(f"pop{kk}__{n}")))
            d = dict(smem_ptrs[k])
            # right after its ballot, a warp stores its bitmap word into every
            # CTA's replica (lane r -> CTA r) and one lane records it
            rec = ""
            for mon in net.monitors:
                if mon.population is not pop or "spike" not in mon.variables:
                    continue
                ml = self.c.mon_layout[mon.id]
                m = mon.id
                rec += f"""
          if (anb_lane == 31 && anb_mon_on{m}) {{
            const long long anb_slot = t - anb_mon_t0{m};
            if (anb_slot >= 0 && anb_slot < {ml['cap_spike']})
              {self.ptr(f'mon{m}__spk')}[anb_slot * {ml['words']} + anb_gw] = anb_m;
            else
              anb_report({self.ptr('err')}, ANB_DEVERR_MONITOR_OVERFLOW);
          }}"""
            hook = f"""
      {{
        const anb_u32 anb_m = __ballot_sync(0xffffffffu, anb_spiked);
        if (anb_q - anb_lane < anb_cnt) {{
          const int anb_gw = (anb_base >> 5) + (anb_q >> 5);
          anb_u32* anb_dstw = (anb_par ? {d['spk1']} : {d['spk0']}) + anb_gw;
          if (anb_lane == (int)anb_rank) *anb_dstw = anb_m;
          else if (anb_lane < {C}) anb_cluster_st_u32(anb_cluster_map(anb_smem_addr(anb_dstw), (unsigned)anb_lane), anb_m);{rec}
        }}
      }}"""
            updates.append(self.neuron_update(pop, local_engine=True, smem=d, cluster={},
                                              ballot_hook=hook))
        mon_pre = "\n    ".join(
            f"const int anb_mon_on{mon.id} = {self.ptr(f'mon{mon.id}__on')}[0];\n    "
            f"const long long anb_mon_t0{mon.id} = {self.ptr(f'mon{mon.id}__t0')}[0];"
            for mon in net.monitors)
        (poff, pct), (woff, wct) = lay["pool"]["post"], lay["pool"]["w"]
        pool_carve = f"{pct}* __restrict__ anb_s_pool_post = reinterpret_cast<{pct}*>(anb_smem + {poff});"
        if woff is not None:
            pool_carve += f"\n    {wct}* __restrict__ anb_s_pool_w = reinterpret_cast<{wct}*>(anb_smem + {woff});"
        dt_t = "double" if self.exact else "float"
        nl = "\n    "
        src = f"""
extern "C" __global__ void __launch_bounds__({block}, 1)
anb_cluster_run(long long t0, int nsteps) {{
    extern __shared__ __align__(16) unsigned char anb_smem[];
    const unsigned anb_rank = anb_cluster_rank();
    const {dt_t} dt = ({dt_t})(*{self.ptr('dt')});
    const int anb_lane = threadIdx.x & 31;
    const int anb_warp = threadIdx.x >> 5;
    const int anb_nwarps = blockDim.x >> 5;
    (void)anb_lane; (void)anb_warp; (void)anb_nwarps;
    {nl.join(carve)}
    {pool_carve}
    {nl.join(ranges)}
    {nl.join(g for g in globals_ if g)}
    {mon_pre}
    int anb_pool_off = 0;
    {nl.join(load)}
    (void)anb_pool_off;
    anb_cluster_sync();
    for (int anb_s = 0; anb_s < nsteps; ++anb_s) {{
      const long long t = t0 + anb_s;
      const int anb_par = anb_s & 1;
      {''.join(prop)}
      __syncthreads();
      {''.join(updates)}
      anb_cluster_sync();
    }}
    {nl.join(store)}
    if (anb_rank == 0 && threadIdx.x == 0) *{self.ptr('t')} = t0 + nsteps;
}}
"""
        return Module(self.assemble([src]), self.options(), "cluster",
                      local=("anb_cluster_run", C, block, lay["smem"], C), kernels=["anb_cluster_run"])

    # ------------------------------------------------------------------ output
    def options(self) -> list:
        opts = ["-diag-suppress=177"]
        if self.exact:
            opts.append("--fmad=false")
        cuda_inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
        if os.path.isdir(cuda_inc):
            opts.append("-I" + cuda_inc)
        return opts

    def user_functions(self) -> str:
        """Device functions of the user functions the network's models use
        (global ones from add_function, then the models' own)."""
        from ..parser.equation import GLOBAL_FUNCTIONS
        funcs: dict = {}
        for f in GLOBAL_FUNCTIONS.values():
            funcs[f["name"]] = f
        for obj in list(self.net.populations) + list(self.net.projections):
            for f in obj.desc.get("functions", []):
                if f["name"] in funcs and funcs[f["name"]]["cpp"] != f["cpp"]:
                    raise ValueError(f"two different functions named {f['name']!r}")
                funcs[f["name"]] = f
        out = []
        for f in funcs.values():
            args = ", ".join(f"{self.real} {a}" for a in f["args"])
            out.append(f"__device__ __forceinline__ {self.real} {f['name']}({args}) {{ "
                       f"return {self.typed(f['cpp'])}; }}")
        return ("\n" + "\n".join(out)) if out else ""

    def assemble(self, kernels: list) -> str:
        header = open(DEVICE_HEADER).read()
        self.ptr("t")
        self.ptr("dt")
        self.ptr("err")
        decl = "\n".join(f"__constant__ {ct}* anb_p_{name};" for name, ct in sorted(self.decls.items()))
        decl += self.user_functions()
        # network constants usable in every equation (set through anb_module_set_constant);
        # an attribute of the same name hides them, as in the reference
        consts = "".join(f"__constant__ {self.real} {c};\n" for c in sorted(self.net._constants))
        types = "".join(self.types[k] for k in sorted(self.types))
        return (f"// generated by annarchy_b200 for network {self.net.id}\n{header}\n"
                f"typedef {self.real} real;\n{types}{consts}{decl}\n" + "".join(kernels))
