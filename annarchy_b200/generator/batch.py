"""CUDA source of the batched-instance engine.

Many independent spiking networks of one structure (the same neuron and
synapse equations, populations and projections; sizes, parameter values,
connectivity and weights free per instance) run in ONE persistent launch.
Every CTA owns a set of whole instances whose state sits in its shared
memory for the whole launch; the instances of a CTA are packed so that the
CTAs of the launch carry about the same number of neurons and synapses.
Instances never exchange data, so the only barriers are the CTA's own:

    for every step:
        deliver the spikes of the previous step of every own instance
        (fast: shared-memory atomics; exact: spike by spike in ascending pre
        rank with one CTA barrier per spike, the reference's per-post order)
        __syncthreads
        update every own instance's neurons, spike bitmap words by ballot
        (and into the spike monitor ring)
        __syncthreads

Per-instance quantities come from small tables indexed by the instance's
slot (its position in the packed order): population sizes, offsets into the
concatenated global arrays, the shared-memory offset of every state array,
global parameter values and the word range of each projection's pre ranks.
A launch copies each slot's row of these tables once into a header at the
start of the CTA's shared memory, so that the steps read none of them from
global memory.

The per-step semantics are the single-network ones of the reference's
generated core (ANNarchy/generator/Template/OpenMPBaseTemplate.py:131-484),
repeated per instance; the reference runs such sweeps as separate processes
(Network.parallel_run, ANNarchy/core/Network.py:751-900).
"""
from __future__ import annotations

import numpy as np

from .codegen import CodeGenerator, Module

BATCH_BLOCK = 1024


class BatchGenerator(CodeGenerator):
    """`batch` provides .net (the template network, instance 0), .exact,
    .native (the device arrays), .smem_arrays ({pop id: [(name, ctype)]}),
    .n_arrays, .array_index ({(pop id, name): column of the offset table}),
    .n_cta, .smem, .idx_t and .packed (projection id -> packed synapse
    words)."""

    def __init__(self, batch):
        super().__init__(batch)
        self.b = batch

    def compensated(self, pop) -> list:
        from .codegen import compensated_vars
        return compensated_vars(pop, self.exact, self.b.comp_config(pop))

    def _hptr(self, key, slot="anb_si") -> str:
        """Pointer to the shared-memory copy of a per-slot quantity (the
        header slots sit at the start of the CTA's shared memory)."""
        if not hasattr(self, "_hpos"):
            longs, reals, ints, self._hbytes = self.b.header_layout()
            self._hpos, off = {}, 0
            for entries, ct, size in ((longs, "long long", 8), (reals, self.real, 8 if self.exact else 4),
                                      (ints, "int", 4)):
                for e in entries:
                    self._hpos[e[0]] = (ct, off)
                    off += size
        ct, off = self._hpos[key]
        return f"reinterpret_cast<const {ct}*>(anb_smem + ({slot} - anb_sb) * {self._hbytes} + {off})"

    def _hx(self, key, slot="anb_si") -> str:
        return f"{self._hptr(key, slot)}[0]"

    def _header_fill(self) -> str:
        """One thread per slot of the CTA copies the slot's row of every
        per-slot table into the slot's header."""
        longs, reals, ints, _ = self.b.header_layout()
        self._hptr(longs[0][0] if longs else ints[0][0])
        lines = []
        for key, arr, stride, col in longs + reals + ints:
            ct, _ = self._hpos[key]
            idx = "anb_si" if stride == 1 else f"anb_si * {stride} + {col}"
            dst = self._hptr(key).replace("const ", "", 1)
            lines.append(f"{dst}[0] = {self.ptr(arr)}[{idx}];")
        nl = "\n      "
        return f"""
    for (int anb_si = anb_sb + threadIdx.x; anb_si < anb_se; anb_si += blockDim.x) {{
      {nl.join(lines)}
    }}
    __syncthreads();"""

    def _pop_gsrc(self, k):
        return lambda name: f"({self.ptr(f'pop{k}__{name}')} + anb_goff{k})"

    def _smem_ptrs(self, pop) -> tuple[list, dict]:
        k = pop.id
        lines, d = [], {}
        for name, ct in self.b.smem_arrays[k]:
            col = self.b.array_index[(k, name)]
            var = f"anb_s{k}_{name}"
            lines.append(f"{ct}* __restrict__ {var} = reinterpret_cast<{ct}*>(anb_smem + anb_so[{col}]);")
            d[name] = var
        return lines, d

    def _instance_header(self, pops) -> str:
        out = [f"const int* __restrict__ anb_so = {self._hptr('so0')};"]
        for pop in pops:
            k = pop.id
            out.append(f"const int anb_n{k} = {self._hx(f'n{k}')};")
            out.append(f"const long long anb_goff{k} = {self._hx(f'goff{k}')};")
            out.append(f"const long long anb_woff{k} = {self._hx(f'woff{k}')};")
            out.append(f"(void)anb_n{k}; (void)anb_goff{k}; (void)anb_woff{k};")
        return "\n      ".join(out)

    def _copy(self, pop, to_smem: bool) -> str:
        k = pop.id
        lines, d = self._smem_ptrs(pop)
        body = []
        for name, ct in self.b.smem_arrays[k]:
            if name == "spk":
                g = f"{self.ptr(f'pop{k}__spk')}[anb_woff{k} + q]"
                n = f"((anb_n{k} + 31) >> 5)"
            else:
                g = f"{self.ptr(f'pop{k}__{name}')}[anb_goff{k} + q]"
                n = f"anb_n{k}"
            if to_smem:
                body.append(f"for (int q = threadIdx.x; q < {n}; q += blockDim.x) {d[name]}[q] = {g};")
            else:
                body.append(f"for (int q = threadIdx.x; q < {n}; q += blockDim.x) {g} = {d[name]}[q];")
        nl = "\n        "
        return f"""
      {{  // population {pop.name}
        {nl.join(lines)}
        {nl.join(body)}
      }}"""

    def _delivery_exact(self, proj) -> str:
        """Exact mode: the spikes of the projection in ascending pre rank, one
        CTA barrier after each, so every post neuron adds its inputs in the
        reference's order (ANNarchy/generator/Projection/OpenMP/CSR.py:870-902)."""
        k = proj.id
        a, b = proj.pre_pop.id, proj.post_pop.id
        spk_col = self.b.array_index[(a, "spk")]
        g_col = self.b.array_index[(b, "g_" + proj.target)]
        it = self.b.idx_t
        cp = self.ptr(f"proj{k}__col_ptr")
        post, w = self.ptr(f"proj{k}__post"), self.ptr(f"proj{k}__w")
        return f"""
      {{  // {proj.name}: spikes in ascending pre rank, one CTA barrier per spike
        const anb_u32* __restrict__ anb_spk = reinterpret_cast<const anb_u32*>(anb_smem + anb_so[{spk_col}]);
        real* __restrict__ anb_g = reinterpret_cast<real*>(anb_smem + anb_so[{g_col}]);
        const int anb_w0 = {self._hx(f'wr{k}_0')};
        const int anb_w1 = {self._hx(f'wr{k}_1')};
        const {it}* __restrict__ anb_cp = {cp} + {self._hx(f'cp{k}')};
        for (int word = anb_w0; word < anb_w1; ++word) {{
          anb_u32 m = anb_spk[word];
          while (m) {{
            const int pre = (word << 5) + __ffs(m) - 1;
            m &= m - 1;
            const {it} beg = anb_cp[pre], end = anb_cp[pre + 1];
            if (end > beg) {{
              for ({it} q = beg + threadIdx.x; q < end; q += blockDim.x)
                anb_g[{post}[q]] += {w}[q];
              __syncthreads();
            }}
          }}
        }}
      }}"""

    def _scratch(self, spk_pops) -> str:
        """Fast-mode scratch after the instances' state: 32 warp sums, the
        spike-list counter, the list, and per projection the list entries'
        synapse ranges (begin, end)."""
        it = self.b.idx_t
        cap = self.b.list_cap
        lines = [f"int* __restrict__ anb_scan = reinterpret_cast<int*>(anb_smem + {self.b.smem_state});",
                 "int* __restrict__ anb_lcnt = anb_scan + 32;  // by step parity",
                 "int* __restrict__ anb_list = anb_scan + 36;"]
        off = self.b.smem_state + 4 * (36 + cap)
        for proj in self.net.projections:
            if proj.pre_pop not in spk_pops:
                continue
            k = proj.id
            for end in ("b", "e"):
                lines.append(f"{it}* __restrict__ anb_l{end}{k} = reinterpret_cast<{it}*>(anb_smem + {off});")
                off += cap * (8 if it == "long long" else 4)
        assert off <= self.b.smem, (off, self.b.smem)
        return "\n    ".join(lines)

    def _append_spikes(self, pop, spk_pops) -> str:
        """Fast mode, inside the update's ballot: the warp's spikes are
        appended to the CTA's list for the next step's delivery, each with its
        synapse range in every projection leaving the population (the column
        pointers are read here, where their latency hides behind the other
        warps' updates), and the range's synapse words are prefetched into L2."""
        if self.exact or pop not in spk_pops:
            return ""
        pi = spk_pops.index(pop)
        P = len(spk_pops)
        cap = self.b.list_cap
        it = self.b.idx_t
        per = []
        for proj in self.net.projections:
            if proj.pre_pop is not pop:
                continue
            k = proj.id
            cp = f"({self.ptr(f'proj{k}__col_ptr')} + {self._hx(f'cp{k}')})"
            if self.b.packed.get(k):
                pref = [(self.ptr(f"proj{k}__syn"), 4)]
            else:
                pref = [(self.ptr(f"proj{k}__post"), 4)]
                wsize = {np.float64: 8, np.float32: 4}.get(self.b.wdtype, 2)
                pref.append((self.ptr(f"proj{k}__w"), wsize))
            pf = []
            for arr, size in pref:
                # aligned to 16 bytes on both ends; the arrays are padded so
                # that the rounded end stays inside them
                g = 16 // size if size < 16 else 1
                pf.append(f"anb_prefetch_l2({arr} + (anb_b & ~({it}){g - 1}), "
                          f"(unsigned)((((anb_e + {g - 1}) & ~({it}){g - 1}) - (anb_b & ~({it}){g - 1})) * {size}));")
            per.append(f"""
              {{
                const {it} anb_b = {cp}[anb_i], anb_e = {cp}[anb_i + 1];
                anb_lb{k}[anb_q] = anb_b;
                anb_le{k}[anb_q] = anb_e;
                if (anb_e > anb_b) {{ {' '.join(pf)} }}
              }}""")
        return f"""
        if (anb_m) {{
          int anb_q0 = 0;
          if ((threadIdx.x & 31) == 0) anb_q0 = atomicAdd(anb_lcnt + (t & 1), __popc(anb_m));
          anb_q0 = __shfl_sync(0xffffffffu, anb_q0, 0);
          if (anb_spiked) {{
            const int anb_q = anb_q0 + __popc(anb_m & ((1u << (threadIdx.x & 31)) - 1u));
            if (anb_q < {cap}) {{
              anb_list[anb_q] = (((anb_si - anb_sb) * {P} + {pi}) << 16) | anb_i;{''.join(per)}
            }}
          }}
        }}"""

    def _delivery_list(self, spk_pops) -> str:
        """Fast mode. The previous step's update appended every spike of the
        CTA's instances to a list in shared memory with its synapse ranges;
        when more spikes came than the list holds (or at the first step of a
        launch) the list is rebuilt from the spike bitmaps instead (each
        thread holds one bitmap word; a CTA prefix sum of the popcounts gives
        every spike its slot), LIST_CAP entries per round. Warp w then
        delivers entries 4w..4w+3 (+128 per pass): the four spikes' synapse
        ranges are read as aligned 4-synapse groups (16-byte loads), lane l
        taking group l of each, all four loads in flight before the
        shared-memory atomics. A burst of spikes in one instance is spread
        over all warps of the CTA."""
        P = len(spk_pops)
        it = self.b.idx_t
        cap = self.b.list_cap
        find = []
        for pi, pop in enumerate(spk_pops):
            k = pop.id
            col = self.b.array_index[(k, "spk")]
            find.append(f"""
          {{
            const int anb_W = ({self._hx(f'n{k}')} + 31) >> 5;
            const int anb_r = (int)threadIdx.x - anb_base;
            if (anb_r >= 0 && anb_r < anb_W) {{
              anb_lw = reinterpret_cast<const anb_u32*>(anb_smem + {self._hx(f'so{col}')})[anb_r];
              anb_lpair = (anb_si - anb_sb) * {P} + {pi};
              anb_lword = anb_r;
            }}
            anb_base += anb_W;
          }}""")
        projs = []
        for proj in self.net.projections:
            pi = spk_pops.index(proj.pre_pop)
            k = proj.id
            g_col = self.b.array_index[(proj.post_pop.id, "g_" + proj.target)]
            U = 4 if self.b.packed.get(k) else 2
            if self.b.packed.get(k):
                syn = self.ptr(f"proj{k}__syn")
                load = f"anb_v[u] = anb_ls_u4(reinterpret_cast<const uint4*>({syn}) + anb_g);"
                regs = "uint4 anb_v[4];"
                add = ("ANB_ADD(anb_v[u].x, 0) ANB_ADD(anb_v[u].y, 1) "
                       "ANB_ADD(anb_v[u].z, 2) ANB_ADD(anb_v[u].w, 3)")
                macro = ("#define ANB_ADD(sw, c) if (anb_g * 4 + c >= anb_bq[u] && anb_g * 4 + c < anb_eq[u]) "
                         "atomicAdd(reinterpret_cast<real*>(anb_smem + anb_go[u]) + ((sw) >> 16), __uint_as_float((sw) << 16));")
            else:
                post, w = self.ptr(f"proj{k}__post"), self.ptr(f"proj{k}__w")
                load = (f"anb_p4[u] = anb_ls_i4(reinterpret_cast<const int4*>({post}) + anb_g); "
                        f"anb_w4v[u] = anb_w4({w} + anb_g * 4);")
                regs = "int4 anb_p4[2]; float4 anb_w4v[2];"
                add = ("ANB_ADD(anb_p4[u].x, anb_w4v[u].x, 0) ANB_ADD(anb_p4[u].y, anb_w4v[u].y, 1) "
                       "ANB_ADD(anb_p4[u].z, anb_w4v[u].z, 2) ANB_ADD(anb_p4[u].w, anb_w4v[u].w, 3)")
                macro = ("#define ANB_ADD(po, wv, c) if (anb_g * 4 + c >= anb_bq[u] && anb_g * 4 + c < anb_eq[u]) "
                         "atomicAdd(reinterpret_cast<real*>(anb_smem + anb_go[u]) + (po), wv);")
            projs.append(f"""
          {{  // {proj.name}
           {it} anb_bq1 = 0, anb_eq1 = 0;
           int anb_go1 = 0;
           if (anb_ent >= 0 && anb_epop == {pi}) {{
             if (anb_fromlist) {{
               anb_bq1 = anb_lb{k}[anb_e0 + anb_lane];
               anb_eq1 = anb_le{k}[anb_e0 + anb_lane];
             }} else {{
               const {it}* __restrict__ anb_cp = {self.ptr(f'proj{k}__col_ptr')} + {self._hx(f'cp{k}', 'anb_eslot')};
               anb_bq1 = anb_cp[anb_rank];
               anb_eq1 = anb_cp[anb_rank + 1];
             }}
             anb_go1 = {self._hx(f'so{g_col}', 'anb_eslot')};
           }}
           for (int anb_sub = 0; anb_sub < 4; anb_sub += {U}) {{
            {it} anb_bq[{U}], anb_eq[{U}];
            int anb_go[{U}];
            {it} anb_ng = 0;
            #pragma unroll
            for (int u = 0; u < {U}; ++u) {{
              anb_bq[u] = __shfl_sync(0xffffffffu, anb_bq1, anb_sub + u);
              anb_eq[u] = __shfl_sync(0xffffffffu, anb_eq1, anb_sub + u);
              anb_go[u] = __shfl_sync(0xffffffffu, anb_go1, anb_sub + u);
              const {it} n = anb_eq[u] > anb_bq[u] ? ((anb_eq[u] + 3) >> 2) - (anb_bq[u] >> 2) : 0;
              anb_ng = n > anb_ng ? n : anb_ng;
            }}
            for ({it} anb_p = anb_lane; anb_p - anb_lane < anb_ng; anb_p += 32) {{
              {regs}
              #pragma unroll
              for (int u = 0; u < {U}; ++u) {{
                const {it} anb_g = (anb_bq[u] >> 2) + anb_p;
                if (anb_eq[u] > anb_bq[u] && anb_g < ((anb_eq[u] + 3) >> 2)) {{ {load} }}
              }}
              #pragma unroll
              for (int u = 0; u < {U}; ++u) {{
                const {it} anb_g = (anb_bq[u] >> 2) + anb_p;
                if (anb_eq[u] > anb_bq[u] && anb_g < ((anb_eq[u] + 3) >> 2)) {{
{macro}
                  {add}
#undef ANB_ADD
                }}
              }}
            }}
           }}
          }}""")
        return f"""
      {{  // delivery: CTA-wide list of the previous step's spikes
        // the previous step's counter; this step's update counts into the
        // other one (last read by the previous step's delivery)
        const int anb_cnt = anb_lcnt[(t - 1) & 1];
        const bool anb_fromlist = anb_cnt <= {cap};
        if (threadIdx.x == 0) anb_lcnt[t & 1] = 0;
        anb_u32 anb_lw = 0u;
        int anb_lpair = 0, anb_lword = 0;
        int anb_total = anb_cnt, anb_excl = 0;
        if (!anb_fromlist) {{
          int anb_base = 0;
          for (int anb_si = anb_sb; anb_si < anb_se; ++anb_si) {{{''.join(find)}
          }}
          anb_excl = anb_block_exclusive_scan(__popc(anb_lw), anb_scan, &anb_total);
        }}
        for (int anb_r0 = 0; anb_r0 < anb_total; anb_r0 += {cap}) {{
          if (!anb_fromlist) {{
            int k = anb_excl;
            anb_u32 m = anb_lw;
            while (m) {{
              const int b = __ffs(m) - 1;
              m &= m - 1;
              if (k >= anb_r0 && k < anb_r0 + {cap})
                anb_list[k - anb_r0] = (anb_lpair << 16) | ((anb_lword << 5) + b);
              ++k;
            }}
            __syncthreads();
          }}
          const int anb_nl = min({cap}, anb_total - anb_r0);
          for (int anb_e0 = anb_warp * 4; anb_e0 < anb_nl; anb_e0 += anb_nwarps * 4) {{
            const int anb_ent = (anb_lane < 4 && anb_e0 + anb_lane < anb_nl) ? anb_list[anb_e0 + anb_lane] : -1;
            const int anb_pair = anb_ent >> 16;
            const int anb_rank = anb_ent & 0xffff;
            const int anb_eslot = anb_sb + (anb_ent >= 0 ? anb_pair / {P} : 0);
            const int anb_epop = anb_ent >= 0 ? anb_pair % {P} : -1;
            (void)anb_rank; (void)anb_eslot;{''.join(projs)}
          }}
          // before the next round's list (the step's own barrier follows the last)
          if (anb_r0 + {cap} < anb_total) __syncthreads();
        }}
      }}"""

    def _spk_pops(self) -> list:
        """Populations with outgoing projections (their spikes are delivered)."""
        return [p for p in self.net.populations if any(pr.pre_pop is p for pr in self.net.projections)]

    def _record(self) -> str:
        """Spike monitors, after the update's barrier: the step's bitmap words
        of every instance of the CTA copied from shared memory into the
        monitor's ring, one thread per word."""
        out = []
        for mon in self.net.monitors:
            if "spike" not in mon.variables:
                continue
            m, k = mon.id, mon.population.id
            col = self.b.array_index[(k, "spk")]
            out.append(f"""
      if (anb_mon_on{m}) {{  // spike monitor {m}
        const long long anb_slot = t - anb_mon_t0{m};
        if (anb_slot >= 0 && anb_slot < {self.b.mon_cap[m]}) {{
          for (int anb_si = anb_sb; anb_si < anb_se; ++anb_si) {{
            const int anb_W = ({self._hx(f'n{k}')} + 31) >> 5;
            const anb_u32* __restrict__ anb_w = reinterpret_cast<const anb_u32*>(anb_smem + {self._hx(f'so{col}')});
            anb_u32* __restrict__ anb_dst = {self.ptr(f'mon{m}__spk')} + anb_slot * {self.b.total_words[k]}LL + {self._hx(f'woff{k}')};
            for (int q = threadIdx.x; q < anb_W; q += blockDim.x) anb_dst[q] = anb_w[q];
          }}
        }} else if (threadIdx.x == 0) {{
          anb_report({self.ptr('err')}, ANB_DEVERR_MONITOR_OVERFLOW);
        }}
      }}""")
        return "".join(out)

    def _update(self, pop) -> str:
        k = pop.id
        lines, d = self._smem_ptrs(pop)
        hook = f"""
      {{
        const anb_u32 anb_m = __ballot_sync(0xffffffffu, anb_spiked);
        if ((threadIdx.x & 31) == 0 && anb_i < anb_n)
          {d['spk']}[anb_i >> 5] = anb_m;{self._append_spikes(pop, self._spk_pops())}
      }}"""
        globals_ = self._globals_preamble(pop, lambda n: self._hptr(f"p{k}_{n}"))
        globals_ += f"\n    const int anb_refr{k} = {self._hx(f'refr{k}')};"
        # a refractory period shared by all neurons of the instance comes from
        # the slot table (no global load in the spike branch)
        refr = (f"(anb_refr{k} >= 0 ? anb_refr{k} : "
                f"({self.ptr(f'pop{k}__refractory')} + anb_goff{k})[anb_i])")
        upd = self.neuron_update(pop, local_engine=True, smem=d, ballot_hook=hook,
                                 size=f"anb_n{k}", gsrc=self._pop_gsrc(k), refractory=refr)
        nl = "\n        "
        return f"""
      {{
        {nl.join(lines)}
        {globals_}
        {upd}
      }}"""

    def module(self) -> Module:
        net = self.net
        pops = net.populations
        for pop in pops:
            if pop.neuron_type.type != "spike":
                raise NotImplementedError("batched instances hold spiking populations only")
        mon_pre = "\n    ".join(
            f"const int anb_mon_on{mon.id} = {self.ptr(f'mon{mon.id}__on')}[0];\n    "
            f"const long long anb_mon_t0{mon.id} = {self.ptr(f'mon{mon.id}__t0')}[0];\n    "
            f"(void)anb_mon_on{mon.id}; (void)anb_mon_t0{mon.id};"
            for mon in net.monitors)
        header = self._instance_header(pops)
        load = "".join(self._copy(p, True) for p in pops)
        store = "".join(self._copy(p, False) for p in pops)
        spk_pops = self._spk_pops()
        if self.exact:
            deliver = (f"for (int anb_si = anb_sb; anb_si < anb_se; ++anb_si) {{\n        {header}"
                       + "".join(self._delivery_exact(pr) for pr in net.projections) + "\n      }")
        elif spk_pops:
            deliver = self._delivery_list(spk_pops)
        else:
            deliver = ""
        update = "".join(self._update(p) for p in pops)
        dt_t = "double" if self.exact else "float"
        scratch = "" if self.exact or not spk_pops else self._scratch(spk_pops)
        if scratch:
            # no list at the first step of a launch: the delivery rebuilds it
            # from the spike bitmaps
            scratch += f"\n    if (threadIdx.x == 0) anb_lcnt[0] = anb_lcnt[1] = {self.b.list_cap} + 1;"
        src = f"""
extern "C" __global__ void __launch_bounds__({BATCH_BLOCK}, 1)
anb_batch_run(long long t0, int nsteps) {{
    extern __shared__ __align__(16) unsigned char anb_smem[];
    const {dt_t} dt = ({dt_t})(*{self.ptr('dt')});
    const int anb_lane = threadIdx.x & 31;
    const int anb_warp = threadIdx.x >> 5;
    const int anb_nwarps = blockDim.x >> 5;
    (void)anb_lane; (void)anb_warp; (void)anb_nwarps;
    const int anb_sb = {self.ptr('bt__cta')}[blockIdx.x];
    const int anb_se = {self.ptr('bt__cta')}[blockIdx.x + 1];
    {scratch}
    {mon_pre}
    {self._header_fill()}
    for (int anb_si = anb_sb; anb_si < anb_se; ++anb_si) {{
      {header}
      {load}
    }}
    __syncthreads();
    for (int anb_s = 0; anb_s < nsteps; ++anb_s) {{
      const long long t = t0 + anb_s;
      {deliver}
      __syncthreads();
      for (int anb_si = anb_sb; anb_si < anb_se; ++anb_si) {{
        {header}
        {update}
      }}
      __syncthreads();{self._record()}
    }}
    for (int anb_si = anb_sb; anb_si < anb_se; ++anb_si) {{
      {header}
      {store}
    }}
    if (blockIdx.x == 0 && threadIdx.x == 0) *{self.ptr('t')} = t0 + nsteps;
}}
"""
        return Module(self.assemble([src]), self.options(), "batch",
                      local=("anb_batch_run", self.b.n_cta, BATCH_BLOCK, self.b.smem),
                      kernels=["anb_batch_run"])
