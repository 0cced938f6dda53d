"""The reference simulator's compiled network module, served by this backend.

The reference (ANNarchy 5.0.3) generates one extension module per network,
``ANNarchyWrapper<id>`` (ANNarchy/generator/NanoBind/Generator.py:18-434,
template ANNarchy/generator/NanoBind/BaseTemplate.py:1-45), loads it in
``Compiler._instantiate`` (ANNarchy/generator/Compiler.py:796-1000) and from
then on drives the simulation only through it: ``set_seed``,
``pyx_create``, ``pyx_initialize``, ``run``, ``run_until``, ``step``,
``set_time``/``get_time``, ``estimate_record_size``, ``set_<constant>``, and
per object ``pop<k>_wrapper`` (attribute properties, refractory, reset),
``proj<k>_wrapper`` (``init_from_lil``, connectivity queries, attribute
getters and setters per locality) and ``PopRecorder<k>_wrapper``
(``record_<var>`` switches, recorded data, ``clear_<var>``).

``ReferenceModule`` is that module with the same names, arguments and
return shapes, implemented over this backend's C ABI
(include/annarchy_b200.h) through ``annarchy_b200.Network``. ``instantiate``
plugs it into a network built with the reference's own Python API: it runs
the reference's ``Compiler._instantiate`` with this module in place of the
library it would have built, so the reference's Population, Projection,
Monitor and simulate() code run unchanged on the B200 kernels. This is the
binding a maintainer adds for a ``paradigm="b200"`` (the reference's hook
points: ANNarchy/intern/ConfigManagement.py:14-46,
ANNarchy/generator/CodeGenerator.py:88-112, Compiler.py:703-723 and
:828-905); no file of the reference is modified.

Errors follow the reference's convention: ``init_from_lil`` returns False on
invalid connectivity instead of raising.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def _ref_neuron_args(nt) -> dict:
    return dict(parameters=nt.parameters, equations=nt.equations, spike=nt.spike,
                reset=nt.reset, refractory=nt.refractory, name=getattr(nt, "name", ""))


def _ref_synapse_args(st) -> dict:
    out = {}
    for k in ("parameters", "equations", "psp", "pre_spike", "post_spike", "name"):
        v = getattr(st, k, None)
        if v not in (None, ""):
            out[k] = v
    op = getattr(st, "operation", "sum")
    if op and op != "sum":
        out["operation"] = op
    return out


class _PopWrapper:
    """pop<k>_wrapper(size, max_delay): the population's attributes as
    properties (a list for local attributes, a float for global ones),
    refractory periods in steps, reset/activate/clear
    (ANNarchy/generator/NanoBind/Population.py:27-54)."""

    def __init__(self, module, pop, size: int, max_delay: int):
        object.__setattr__(self, "_m", module)
        object.__setattr__(self, "_pop", pop)
        object.__setattr__(self, "size", int(size))
        object.__setattr__(self, "max_delay", int(max_delay))
        object.__setattr__(self, "refractory_dirty", False)

    def _names(self):
        return self._pop._host

    def __getattr__(self, name):
        if name.startswith("_") and not name.startswith("_sum_"):
            raise AttributeError(name)
        if name.startswith("_sum_") or name in self._names():
            v = self._pop.sum(name[5:]) if name.startswith("_sum_") else self._pop.get(name)
            if np.ndim(v) == 0:
                return float(v)
            return np.asarray(v).reshape(-1).tolist()
        raise AttributeError(f"pop{self._pop.id}_wrapper has no attribute {name!r}")

    def __setattr__(self, name, value):
        if name == "refractory":
            # the reference passes whole steps (int(refractory / dt), truncated)
            self._pop._set_refractory_steps(np.asarray(value, dtype=np.int32).reshape(-1))
            return
        if name in ("refractory_dirty", "max_delay"):
            object.__setattr__(self, name, value)
            return
        if name in self._names():
            v = np.asarray(value, dtype=np.float64)
            self._pop.set({name: v.reshape(-1) if v.ndim else float(v)})
            return
        raise AttributeError(f"pop{self._pop.id}_wrapper has no attribute {name!r}")

    def get_refractory(self):
        return self._pop.refractory_steps.tolist()

    def compute_firing_rate(self, window: float):
        """The reference's sliding-window mean rate; a window <= 0 (the
        default, -1) disables it."""
        if window > 0:
            raise NotImplementedError("compute_firing_rate is not supported by this backend")

    def activate(self, enabled: bool):
        if not enabled:
            raise NotImplementedError("disabled populations are not supported by this backend")

    def reset(self):
        """Spike state back to its initial value (the reference's
        PopStruct::reset()): refractory counters, last spike, spike bitmaps."""
        if self._m._net.compiled:
            self._m._net._backend.reset_spike_state(self._pop)

    def clear(self):
        pass

    def device_to_host(self, *args):
        pass

    def size_in_bytes(self) -> int:
        return int(sum(np.asarray(a).nbytes for a in self._pop._host.values()))

    def update_max_delay(self, d: int):
        object.__setattr__(self, "max_delay", int(d))


class _ProjWrapper:
    """proj<k>_wrapper(): connectivity from init_from_lil, its queries and the
    synaptic attributes per locality (ANNarchy/generator/NanoBind/
    Projection.py:20-179)."""

    def __init__(self, module, proj):
        self._m = module
        self._proj = proj
        self._transmission = True
        self._axon_transmission = True
        self._update = True
        self._plasticity = True
        self._update_period = 1
        self._update_offset = 0

    def init_from_lil(self, post_ranks, pre_ranks, w, delays, requires_sorting=False) -> bool:
        """LIL connectivity (post ranks; per post the pre ranks, weights and
        delays in steps) into the projection's CSR; False when it is not
        valid (ranks outside the populations, ragged rows)."""
        try:
            self._proj._from_lil(post_ranks, pre_ranks, w, delays, bool(requires_sorting))
        except (ValueError, IndexError) as e:
            self._m.last_error = str(e)
            return False
        return True

    # connectivity queries
    def post_rank(self):
        return [int(r) for r in self._proj.post_ranks]

    def pre_ranks(self):
        return [list(map(int, r)) for r in self._proj._pre_ranks_of()]

    def pre_rank(self, idx: int):
        return list(map(int, self._proj._pre_ranks_of()[idx]))

    def dendrite_size(self, idx: int) -> int:
        return int(self._proj.dendrite_sizes()[idx])

    def nb_dendrites(self) -> int:
        return int(self._proj.size)

    def nb_synapses(self) -> int:
        return int(self._proj.nb_synapses)

    def nb_efferent_synapses(self) -> int:
        return int(self._proj.nb_synapses)

    # attributes: get/set_{local,semiglobal,global}_attribute[_all|_row]_<ctype>
    def __getattr__(self, name):
        if name.startswith("_"):
            raise AttributeError(name)
        for prefix in ("get_local_attribute_all_", "get_local_attribute_row_",
                       "get_local_attribute_", "set_local_attribute_all_",
                       "set_local_attribute_row_", "set_local_attribute_",
                       "get_semiglobal_attribute_all_", "get_semiglobal_attribute_",
                       "set_semiglobal_attribute_all_", "set_semiglobal_attribute_",
                       "get_global_attribute_", "set_global_attribute_"):
            if name.startswith(prefix):
                op = prefix.rstrip("_")
                return lambda *a, _op=op: self._attr(_op, *a)
        raise AttributeError(f"proj{self._proj.id}_wrapper has no attribute {name!r}")

    def _attr(self, op: str, name: str, *args):
        p = self._proj
        if op == "get_local_attribute_all":
            return [list(map(float, r)) for r in p.get(name)]
        if op == "get_local_attribute_row":
            return list(map(float, p.get(name)[args[0]]))
        if op == "get_local_attribute":
            return float(p.get(name)[args[0]][args[1]])
        if op == "set_local_attribute_all":
            p.set({name: [np.asarray(r, dtype=np.float64) for r in args[0]]})
            return None
        if op in ("set_local_attribute_row", "set_local_attribute"):
            rows = p.get(name)
            if op == "set_local_attribute_row":
                rows[args[0]] = np.asarray(args[1], dtype=np.float64)
            else:
                rows[args[0]][args[1]] = float(args[2])
            p.set({name: rows})
            return None
        if op == "get_semiglobal_attribute_all":
            return list(map(float, p.get(name)))
        if op == "get_semiglobal_attribute":
            return float(p.get(name)[args[0]])
        if op in ("set_semiglobal_attribute_all", "set_semiglobal_attribute"):
            if op == "set_semiglobal_attribute_all":
                p.set({name: np.asarray(args[0], dtype=np.float64)})
            else:
                cur = np.asarray(p.get(name), dtype=np.float64)
                cur[args[0]] = float(args[1])
                p.set({name: cur})
            return None
        if op == "get_global_attribute":
            return float(p.get(name))
        if op == "set_global_attribute":
            p.set({name: float(args[0])})
            return None
        raise AttributeError(op)

    def size_in_bytes(self) -> int:
        return int(p_nnz_bytes(self._proj))

    def clear(self):
        pass


def p_nnz_bytes(proj) -> int:
    """Host estimate of a projection's connectivity bytes: per synapse an
    index and a weight, per dendrite a row pointer and a post rank."""
    return proj.nb_synapses * 12 + proj.size * 8


class _Recorder:
    """PopRecorder<k>_wrapper(ranks, period, period_offset, offset): switches
    record_<var>, the recorded data <var> (spike: dict rank -> steps) and
    clear_<var>() over this backend's device monitor of the same
    population (ANNarchy/generator/Monitor/BaseTemplates.py)."""

    def __init__(self, module, mon, ranks, period, period_offset, offset):
        object.__setattr__(self, "_m", module)
        object.__setattr__(self, "_mon", mon)
        object.__setattr__(self, "ranks", list(ranks))
        object.__setattr__(self, "period", int(period))
        object.__setattr__(self, "period_offset", int(period_offset))
        object.__setattr__(self, "offset", int(offset))
        object.__setattr__(self, "_on", set())
        object.__setattr__(self, "_started", False)

    @staticmethod
    def _var(name: str) -> str:
        return f"sum({name[5:]})" if name.startswith("_sum_") else name

    def __setattr__(self, name, value):
        if name.startswith("record_"):
            var = self._var(name[len("record_"):])
            if var not in self._mon.variables:
                raise AttributeError(f"{var} is not recorded by this monitor")
            on = set(self._on)
            (on.add if value else on.discard)(var)
            object.__setattr__(self, "_on", on)
            if on and not self._mon._recording:
                if self._started:
                    self._mon.resume()
                else:
                    self._mon.start()
                    object.__setattr__(self, "_started", True)
            elif not on and self._mon._recording:
                self._mon.pause()
            return
        object.__setattr__(self, name, value)

    def __getattr__(self, name):
        if name.startswith("clear_"):
            var = self._var(name[len("clear_"):])
            return lambda: self._mon.get(var, keep=False, reshape=False)
        if name.startswith("_"):
            raise AttributeError(name)
        var = self._var(name)
        if var in self._mon.variables:
            return self._mon.get(var, keep=True, reshape=False)
        raise AttributeError(name)

    def clear(self):
        for v in self._mon.variables:
            self._mon.get(v, keep=False, reshape=False)

    def size_in_bytes(self) -> int:
        return 0


class ReferenceModule:
    """ANNarchyWrapper<id> over this backend for one reference network.

    `ref_net` is an ANNarchy.Network (or the reference's default network)
    whose populations, projections and monitors are declared but not
    compiled; `config` goes to annarchy_b200.Network.config (precision
    follows the reference's dtype unless given)."""

    def __init__(self, ref_net, dry: bool = False, **config):
        from . import Network, Neuron, Synapse
        self.ref = ref_net
        self.dry = dry
        self.last_error = ""
        dt = float(ref_net._get_config("dt"))
        seed = ref_net._get_config("seed")
        self._net = Network(dt=dt, seed=seed)
        prec = "float" if "32" in str(ref_net._get_config("dtype")) else "double"
        cfg = {"precision": prec}
        cfg.update(config)
        self._net.config(**cfg)
        # our monitors per population, in the reference's monitor order: its
        # _init_monitoring creates one PopRecorder<pop>_wrapper per monitor in
        # that order
        self._pops, self._projs, self._mons = {}, {}, {}
        for pop in ref_net.get_populations():
            nt = pop.neuron_type
            ours = self._net.create(tuple(pop.geometry), Neuron(**_ref_neuron_args(nt)),
                                    name=pop.name)
            self._pops[pop.id] = ours

        def view_of(obj):
            ours = self._pops[(obj.population if hasattr(obj, "population") and
                               not hasattr(obj, "neuron_type") else obj).id]
            if hasattr(obj, "ranks") and len(obj.ranks) != ours.size:
                return ours[np.asarray(obj.ranks)]
            return ours

        for proj in ref_net.get_projections():
            pre, post = view_of(proj.pre), view_of(proj.post)
            if proj.pre is proj.post:
                post = pre
            syn = Synapse(**_ref_synapse_args(proj.synapse_type))
            self._projs[proj.id] = self._net.connect(pre, post, proj.target, synapse=syn,
                                                     name=proj.name)
        for mon in ref_net.get_monitors():
            obj = mon.object
            if not hasattr(obj, "neuron_type") and not hasattr(obj, "population"):
                raise NotImplementedError("only population monitors are served by this backend")
            self._mons.setdefault(obj.id, []).append(
                self._net.monitor(view_of(obj), list(mon.variables), period=mon.period,
                                  start=False))
        self._next_mon = {k: 0 for k in self._mons}

    # -- device / threads / seeds -----------------------------------------------------
    def set_device(self, device: int):
        self._net.config(device=int(device))

    def set_number_threads(self, n: int, cores=()):
        pass                                    # one GPU; host threads are not used

    def pyx_create(self):
        pass

    def set_seed(self, seed: int, num_sources: int = 1, use_seed_seq: bool = True):
        """The seed of the network's generator, from which the key of the
        device's random draws is taken at compile (anb_set_seed); afterwards
        the key itself. num_sources and use_seed_seq concern the reference's
        per-thread std::mt19937 engines and have no effect."""
        if self._net.compiled and not self.dry:
            self._net._backend.native.set_seed(int(seed), int(num_sources), bool(use_seed_seq))
        else:
            self._net.config(seed=int(seed))

    def pyx_initialize(self, dt: float):
        """All connectivity has arrived through init_from_lil: build the
        device network (storage formats, kernels) for time step dt."""
        if abs(float(dt) - self._net.dt) > 1e-15:
            raise ValueError(f"dt {dt} differs from the network's {self._net.dt}")
        if self.dry:
            from .core.backend import CompiledNetwork
            self.dry_backend = CompiledNetwork(self._net, dry=True)
            self.dry_backend.build()
            return
        self._net.compile()

    # -- simulation --------------------------------------------------------------------
    def run(self, nsteps: int):
        self._net.simulate_steps(int(nsteps))

    def step(self):
        self._net.simulate_steps(1)

    def run_until(self, steps: int, populations, or_and: bool = True) -> int:
        pops = [self._pops[int(p)] for p in populations]
        return int(self._net._backend.run_until(int(steps), pops, bool(or_and)))

    def set_time(self, t: int):
        self._net.set_current_step(int(t))

    def get_time(self) -> int:
        return int(self._net.current_step)

    def estimate_record_size(self, nsteps: int) -> int:
        """MiB the recorded state variables take after nsteps more steps
        (anb_estimate_record_size; spikes are not counted, as in the
        reference)."""
        if self.dry or not self._net.compiled:
            return 0
        return self._net._backend.native.estimate_record_size(int(nsteps))

    # -- per-object wrappers ---------------------------------------------------------------
    def _recorder(self, pop_id, ranks, period, period_offset, offset):
        mons = self._mons.get(pop_id, [])
        i = self._next_mon.get(pop_id, 0)
        if i >= len(mons):
            raise NotImplementedError("monitors are fixed when the network is built on this "
                                      "backend; create them before compile()")
        self._next_mon[pop_id] = i + 1
        return _Recorder(self, mons[i], ranks, period, period_offset, offset)

    def __getattr__(self, name):
        if name.startswith("pop") and name.endswith("_wrapper"):
            k = int(name[3:-8])
            return lambda size, max_delay, _k=k: _PopWrapper(self, self._pops[_k], size, max_delay)
        if name.startswith("proj") and name.endswith("_wrapper"):
            k = int(name[4:-8])
            return lambda _k=k: _ProjWrapper(self, self._projs[_k])
        if name.startswith("PopRecorder") and name.endswith("_wrapper"):
            k = int(name[len("PopRecorder"):-8])
            return lambda ranks, period, period_offset, offset, _k=k: self._recorder(
                _k, ranks, period, period_offset, offset)
        if name.startswith("set_"):
            cname = name[4:]
            if cname in self._net._constants:
                return lambda value, _c=cname: self._net.get_constant(_c).set(float(value))
        raise AttributeError(name)


def instantiate(ref_net, dry: bool = False, **config) -> ReferenceModule:
    """Compile and instantiate a network built with the reference's API on
    this backend: the reference's own Compiler._instantiate runs with a
    ReferenceModule in place of the extension module it would have built
    and loaded. Returns the module (also ref_net.instance)."""
    from ANNarchy.generator import Compiler as RC
    module = ReferenceModule(ref_net, dry=dry, **config)
    if ref_net.compiled:
        raise RuntimeError("the reference network is already compiled")
    loader = RC.load_cython_lib
    RC.load_cython_lib = lambda libname, libpath: module
    try:
        ref_net.directory = "<annarchy_b200>"
        ref_net.compiled = True
        RC._instantiate(ref_net.id)
    finally:
        RC.load_cython_lib = loader
    return module
