"""Neuron and Synapse model containers and the built-in models used by the
benchmark configurations.

Same constructor arguments as the reference (ANNarchy/core/Neuron.py,
ANNarchy/core/Synapse.py): equation strings (or lists of them), a spike
condition and reset for spiking neurons, pre_spike / post_spike statements
for event-driven synapses. A neuron is spiking when it has a ``spike``
condition; a synapse is spiking when it has ``pre_spike`` or ``post_spike``.
"""
from __future__ import annotations

import copy
from dataclasses import dataclass

from .random import RandomDistribution

# analysed descriptions by defining strings: the equations of identical
# models (e.g. the copies of a parameter sweep) are parsed once
_DESC_CACHE: dict = {}


def _global_functions_key():
    from ..parser.equation import GLOBAL_FUNCTIONS
    return tuple(sorted((k, v["cpp"]) for k, v in GLOBAL_FUNCTIONS.items()))


def add_function(function: str):
    """Define a function usable in every neuron and synapse defined
    afterwards, e.g. ``add_function("sigmoid(x) = 1.0 / (1.0 + exp(-x))")``
    (ANNarchy/core/Global.py, add_function)."""
    from ..parser.analysis import analyse_functions
    from ..parser.equation import GLOBAL_FUNCTIONS
    for f in analyse_functions(function):
        GLOBAL_FUNCTIONS[f["name"]] = f


def functions(name: str):
    """A function defined by add_function, as a host callable on arrays."""
    from ..parser.equation import GLOBAL_FUNCTIONS
    from .functions import evaluator
    if name not in GLOBAL_FUNCTIONS:
        raise KeyError(f"no function {name!r} was added")
    return evaluator(GLOBAL_FUNCTIONS[name])


def _cached(kind, key, analyse, model):
    key = (kind, repr(key))
    if key not in _DESC_CACHE:
        _DESC_CACHE[key] = analyse(model)
    return copy.deepcopy(_DESC_CACHE[key])


@dataclass
class Parameter:
    """A parameter of a neuron or synapse given as an object in the dict
    form of `parameters` (ANNarchy/core/Attributes.py:11-48): its value (a
    number or a random distribution drawn at creation), locality ('global',
    the default of plain values, 'semiglobal' or 'local') and type."""
    value: object
    locality: str = "global"
    type: object = "float"


@dataclass
class Variable:
    """A variable of a neuron or synapse given as an object in the list form
    of `equations` (ANNarchy/core/Attributes.py:51-130): its equation and
    flags, written out as the equation line `eq : init=..., min=..., max=...,
    method, type, locality`."""
    equation: str
    init: object = None
    min: object = None
    max: object = None
    method: str | None = None
    locality: str = "local"
    type: object = "float"

    def __str__(self):
        flags = []
        if self.init is not None:
            flags.append(f"init={self.init!r}" if isinstance(self.init, RandomDistribution)
                         else f"init={self.init}")
        if self.min is not None:
            flags.append(f"min={self.min}")
        if self.max is not None:
            flags.append(f"max={self.max}")
        if self.method is not None:
            flags.append(str(self.method))
        kind = {float: "float", int: "int", bool: "bool"}.get(self.type, str(self.type))
        if kind != "float":
            flags.append(kind)
        if self.locality != "local":
            flags.append("postsynaptic" if self.locality == "semiglobal" else "population")
        return self.equation + (" : " + ", ".join(flags) if flags else "")


class Neuron:
    def __init__(self, parameters="", equations="", spike=None, axon_spike=None, reset=None,
                 axon_reset=None, refractory=None, functions=None, name="", description=""):
        if axon_spike or axon_reset:
            raise NotImplementedError("axonal spikes are not supported by this backend")
        self.parameters = parameters
        self.equations = equations
        self.spike = spike
        self.reset = reset
        self.refractory = refractory
        self.functions = functions
        self.name = name or ("Spiking neuron" if spike else "Rate-coded neuron")
        self.description = description
        self.type = "spike" if spike else "rate"
        self._desc = None

    @property
    def desc(self):
        if self._desc is None:
            from ..parser.analysis import analyse_neuron
            self._desc = _cached("neuron", (self.parameters, self.equations, self.spike,
                                            self.reset, self.refractory, self.type,
                                            self.functions, _global_functions_key()),
                                 analyse_neuron, self)
        return self._desc

    def __repr__(self):
        return f"Neuron({self.name!r}, type={self.type})"


class Synapse:
    def __init__(self, parameters="", equations="", psp=None, operation="sum", pre_spike=None,
                 post_spike=None, pre_axon_spike=None, functions=None, pruning=None,
                 creating=None, name=None, description=None):
        if operation not in ("sum", "max", "min", "mean"):
            raise ValueError(f"operation {operation!r}: sum, max, min or mean")
        if pre_axon_spike or pruning or creating:
            raise NotImplementedError("axonal spikes and structural plasticity are "
                                      "not supported by this backend")
        self.parameters = parameters
        self.equations = equations
        self.psp = psp
        self.operation = operation
        self.pre_spike = pre_spike
        self.post_spike = post_spike
        self.functions = functions
        self.type = "spike" if (pre_spike or post_spike) else "rate"
        self.name = name or ("Spiking synapse" if self.type == "spike" else "Rate-coded synapse")
        self.description = description
        self._desc = None

    @property
    def desc(self):
        if self._desc is None:
            from ..parser.analysis import analyse_synapse
            self._desc = _cached("synapse", (self.parameters, self.equations, self.psp,
                                             self.pre_spike, self.post_spike, self.type,
                                             self.functions, _global_functions_key()),
                                 analyse_synapse, self)
        return self._desc

    def __repr__(self):
        return f"Synapse({self.name!r}, type={self.type})"


# ---------------------------------------------------------------------------
# built-in models (ANNarchy/models/Neurons.py, ANNarchy/models/Synapses.py)
# ---------------------------------------------------------------------------

class LeakyIntegrator(Neuron):
    """tau * dr/dt + r = sum(exc) - sum(inh) + baseline, rectified (r >= 0)."""

    def __init__(self, tau=10.0, B=0.0):
        super().__init__(parameters=dict(tau=tau, B=B),
                         equations="tau * dr/dt + r = sum(exc) - sum(inh) + B : min=0.0",
                         name="Leaky-Integrator")


class IF_cond_exp(Neuron):
    """Conductance-based leaky integrate-and-fire neuron with exponentially
    decaying conductances (explicit Euler)."""

    def __init__(self, v_rest=-65.0, cm=1.0, tau_m=20.0, tau_refrac=0.0, tau_syn_E=5.0,
                 tau_syn_I=5.0, e_rev_E=0.0, e_rev_I=-70.0, v_thresh=-50.0, v_reset=-65.0,
                 i_offset=0.0):
        super().__init__(
            parameters=dict(v_rest=v_rest, cm=cm, tau_m=tau_m, tau_refrac=tau_refrac,
                            tau_syn_E=tau_syn_E, tau_syn_I=tau_syn_I, e_rev_E=e_rev_E,
                            e_rev_I=e_rev_I, v_thresh=v_thresh, v_reset=v_reset,
                            i_offset=i_offset),
            equations="""
                cm * dv/dt = cm/tau_m*(v_rest -v) + g_exc*(e_rev_E - v) + g_inh*(e_rev_I - v) + i_offset : init=-65.0
                tau_syn_E * dg_exc/dt = - g_exc
                tau_syn_I * dg_inh/dt = - g_inh
            """,
            spike="v > v_thresh", reset="v = v_reset", refractory=tau_refrac,
            name="IF_cond_exp")


class STDP(Synapse):
    """Pair-based spike-timing dependent plasticity with event-driven traces
    x (pre) and y (post)."""

    def __init__(self, tau_plus=20.0, tau_minus=20.0, A_plus=0.01, A_minus=0.01, w_min=0.0,
                 w_max=1.0):
        super().__init__(
            parameters=f"""
                tau_plus = {tau_plus} : projection
                tau_minus = {tau_minus} : projection
                A_plus = {A_plus} : projection
                A_minus = {A_minus} : projection
                w_min = {w_min} : projection
                w_max = {w_max} : projection
            """,
            equations="""
                tau_plus  * dx/dt = -x : event-driven
                tau_minus * dy/dt = -y : event-driven
            """,
            pre_spike="""
                g_target += w
                x += A_plus * w_max
                w = clip(w + y, w_min , w_max)
            """,
            post_spike="""
                y -= A_minus * w_max
                w = clip(w + x, w_min , w_max)
            """,
            name="Spike-timing dependent plasticity")
