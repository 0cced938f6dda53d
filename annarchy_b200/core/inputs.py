"""Input populations.

PoissonPopulation follows the reference (ANNarchy/inputs/PoissonPopulation.py:
100-202): a spiking population whose neurons draw ``p = Uniform(0.0, 1.0) *
1000.0 / dt`` every step and spike when ``p < rates``, i.e. with probability
rates * dt / 1000 per step (Bernoulli approximation of a Poisson process).
``rates`` is a number, an array (one rate per neuron, settable later as
``pop.rates``) or an equation of time and of the given parameters
(``"amp * (1.0 + sin(2*pi*frequency*t/1000.0))/2.0"``). The draws come from
the device's counter-based generator (Philox4x32-10 keyed by the network's
seed), not from the reference's std::mt19937 stream.
"""
from __future__ import annotations

import numpy as np

from .models import Neuron
from .population import Population


def _parameter_text(parameters) -> str:
    if not parameters:
        return ""
    if isinstance(parameters, str):
        return parameters
    return "\n".join(f"{k} = {float(v)}" for k, v in parameters.items())


class PoissonPopulation(Population):
    """Population of neurons emitting spikes with the given mean rates (Hz).

        inp = net.create(PoissonPopulation(100, rates=20.0))
    """

    def __init__(self, geometry, name: str | None = None, rates=None, target: str | None = None,
                 parameters=None, refractory: float | None = None, copied: bool = False,
                 net_id: int = 0):
        if rates is None and target is None:
            raise ValueError("a PoissonPopulation must define either rates or target")
        if target is not None:
            raise NotImplementedError("PoissonPopulation(target=...) (rates from rate-coded "
                                      "projections) is not supported by this backend")
        extra = _parameter_text(parameters)
        draw = "p = Uniform(0.0, 1.0) * 1000.0 / dt"
        if isinstance(rates, str):
            neuron = Neuron(parameters=extra, equations=f"rates = {rates}\n{draw}",
                            spike="p < rates", refractory=refractory, name="Poisson")
        else:
            value = 10.0 if isinstance(rates, np.ndarray) else float(rates)
            params = f"rates = {value}" + (f"\n{extra}" if extra else "")
            neuron = Neuron(parameters=params, equations=draw, spike="p < rates",
                            refractory=refractory, name="Poisson")
        super().__init__(geometry, neuron, name=name)
        object.__setattr__(self, "_auto_name", name is None)
        self.rates_init = rates
        if isinstance(rates, np.ndarray):
            self.rates = rates
