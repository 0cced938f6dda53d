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


class TimedArray(Population):
    """Rate-coded population whose rates follow a buffer of input vectors
    (ANNarchy/inputs/TimedArray.py:95-300): `rates` has shape (blocks,
    *geometry); block b is set at the steps where the internal time (steps
    since the last reset, taken modulo `period` when it is positive) equals
    schedule[b], and r keeps its value in between. `schedule` is a step size
    in ms (0: every step) or a list of times; `period` in ms (-1: no cycling).

        inp = net.create(TimedArray(rates=inputs, schedule=10.0, period=100.0))
    """

    def __init__(self, rates=None, geometry=None, schedule=0.0, period: float = -1.0,
                 name: str | None = None, copied: bool = False, net_id: int = 0):
        if rates is None and geometry is None:
            raise ValueError("TimedArray: either rates or geometry must be set")
        if rates is not None:
            rates = np.asarray(rates, dtype=np.float64)
            if geometry is None:
                geometry = rates.shape[1:]
        if isinstance(geometry, int):
            geometry = (geometry,)
        super().__init__(tuple(geometry), Neuron(equations="r = 0.0", name="Timed Array"), name=name)
        object.__setattr__(self, "_auto_name", name is None)
        object.__setattr__(self, "_ta_rates", None)
        object.__setattr__(self, "_ta_schedule_ms", [])
        object.__setattr__(self, "_ta_period_ms", -1.0)
        object.__setattr__(self, "_ta_t0", 0)
        if rates is not None:
            self.update(rates, schedule=schedule, period=period)
        else:
            s0 = np.atleast_1d(schedule)
            object.__setattr__(self, "_ta_schedule_ms",
                               None if s0.size == 1 and float(s0[0]) <= 0.0 else schedule)
            object.__setattr__(self, "_ta_period_ms", float(period))

    # -- schedule -----------------------------------------------------------------
    def _dt(self):
        return self.net.dt if self.net is not None else 1.0

    def steps(self):
        """(schedule in steps, period in steps) with the reference's rounding
        (np.rint(ms / dt), ANNarchy/core/Utils.py:22-50); a schedule of 0 ms
        is every step."""
        dt = self._dt()
        blocks = 0 if self._ta_rates is None else self._ta_rates.shape[0]
        if self._ta_schedule_ms is None:
            sched = list(range(blocks))
        else:
            sched = [int(np.rint(s / dt)) for s in self._ta_schedule_ms]
        per = int(np.rint(self._ta_period_ms / dt)) if self._ta_period_ms > 0 else -1
        return sched, per

    @property
    def schedule(self):
        if self._ta_schedule_ms is None:
            blocks = 0 if self._ta_rates is None else self._ta_rates.shape[0]
            return [self._dt() * i for i in range(blocks)]
        return list(self._ta_schedule_ms)

    @property
    def period(self):
        return self._ta_period_ms

    @property
    def rates(self):
        return None if self._ta_rates is None else self._ta_rates.copy()

    def update(self, rates, schedule=None, period=None, reset: bool = True):
        """New input vectors (blocks, *geometry); optionally a new schedule
        and period. With `reset` the internal time restarts at the next step
        (ANNarchy/inputs/TimedArray.py:166-300)."""
        rates = np.asarray(rates, dtype=np.float64)
        if rates.ndim < 1 or rates.shape[0] == 0:
            raise ValueError("TimedArray: the first dimension of rates must not be empty")
        if tuple(rates.shape[1:]) != tuple(self.geometry):
            raise ValueError(f"TimedArray: rates of shape {rates.shape} do not match the geometry "
                             f"{self.geometry}")
        if schedule is None:
            schedule = self._ta_schedule_ms if self._ta_schedule_ms is not None else 0.0
        if period is None:
            period = self._ta_period_ms
        if np.ndim(schedule) == 0 or len(schedule) == 1:
            step = float(np.atleast_1d(schedule)[0])
            # every step (0 ms) stays symbolic: the step size is only known in the network
            schedule = None if step <= 0.0 else [step * i for i in range(rates.shape[0])]
        if schedule is not None:
            schedule = [float(s) for s in schedule]
            if len(schedule) > rates.shape[0]:
                raise ValueError("TimedArray: the schedule is longer than the rates")
            if any(b <= a for a, b in zip(schedule, schedule[1:])):
                raise ValueError("TimedArray: the schedule must be increasing")
            rates = rates[: len(schedule)]
        object.__setattr__(self, "_ta_rates", rates.reshape(rates.shape[0], -1).copy())
        object.__setattr__(self, "_ta_schedule_ms", schedule)
        object.__setattr__(self, "_ta_period_ms", float(period))
        if self._compiled():
            if reset:
                object.__setattr__(self, "_ta_t0", self.net.current_step)
            self.net._backend.write_timed_array(self)

    def reset(self, attributes=None):
        super().reset(attributes)
        object.__setattr__(self, "_ta_t0", self.net.current_step if self._compiled() else 0)
        if self._compiled():
            self.net._backend.write_timed_array(self)
