"""Monitors: recording of spikes and state variables.

Semantics follow the reference (ANNarchy/core/Monitor.py:220-595 and the
recorder templates in ANNarchy/generator/Monitor/BaseTemplates.py): a
variable is recorded at the end of step t (after the neuron update) when
(t - start) % period == 0; spikes are recorded as the step index at which
they were emitted. The reference copies whole arrays device->host at every
recorded step (ANNarchy/generator/Monitor/CUDATemplates.py:83); here the
kernels append into device buffers that are drained once per simulated
chunk.
"""
from __future__ import annotations

import numpy as np

from .population import Population, PopulationView


class Monitor:
    def __init__(self, obj, variables=None, period: float | None = None,
                 period_offset: float | None = None, start: bool = True, name: str | None = None,
                 net=None, mon_id: int = 0):
        if isinstance(variables, str):
            variables = [variables]
        variables = list(variables or [])
        if not isinstance(obj, (Population, PopulationView)):
            raise NotImplementedError("only populations and population views can be monitored")
        self.object = obj
        self.population = obj.population if isinstance(obj, PopulationView) else obj
        self.ranks = None if isinstance(obj, Population) else np.asarray(obj.ranks)
        self.net = net
        self.id = mon_id
        self.name = name or f"monitor{mon_id}"
        for v in variables:
            if v == "spike":
                if self.population.neuron_type.type != "spike":
                    raise ValueError("spikes can only be recorded from spiking populations")
            elif v not in self.population._host:
                raise ValueError(f"{self.population.name} has no attribute {v!r}")
        self.variables = variables
        dt = net.dt if net is not None else 1.0
        self.period_steps = max(1, int(round((period if period is not None else dt) / dt)))
        self.period_offset_steps = int(round((period_offset or 0.0) / dt))
        self._recording = bool(start)
        self._start_step = 0
        self._data: dict[str, list] = {v: [] for v in variables if v != "spike"}
        self._spike_steps: list[np.ndarray] = []
        self._spike_ranks: list[np.ndarray] = []
        self._record_steps: list[int] = []

    @property
    def period(self) -> float:
        return self.period_steps * (self.net.dt if self.net is not None else 1.0)

    # -- control -----------------------------------------------------------------
    def start(self, variables=None, period=None):
        if variables is not None:
            raise NotImplementedError("changing the recorded variables after creation is not "
                                      "supported by this backend")
        if period is not None:
            self.period_steps = max(1, int(round(period / self.net.dt)))
        self._recording = True
        if self.net is not None and self.net._compiled:
            self._start_step = self.net.current_step

    def pause(self):
        self._recording = False

    def resume(self):
        self._recording = True

    def stop(self):
        self._recording = False

    def reset(self):
        """Empty the recordings (ANNarchy/core/Monitor.py reset)."""
        self._data = {v: [] for v in self.variables if v != "spike"}
        self._spike_steps, self._spike_ranks = [], []
        self._record_steps = []
        self._start_step = 0

    # -- results -------------------------------------------------------------------
    def _append_spikes(self, steps: np.ndarray, ranks: np.ndarray):
        if steps.size:
            self._spike_steps.append(steps)
            self._spike_ranks.append(ranks)

    def _append_values(self, var: str, values: np.ndarray, steps):
        self._data[var].append(values)
        if var == next((v for v in self.variables if v != "spike"), None):
            self._record_steps.extend(int(s) for s in steps)

    def spike_arrays(self):
        """(steps, ranks) of all recorded spikes, sorted by step then rank."""
        if not self._spike_steps:
            return np.zeros(0, np.int64), np.zeros(0, np.int64)
        s = np.concatenate(self._spike_steps)
        r = np.concatenate(self._spike_ranks)
        # chunks arrive in time order, each sorted by (step, rank)
        if s.size > 1 and (np.any(np.diff(s) < 0)):
            order = np.lexsort((r, s))
            s, r = s[order], r[order]
        return s, r

    def get(self, variables=None, keep: bool = False, reshape: bool = False,
            force_dict: bool = False):
        if variables is None:
            variables = self.variables
        single = isinstance(variables, str)
        if single:
            variables = [variables]
        out = {}
        for v in variables:
            if v == "spike":
                s, r = self.spike_arrays()
                size = self.population.size
                # by rank, steps stay ascending (radix sort for 16-bit ranks)
                key = r.astype(np.uint16) if size <= 65536 else r
                order = np.argsort(key, kind="stable")
                counts = np.bincount(r, minlength=size)
                offs = np.zeros(size + 1, dtype=np.int64)
                np.cumsum(counts, out=offs[1:])
                # one conversion to Python ints, then list slices per neuron
                steps = s[order].tolist()
                lo, hi = offs[:-1].tolist(), offs[1:].tolist()
                if self.ranks is None:
                    d = {k: steps[a:b] for k, (a, b) in enumerate(zip(lo, hi))}
                else:
                    d = {int(k): steps[lo[int(k)]:hi[int(k)]] for k in self.ranks}
                out[v] = d
                if not keep:
                    self._spike_steps, self._spike_ranks = [], []
            else:
                chunks = self._data[v]
                n = self.population.size if self.ranks is None else len(self.ranks)
                arr = np.concatenate(chunks, axis=0) if chunks else np.zeros((0, n))
                if reshape and self.ranks is None and len(self.population.geometry) > 1:
                    arr = arr.reshape((arr.shape[0],) + self.population.geometry)
                out[v] = arr
                if not keep:
                    self._data[v] = []
        if not keep:
            self._record_steps = []
        if single and not force_dict:
            return out[variables[0]]
        return out

    def times(self, variables=None):
        return {"start": [self._start_step], "stop": [self.net.current_step if self.net else 0]}

    # -- analysis helpers (ANNarchy/core/Monitor.py:712-995) ------------------------
    def raster_plot(self, spikes=None):
        """(times in ms, ranks) of the recorded spikes."""
        if spikes is None:
            s, r = self.spike_arrays()
            return s * self.net.dt, r
        t, n = [], []
        for rank, steps in spikes.items():
            t.extend(steps)
            n.extend([rank] * len(steps))
        return np.asarray(t, dtype=np.float64) * self.net.dt, np.asarray(n, dtype=np.int64)

    def mean_fr(self, spikes=None, duration_ms: float | None = None):
        """Mean firing rate (Hz) over all recorded neurons."""
        if spikes is None:
            s, r = self.spike_arrays()
            count = s.size
        else:
            count = sum(len(v) for v in spikes.values())
        n = self.population.size if self.ranks is None else len(self.ranks)
        if duration_ms is None:
            duration_ms = (self.net.current_step - self._start_step) * self.net.dt
        return 1000.0 * count / max(1, n) / max(duration_ms, 1e-12)

    def histogram(self, spikes=None, bins: float | None = None):
        """Spike counts per time bin (bins in ms, default dt)."""
        s, _ = self.spike_arrays() if spikes is None else self.raster_plot(spikes)
        if spikes is not None:
            s = np.round(s / self.net.dt).astype(np.int64)
        width = max(1, int(round((bins or self.net.dt) / self.net.dt)))
        if s.size == 0:
            return np.zeros(0, dtype=np.int64)
        return np.bincount((s - s.min()) // width)

    def population_rate(self, spikes=None, smooth: float = 0.0):
        """Instantaneous population rate (Hz) per step."""
        h = self.histogram(spikes)
        n = self.population.size if self.ranks is None else len(self.ranks)
        rate = h / n / (self.net.dt / 1000.0)
        if smooth > 0 and rate.size:
            k = max(1, int(round(smooth / self.net.dt)))
            rate = np.convolve(rate, np.ones(k) / k, mode="same")
        return rate
