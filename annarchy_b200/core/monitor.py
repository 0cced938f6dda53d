"""Monitors: recording of spikes and state variables, and the spike analysis
functions.

Semantics follow the reference (ANNarchy/core/Monitor.py:220-995 and the
recorder templates in ANNarchy/generator/Monitor/BaseTemplates.py): a
variable is recorded at the end of step t (after the neuron update) when
(t - start) % period == offset; spikes are recorded as the step index at
which they were emitted; ``sum(target)`` records the weighted sums of a
rate-coded population. The reference copies whole arrays device->host at
every recorded step (ANNarchy/generator/Monitor/CUDATemplates.py:83); here
the kernels append into device buffers that are drained once per simulated
chunk.

The analysis functions (raster_plot, histogram, inter_spike_interval,
coefficient_of_variation, mean_fr, smoothed_rate, population_rate) restate
the reference's module functions (Monitor.py:1091-1330) and its Cython
transformations (ANNarchy/cython_ext/Transformations.pyx:23-108), including
their float32 step size in the rate transformations.
"""
from __future__ import annotations

import copy
import gc
import re

import numpy as np

from .population import Population, PopulationView

_SUM = re.compile(r"^sum\((\w+)\)$")


def array_name(var: str) -> str:
    """Suffix of the recording buffer of a variable ('sum(exc)' -> '_sum_exc')."""
    m = _SUM.match(var)
    return f"_sum_{m.group(1)}" if m else var


def source_name(var: str) -> str:
    """Population array a variable is recorded from: the weighted sums of the
    step just finished are kept in '_last_sum_<target>' (the update kernel
    consumes and clears '_sum_<target>')."""
    m = _SUM.match(var)
    return f"_last_sum_{m.group(1)}" if m else var


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
            self._check_variable(v)
        self.variables = variables
        dt = self.dt
        self.period_steps = max(1, int(round((period if period is not None else dt) / dt)))
        self.period_offset_steps = int(round((period_offset or 0.0) / dt))
        self._recording = bool(start)
        self._start_step = 0
        self._data: dict[str, list] = {v: [] for v in variables if v != "spike"}
        self._spike_steps: list[np.ndarray] = []
        self._spike_ranks: list[np.ndarray] = []
        self._record_steps: list[int] = []
        # start/stop steps of every variable (Monitor.py:284-300, 577-590)
        self._recorded: dict[str, dict] = {}
        self._last_recorded: dict[str, dict] = {}
        for v in variables:
            self._add_variable(v)

    def _check_variable(self, v):
        if v == "spike":
            if self.population.neuron_type.type != "spike":
                raise ValueError("spikes can only be recorded from spiking populations")
        elif _SUM.match(v):
            if self.population.neuron_type.type != "rate":
                raise ValueError(f"{v}: weighted sums are recorded for rate-coded populations")
            if _SUM.match(v).group(1) not in self.population.targets:
                raise ValueError(f"{self.population.name} receives no target "
                                 f"{_SUM.match(v).group(1)!r}")
        elif v not in self.population._host:
            raise ValueError(f"{self.population.name} has no attribute {v!r}")

    # -- bookkeeping ------------------------------------------------------------------
    @property
    def dt(self) -> float:
        return self.net.dt if self.net is not None else 1.0

    def _now(self) -> int:
        return int(self.net.current_step) if self.net is not None else 0

    def _compiled(self) -> bool:
        return self.net is not None and self.net._compiled

    def _add_variable(self, var):
        self._recorded[var] = {"start": [self._now()], "stop": [None]}
        self._last_recorded[var] = {"start": [self._now()], "stop": [None]}

    def _update_stopping_time(self, var, keep):
        rec = self._recorded[var]
        rec["stop"][-1] = self._now()
        self._last_recorded[var] = {"start": list(rec["start"]), "stop": list(rec["stop"])}
        if not keep:
            self._recorded[var] = {"start": [self._now()], "stop": [None]}

    @property
    def period(self) -> float:
        return self.period_steps * self.dt

    @period.setter
    def period(self, val: float):
        steps = max(1, int(round(val / self.dt)))
        if self._compiled() and steps != self.period_steps:
            raise NotImplementedError("the recording period is compiled into the network in this "
                                      "backend; set it before compile()")
        self.period_steps = steps

    @property
    def period_offset(self) -> float:
        return self.period_offset_steps * self.dt

    @period_offset.setter
    def period_offset(self, val: float):
        steps = int(round(val / self.dt))
        if self._compiled() and steps != self.period_offset_steps:
            raise NotImplementedError("the recording offset is compiled into the network in this "
                                      "backend; set it before compile()")
        self.period_offset_steps = steps

    # -- control ----------------------------------------------------------------------
    def start(self, variables=None, period=None):
        """Start (or restart) recording (Monitor.py:375-435). Variables can be
        added before compile() only."""
        if variables is not None:
            variables = [variables] if isinstance(variables, str) else list(variables)
            new = [v for v in variables if v not in self.variables]
            if new and self._compiled():
                raise NotImplementedError("recorded variables are fixed at compile() in this "
                                          "backend")
            for v in new:
                self._check_variable(v)
                self.variables.append(v)
                if v != "spike":
                    self._data[v] = []
        if period is not None:
            self.period = period
        self._recording = True
        if self._compiled():
            self._start_step = self.net.current_step
        for v in self.variables:
            self._add_variable(v)

    def pause(self):
        self._recording = False
        for v in self.variables:
            self._recorded[v]["stop"][-1] = self._now()

    def resume(self):
        self._recording = True
        for v in self.variables:
            self._recorded[v]["start"].append(self._now())
            self._recorded[v]["stop"].append(None)

    def stop(self):
        self._recording = False

    def reset(self):
        """Empty the recordings and restart their timings (Monitor.py:543-552)."""
        self._data = {v: [] for v in self.variables if v != "spike"}
        self._spike_steps, self._spike_ranks = [], []
        self._record_steps = []
        self._start_step = 0
        for v in self.variables:
            self._add_variable(v)

    # -- results ------------------------------------------------------------------------
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

    def _spike_dict(self, keep: bool) -> dict:
        s, r = self.spike_arrays()
        size = self.population.size
        # by rank, steps stay ascending (radix sort for 16-bit ranks)
        key = r.astype(np.uint16) if size <= 65536 else r
        order = np.argsort(key, kind="stable")
        counts = np.bincount(r, minlength=size)
        offs = np.zeros(size + 1, dtype=np.int64)
        np.cumsum(counts, out=offs[1:])
        # one conversion to Python ints, then list slices per neuron; the
        # collector stays off meanwhile (thousands of new lists, no cycles: in
        # a process holding many objects its passes would cost more than the
        # construction)
        was_enabled = gc.isenabled()
        gc.disable()
        try:
            steps = s[order].tolist()
            lo, hi = offs[:-1].tolist(), offs[1:].tolist()
            if self.ranks is None:
                d = dict(zip(range(size), map(steps.__getitem__, map(slice, lo, hi))))
            else:
                d = {int(k): steps[lo[int(k)]:hi[int(k)]] for k in self.ranks}
        finally:
            if was_enabled:
                gc.enable()
        if not keep:
            self._spike_steps, self._spike_ranks = [], []
        return d

    def get(self, variables=None, keep: bool = False, reshape: bool = True,
            force_dict: bool = False):
        """Recorded values (Monitor.py:220-266): an array (time, neurons) per
        variable, reshaped to the population's geometry when `reshape` (not
        for views), or for 'spike' a dict rank -> steps; a dict when several
        variables (or none, meaning all) are asked for or `force_dict`."""
        if variables:
            if not isinstance(variables, list):
                variables = [variables]
        else:
            variables = list(self.variables)
            force_dict = True
        out = {}
        for v in variables:
            if v not in self.variables:
                raise ValueError(f"{v!r} is not recorded by this monitor")
            if v == "spike":
                out[v] = self._spike_dict(keep)
            else:
                chunks = self._data[v]
                n = self.population.size if self.ranks is None else len(self.ranks)
                arr = np.concatenate(chunks, axis=0) if chunks else np.zeros((0, n))
                if reshape and self.ranks is None:
                    arr = arr.reshape((arr.shape[0],) + tuple(self.population.geometry))
                out[v] = arr
                if not keep:
                    self._data[v] = []
            self._update_stopping_time(v, keep)
        if not keep:
            self._record_steps = []
        if not force_dict and len(variables) == 1:
            return out[variables[0]]
        return out

    def __getitem__(self, key):
        return self.get(key)

    def save(self, filename: str, variables=None, keep: bool = False, reshape: bool = False,
             force_dict: bool = False):
        """Save recorded values (Monitor.py:596-659): '.npy' holds one
        variable, '.hdf5' one dataset per variable (needs h5py)."""
        if variables:
            variables = variables if isinstance(variables, list) else [variables]
        else:
            variables = list(self.variables)
        if filename.endswith(".npy"):
            if len(variables) != 1:
                raise ValueError("Monitor.save: a .npy file holds a single variable")
            np.save(filename, self.get(variables[0], keep=keep, reshape=reshape))
        elif filename.endswith(".hdf5"):
            try:
                import h5py
            except ImportError as e:
                raise ImportError("Monitor.save: .hdf5 files need h5py") from e
            data = self.get(variables, keep=keep, reshape=reshape, force_dict=True)
            with h5py.File(filename, "w") as f:
                for var, val in data.items():
                    if var == "spike":
                        grp = f.create_group("/spike")
                        for rank, steps in val.items():
                            grp[str(rank)] = np.asarray(steps, dtype=np.int64)
                    else:
                        f["/" + var] = val
        else:
            raise ValueError("Monitor.save: file type not recognized (must be .hdf5 or .npy)")

    def times(self, variables=None):
        """Start and stop steps of the last retrieved recordings
        (Monitor.py:684-710)."""
        if variables:
            variables = variables if isinstance(variables, list) else [variables]
        else:
            variables = list(self.variables)
        return {v: copy.deepcopy(self._last_recorded[v]) for v in variables
                if v in self._last_recorded}

    # -- analysis (Monitor.py:712-995) -----------------------------------------------
    def _spikes_arg(self, spikes):
        if "spike" not in self.variables:
            raise ValueError("Monitor: spike was not recorded")
        if not spikes:
            return self.get("spike")
        if "spike" in spikes:
            return spikes["spike"]
        if "axon_spike" in spikes:
            return spikes["axon_spike"]
        return spikes

    def _window(self):
        rec = self._last_recorded["spike"]
        start = rec["start"][-1]
        stop = rec["stop"][-1] if rec["stop"][-1] is not None else self._now()
        return start, stop

    def raster_plot(self, spikes=None):
        """(times in ms, ranks) of every recorded spike, neuron by neuron."""
        return raster_plot(self._spikes_arg(spikes), dt=self.dt)

    def histogram(self, spikes=None, bins=None, per_neuron: bool = False, recording_window=None):
        return histogram(self._spikes_arg(spikes), bins=bins, per_neuron=per_neuron,
                         recording_window=recording_window, dt=self.dt)

    def inter_spike_interval(self, spikes=None, ranks=None, per_neuron: bool = False):
        return inter_spike_interval(self._spikes_arg(spikes), ranks=ranks, per_neuron=per_neuron,
                                    dt=self.dt)

    def coefficient_of_variation(self, spikes=None, ranks=None):
        return coefficient_of_variation(self._spikes_arg(spikes), ranks=ranks, dt=self.dt)

    def mean_fr(self, spikes=None):
        """Mean firing rate (Hz) of the recorded neurons over the last
        recording window."""
        data = self._spikes_arg(spikes)
        start, stop = self._window()
        neurons = list(self.ranks) if self.ranks is not None else range(self.population.size)
        count = sum(len(data[int(k)]) for k in neurons)
        return count / float(len(neurons)) / (stop - start) / self.dt * 1000.0

    def smoothed_rate(self, spikes=None, smooth: float = 0.0):
        """Per-neuron instantaneous rate (inverse inter-spike interval),
        exponentially smoothed; (neurons, steps) over the last window."""
        data = self._spikes_arg(spikes)
        start, stop = self._window()
        return _smoothed_rate(data, start, stop, smooth, self.dt)

    def population_rate(self, spikes=None, smooth: float = 0.0):
        """Population rate (Hz) per step over the last window, exponentially
        smoothed when smooth > dt."""
        data = self._spikes_arg(spikes)
        start, stop = self._window()
        return _population_rate(data, start, stop, smooth, self.dt)


# ------------------------------------------------------------ analysis functions
def raster_plot(spikes: dict, dt: float = 1.0):
    """(times in ms, ranks) of every spike of a dict rank -> steps, neuron by
    neuron (Monitor.py:1091-1108)."""
    times, ranks = [], []
    for n, steps in spikes.items():
        times.extend(steps)
        ranks.extend([n] * len(steps))
    return dt * np.array(times), np.array(ranks)


def _span(spikes: dict):
    lens = [s for s in spikes.values() if len(s)]
    return int(np.max([np.max(s) for s in lens])), int(np.min([np.min(s) for s in lens]))


def histogram(spikes: dict, bins: float | None = None, per_neuron: bool = False,
              recording_window=None, dt: float = 1.0):
    """Spike counts per bin of `bins` ms (default dt) from the first spike
    (or recording_window[0]) on (Monitor.py:1111-1169): int(bins / dt) steps
    per bin, int(duration / steps) + 1 bins; per neuron a (max rank + 1,
    bins) array."""
    if bins is None:
        bins = dt
    bin_step = int(bins / dt)
    if recording_window is None:
        t_max, t_min = _span(spikes)
    else:
        t_min, t_max = recording_window[0], recording_window[1]
    nb_bins = int((t_max - t_min) / bin_step)
    if per_neuron:
        histo = np.zeros((int(np.amax(list(spikes.keys()))) + 1, nb_bins + 1), dtype=np.int64)
    else:
        histo = np.zeros(nb_bins + 1, dtype=np.int64)
    for neuron, steps in spikes.items():
        if not len(steps):
            continue
        # int() truncates toward zero; a negative index counts from the end
        idx = np.trunc((np.asarray(steps, dtype=np.int64) - t_min) / float(bin_step)).astype(np.int64)
        if per_neuron:
            np.add.at(histo[neuron], idx, 1)
        else:
            np.add.at(histo, idx, 1)
    return histo


def inter_spike_interval(spikes: dict, ranks=None, per_neuron: bool = False, dt: float = 1.0):
    """Inter-spike intervals in ms of the neurons with at least two spikes
    (Monitor.py:1172-1207): a dict rank -> list, or one list."""
    isi = {}
    for rank, steps in spikes.items():
        if len(steps) < 2 or (ranks is not None and rank not in ranks):
            continue
        isi[rank] = (np.diff(np.asarray(steps, dtype=np.int64)) * dt).tolist()
    if per_neuron:
        return isi
    return [v for vals in isi.values() for v in vals]


def coefficient_of_variation(spikes: dict, ranks=None, per_neuron: bool = False, dt: float = 1.0):
    """Standard deviation over mean of each neuron's inter-spike intervals,
    for neurons with at least two intervals (Monitor.py:1210-1242)."""
    cv = {}
    for rank, values in inter_spike_interval(spikes, ranks=ranks, per_neuron=True, dt=dt).items():
        if len(values) < 2:
            continue
        cv[rank] = np.std(values) / np.mean(values)
    return cv if per_neuron else list(cv.values())


def mean_fr(spikes: dict, duration=None, dt: float = 1.0):
    """Mean firing rate (Hz) over `duration` steps (default: first to last
    spike) (Monitor.py:1300-1330)."""
    if duration is None:
        t_max, t_min = _span(spikes)
        duration = t_max - t_min
    count = sum(len(v) for v in spikes.values())
    return count / float(len(spikes)) / duration / dt * 1000.0


def _smoothed_rate(spikes: dict, start: int, stop: int, smooth: float, dt: float):
    """Transformations.pyx:23-66 with its float32 step size: the inverse of
    each inter-spike interval fills columns [previous spike, spike) (absolute
    steps, as there), then first-order smoothing with delta = dt / smooth."""
    dt32 = np.float32(dt)
    d = int(stop) - int(start)
    rates = np.zeros((len(spikes), d))
    first = int(start) - int(100.0 / float(dt32))
    for idx, steps in enumerate(spikes.values()):
        last = first
        for timing in steps:
            if last > start:
                rates[idx, last:timing] = 1000.0 / float(dt32) / float(timing - last)
            last = timing
    s32 = np.float32(smooth)
    if s32 == 0.0:
        return rates
    out = np.zeros((len(spikes), d))
    out[:, 0] = rates[:, 0]
    delta = float(np.float32(dt32 / s32))
    for t in range(d - 1):
        out[:, t + 1] = out[:, t] + (rates[:, t + 1] - out[:, t]) * delta
    return out


def _population_rate(spikes: dict, start: int, stop: int, smooth: float, dt: float):
    """Transformations.pyx:68-108: spike counts per step from `start` to
    `stop` (inclusive) over dt * N / 1000 (dt float32), then first-order
    smoothing with delta = dt / smooth when smooth > dt."""
    dt32 = np.float32(dt)
    d = int(stop) - int(start) + 1
    rates = np.zeros(d)
    for steps in spikes.values():
        for t in steps:
            rates[t - start] += 1
    rates /= float(np.float32(dt32 * np.float32(len(spikes)))) / 1000.0
    s32 = np.float32(smooth)
    if s32 <= dt32:
        return rates
    out = np.zeros(d)
    out[0] = rates[0]
    delta = float(np.float32(dt32 / s32))
    for t in range(d - 1):
        out[t + 1] = out[t] + (rates[t + 1] - out[t]) * delta
    return out


def smoothed_rate(spikes: dict, smooth: float = 0.0, dt: float = 1.0):
    """Per-neuron smoothed rate between the first and last spike
    (Monitor.py:1272-1296)."""
    t_max, t_min = _span(spikes)
    return _smoothed_rate(spikes, t_min, t_max, smooth, dt)


def population_rate(spikes: dict, smooth: float = 0.0, dt: float = 1.0):
    """Population rate between the first and last spike (Monitor.py:1245-1269)."""
    t_max, t_min = _span(spikes)
    return _population_rate(spikes, t_min, t_max, smooth, dt)
