"""Populations and population views.

Attribute access follows the reference (ANNarchy/core/Population.py:375-500):
every parameter and variable of the neuron type is an attribute; local
ones are arrays of the population's size, global ones scalars. Before
compile() values live on the host; afterwards the device arrays are the
state and every get/set copies through the C ABI (like the reference's
pop<k>_wrapper properties, which also copy).

The refractory period is given in ms and converted to whole steps by
truncation, int(refractory / dt) (Population.py:659-690).
"""
from __future__ import annotations

import numpy as np

from .random import RandomDistribution, values as draw

_RESERVED = {"size", "geometry", "neuron_type", "name", "id", "ranks", "net", "refractory",
             "desc", "population", "targets", "attributes"}


class Population:
    def __init__(self, geometry, neuron, name: str | None = None, net=None, pop_id: int = 0,
                 stop_condition=None, storage_order="post_to_pre", copied=False):
        if isinstance(geometry, int):
            geometry = (geometry,)
        object.__setattr__(self, "_ready", False)
        self.geometry = tuple(int(g) for g in geometry)
        self.size = int(np.prod(self.geometry))
        self.neuron_type = neuron
        self.net = net
        self.id = pop_id
        self.stop_condition = stop_condition
        self.name = name or f"pop{pop_id}"
        self.desc = neuron.desc
        self.targets = list(self.desc["targets"])
        self._host: dict[str, np.ndarray] = {}
        self._ctype: dict[str, str] = {}
        self._locality: dict[str, str] = {}
        for p in self.desc["parameters"] + self.desc["variables"]:
            self._locality[p["name"]] = p["locality"]
            self._ctype[p["name"]] = p.get("ctype", "double")
        for p in self.desc["parameters"] + self.desc["variables"]:
            self._host[p["name"]] = self._initial(p)
        self._globalops = []
        for op in self.desc.get("global_operations", []):
            self._add_globalop(op)
        if self.neuron_type.type == "rate":
            for t in self.targets:
                self._host["_sum_" + t] = np.zeros(self.size)
                self._locality["_sum_" + t] = "local"
                self._ctype["_sum_" + t] = "double"
        refr = self.neuron_type.refractory if self.neuron_type.type == "spike" else None
        self._refractory_ms = np.full(self.size, float(refr or 0.0))
        self._has_refractory = bool(refr)
        object.__setattr__(self, "_ready", True)

    def _add_globalop(self, op: dict):
        """A population-wide reduction (the previous step's value) that the
        neuron's or a projection's equations use: `_<op>_<variable>`."""
        if op["variable"] not in self.desc["local"]:
            raise ValueError(f"{op['function']}({op['variable']}): {op['variable']!r} is not a "
                             f"local attribute of {self.name!r}")
        if op in self._globalops:
            return
        self._globalops.append(dict(op))
        name = "_" + op["function"] + "_" + op["variable"]
        self._host[name] = np.float64(0.0)
        self._locality[name] = "global"
        self._ctype[name] = "double"

    def _add_spike_target(self, target: str):
        """A projection's target that the spiking neuron's equations do not
        mention: a conductance g_<target> that only the transmissions change
        (the reference adds the target to the population,
        ANNarchy/core/Projection.py:105-110, and declares g_<target>)."""
        if target in self.targets:
            return
        self.targets.append(target)
        name = "g_" + target
        if name not in self._host:
            self._host[name] = np.zeros(self.size)
            self._locality[name] = "local"
            self._ctype[name] = "double"

    def _add_rate_target(self, target: str):
        """A projection's target that the neuron's equations do not use: its
        weighted sum array (zero until compile)."""
        if target in self.targets:
            return
        self.targets.append(target)
        self._host["_sum_" + target] = np.zeros(self.size)
        self._locality["_sum_" + target] = "local"
        self._ctype["_sum_" + target] = "double"

    # -- helpers --------------------------------------------------------------
    def _initial(self, p):
        init = p["init"]
        shape = (self.size,) if p["locality"] == "local" else ()
        dtype = np.int32 if p.get("ctype") in ("int", "bool") else np.float64
        if isinstance(init, str):
            ref = [q for q in self.desc["parameters"] if q["name"] == init]
            if not ref:
                raise ValueError(f"init value {init!r} of {p['name']} is not a parameter")
            init = ref[0]["init"]
        if isinstance(init, RandomDistribution):
            return draw(init, shape, self._rng(), dtype)
        return np.full(shape, init, dtype=dtype)

    def _rng(self):
        return self.net._rng if self.net is not None else np.random.default_rng()

    def _device_name(self, attr: str) -> str:
        return f"pop{self.id}__{attr}"

    @property
    def attributes(self):
        return list(self.desc["attributes"])

    @property
    def parameters(self):
        """Names of the neuron's parameters (Population.py, `parameters`)."""
        return [p["name"] for p in self.desc["parameters"]]

    @property
    def variables(self):
        """Names of the neuron's variables (Population.py, `variables`)."""
        return [v["name"] for v in self.desc["variables"]]

    @property
    def ranks(self):
        return np.arange(self.size)

    @property
    def population(self):
        return self

    def _compiled(self) -> bool:
        return self.net is not None and self.net._compiled

    # -- attribute access -----------------------------------------------------
    def __getattr__(self, name):
        if name.startswith("__") or not object.__getattribute__(self, "_ready"):
            raise AttributeError(name)
        host = object.__getattribute__(self, "_host")
        if name in host:
            return self.get(name)
        fn = _model_function(self.desc, name)
        if fn is not None:
            return fn
        raise AttributeError(f"population {self.name!r} has no attribute {name!r}")

    def __setattr__(self, name, value):
        if not self.__dict__.get("_ready", False) or name.startswith("_") and name not in self._host:
            object.__setattr__(self, name, value)
            return
        if name in self._host:
            self.set({name: value})
            return
        if name == "refractory":
            self.set_refractory(value)
            return
        object.__setattr__(self, name, value)

    def get(self, name: str):
        if self._compiled():
            arr = self.net._backend.read_population_attribute(self, name)
        else:
            arr = self._host[name].copy()
        if self._locality.get(name) != "local":
            return arr.reshape(()).item()
        return arr.reshape(self.geometry) if len(self.geometry) > 1 else arr

    def set(self, values: dict):
        for name, value in values.items():
            if name not in self._host:
                raise AttributeError(f"population {self.name!r} has no attribute {name!r}")
            cur = self._host[name]
            if self._compiled() and isinstance(value, np.ndarray) and value.size == cur.size:
                # straight to the device: no host copy when the array already
                # has the device dtype (e.g. a pinned buffer)
                self.net._backend.write_population_attribute(self, name, value)
                continue
            arr = draw(value, cur.shape, self._rng(), cur.dtype)
            if self._compiled():
                self.net._backend.write_population_attribute(self, name, arr)
            else:
                self._host[name] = arr

    def _set_ranks(self, name: str, ranks: np.ndarray, value):
        if self._locality.get(name) != "local":
            raise AttributeError(f"{name} is global; set it on the population")
        cur = self.get(name).reshape(-1).astype(self._host[name].dtype)
        cur[ranks] = draw(value, (len(ranks),), self._rng(), cur.dtype)
        self.set({name: cur})

    def reset(self, attributes=None):
        """Attributes (all, or the listed ones) back to the values they had at
        compile() (ANNarchy/core/Population.py:309-353), spikes and delay
        queues cleared as by the reference's PopStruct::reset()."""
        if attributes is not None:
            for a in attributes:
                if a not in self._host:
                    raise AttributeError(f"population {self.name!r} has no attribute {a!r}")
        if self._compiled():
            self.net._backend.reset_population(self, attributes)
        else:
            for p in self.desc["parameters"] + self.desc["variables"]:
                if attributes is None or p["name"] in attributes:
                    self._host[p["name"]] = self._initial(p)

    def sum(self, target: str):
        """Weighted sum of the inputs on `target` computed in the last step
        (rate-coded populations; ANNarchy/core/Population.py, sum)."""
        if self.neuron_type.type != "rate":
            raise NotImplementedError("sum(target) is available for rate-coded populations")
        if target not in self.targets:
            raise ValueError(f"population {self.name!r} has no target {target!r}")
        if not self._compiled():
            return np.zeros(self.geometry if len(self.geometry) > 1 else self.size)
        arr = self.net._backend.native.read(f"pop{self.id}___last_sum_{target}").astype(np.float64)
        return arr.reshape(self.geometry) if len(self.geometry) > 1 else arr

    def save(self, filename: str):
        """Every parameter and variable into a file (.npz, .gz, .mat or
        pickle), in the reference's layout (Population.py:1000-1066)."""
        from .io import population_data, save_data
        save_data(filename, population_data(self))

    def load(self, filename: str, pickle_encoding: str | None = None):
        """Attributes from a file saved by save() (or by the reference)."""
        from .io import load_data, load_population_data
        load_population_data(self, load_data(filename, pickle_encoding))

    # -- coordinates (ANNarchy/core/Population.py:915-1000) ---------------------------
    def rank_from_coordinates(self, coord) -> int:
        """Rank of the neuron at `coord` (row-major)."""
        coord = tuple(int(c) for c in np.atleast_1d(coord))
        if len(coord) != len(self.geometry) or any(not 0 <= c < g for c, g in zip(coord, self.geometry)):
            raise ValueError(f"rank_from_coordinates(): there is no neuron of coordinates {coord} "
                             f"in the population {self.name} {self.geometry}")
        return int(np.ravel_multi_index(coord, self.geometry))

    def coordinates_from_rank(self, rank: int) -> tuple:
        """Coordinates of neuron `rank` (row-major)."""
        if not 0 <= int(rank) < self.size:
            raise ValueError(f"the given rank {rank} is larger than the size of the population "
                             f"{self.size}")
        c = np.unravel_index(int(rank), self.geometry)
        return tuple(int(x) for x in c)

    def normalized_coordinates_from_rank(self, rank: int, norm: float = 1.0) -> tuple:
        """Coordinates mapped to [0, 1]^d. Up to three dimensions the
        reference rounds them to float32 and ignores `norm`
        (cython_ext/Coordinates.pyx:122-176); beyond, norm * c / (extent - 1)."""
        coord = self.coordinates_from_rank(rank)
        if len(self.geometry) <= 3:
            return tuple(float(np.float32(c / (g - 1))) if g > 1 else 0.0
                         for c, g in zip(coord, self.geometry))
        return tuple(norm * float(c) / float(g - 1) if g > 1 else 0.0
                     for c, g in zip(coord, self.geometry))

    def enable(self):
        """Not supported: populations are always updated in this backend."""
        raise NotImplementedError("Population.enable()/disable() are not supported by this backend")

    def disable(self):
        """Not supported: populations are always updated in this backend."""
        raise NotImplementedError("Population.enable()/disable() are not supported by this backend")

    def compute_firing_rate(self, window: float):
        """Not supported (record spikes with a monitor and use its
        population_rate() or smoothed_rate())."""
        raise NotImplementedError("Population.compute_firing_rate() is not supported by this "
                                  "backend; record spikes and use Monitor.smoothed_rate()")

    @property
    def dimension(self) -> int:
        return len(self.geometry)

    @property
    def refractory(self):
        """Refractory period in ms (a value, or one per neuron when they differ)."""
        r = self._refractory_ms
        return float(r[0]) if r.size and np.all(r == r[0]) else r.copy()

    def set_refractory(self, value):
        object.__setattr__(self, "_refractory_steps", None)
        self._refractory_ms = draw(value, (self.size,), self._rng())
        self._has_refractory = self._has_refractory or bool(np.any(self._refractory_ms > 0))
        if self._compiled():
            self.net._backend.write_refractory(self)

    @property
    def refractory_steps(self) -> np.ndarray:
        steps = self.__dict__.get("_refractory_steps")
        if steps is not None:
            return steps
        dt = self.net.dt if self.net is not None else 1.0
        return (self._refractory_ms / dt).astype(np.int32)  # truncation, like int(x/dt)

    def _set_refractory_steps(self, steps: np.ndarray):
        """Refractory periods given in whole steps (as the reference's Python
        layer hands them to its generated module, already truncated)."""
        steps = np.broadcast_to(np.asarray(steps, dtype=np.int32), (self.size,)).copy()
        dt = self.net.dt if self.net is not None else 1.0
        object.__setattr__(self, "_refractory_steps", steps)
        object.__setattr__(self, "_refractory_ms", steps * dt)
        self._has_refractory = self._has_refractory or bool(np.any(steps > 0))
        if self._compiled():
            self.net._backend.write_refractory(self)

    # -- views ----------------------------------------------------------------
    def __getitem__(self, idx):
        """A rank, a slice or a list of ranks gives a view; coordinates
        without slices give that neuron; coordinates with slices give the
        view of the neurons they cover, in row-major order
        (ANNarchy/core/Population.py:782-890)."""
        if isinstance(idx, tuple):
            if not any(isinstance(i, slice) for i in idx):
                return self.neuron(idx)
            grid = np.arange(self.size).reshape(tuple(self.geometry))
            return PopulationView(self, np.asarray(grid[idx]).reshape(-1))
        ranks = np.arange(self.size)[idx]
        return PopulationView(self, np.atleast_1d(ranks))

    def __len__(self):
        return self.size

    def __repr__(self):
        return f"Population({self.name!r}, size={self.size}, {self.neuron_type.type})"

    def neuron(self, *coord) -> "IndividualNeuron":
        """The neuron of the given rank or coordinates
        (ANNarchy/core/Population.py:728-757)."""
        if len(coord) == 1 and isinstance(coord[0], (int, np.integer)):
            rank = int(coord[0])
        else:
            rank = self.rank_from_coordinates(coord[0] if len(coord) == 1 else tuple(coord))
        if rank is None or not 0 <= rank < self.size:
            raise IndexError(f"population {self.name!r} has no neuron {coord}")
        return IndividualNeuron(self, rank)

    def neurons(self):
        """Every neuron of the population, in rank order."""
        return (IndividualNeuron(self, r) for r in range(self.size))

    # spikes of the last step (spiking populations)
    @property
    def spiked(self):
        if not self._compiled():
            return np.array([], dtype=np.int64)
        return self.net._backend.read_spiked(self)


def _model_function(desc, name):
    """A model's own user function as a host callable, or None."""
    funcs = {f["name"]: f for f in desc.get("functions", [])}
    if name not in funcs:
        return None
    from .functions import evaluator
    return evaluator(funcs[name], {k: v for k, v in funcs.items() if k != name})


class PopulationView:
    """A subset of a population's neurons (ANNarchy/core/PopulationView.py)."""

    def __init__(self, population: Population, ranks):
        object.__setattr__(self, "population", population)
        object.__setattr__(self, "ranks", np.asarray(ranks, dtype=np.int64))
        object.__setattr__(self, "size", int(len(ranks)))

    @property
    def id(self):
        return self.population.id

    @property
    def neuron_type(self):
        return self.population.neuron_type

    @property
    def net(self):
        return self.population.net

    def __getattr__(self, name):
        if name.startswith("__"):
            raise AttributeError(name)
        pop = object.__getattribute__(self, "population")
        val = pop.get(name)
        if np.ndim(val) == 0:
            return val
        return np.asarray(val).reshape(-1)[self.ranks]

    def __setattr__(self, name, value):
        self.population._set_ranks(name, self.ranks, value)

    def __getitem__(self, idx):
        return PopulationView(self.population, self.ranks[idx])

    def __len__(self):
        return self.size

    def __repr__(self):
        return f"PopulationView({self.population.name!r}, size={self.size})"

    def __add__(self, other):
        """The union of two views (or a view and a neuron) of the same
        population, in ascending rank (ANNarchy/core/PopulationView.py:
        320-332)."""
        return _join(self, other)


def _join(a, b):
    pa = a.population if not isinstance(a, Population) else a
    pb = b.population if not isinstance(b, Population) else b
    if pa is not pb:
        raise ValueError("can only add two PopulationViews of the same population")
    ranks = lambda x: np.arange(x.size) if isinstance(x, Population) else np.asarray(x.ranks)
    return PopulationView(pa, np.array(sorted(set(ranks(a).tolist()) | set(ranks(b).tolist()))))


class IndividualNeuron:
    """One neuron of a population: its attributes read and written by rank
    (ANNarchy/core/Neuron.py:219-300)."""

    def __init__(self, population: Population, rank: int):
        object.__setattr__(self, "population", population)
        object.__setattr__(self, "rank", int(rank))

    @property
    def ranks(self):
        return np.array([self.rank], dtype=np.int64)

    @property
    def size(self):
        return 1

    @property
    def id(self):
        return self.population.id

    @property
    def neuron_type(self):
        return self.population.neuron_type

    @property
    def net(self):
        return self.population.net

    def __getattr__(self, name):
        if name.startswith("__"):
            raise AttributeError(name)
        val = self.population.get(name)
        if np.ndim(val) == 0:
            return val
        return np.asarray(val).reshape(-1)[self.rank]

    def __setattr__(self, name, value):
        self.population._set_ranks(name, np.array([self.rank]), value)

    def __add__(self, other):
        return _join(self, other)

    def __repr__(self):
        return f"IndividualNeuron({self.population.name!r}, rank={self.rank})"
