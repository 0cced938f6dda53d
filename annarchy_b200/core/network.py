"""Network: container of populations, projections and monitors.

Same methods as the reference's Network (ANNarchy/core/Network.py:73-1521):
create / connect / monitor / compile / simulate / step / get_time ...
compile() generates and loads the network's CUDA module instead of
generating C++ and running CMake (Network.py:517, Compiler.py:81-320).

Configuration (``Network.config``):
  precision    "double" (default): reference operation order, bit-identical
               results; "float": fast single-precision kernels.
  weight_dtype "float32" or "bfloat16" storage of static weights (float mode).
  engine       "auto" | "grid" | "local" (see annarchy_b200.generator.codegen).
  graph_steps  steps captured per CUDA graph in the grid engine.
  pdl          True (default) | False: launch the grid engine's step kernels
               with programmatic dependent launch (each may be scheduled
               while its predecessor runs and waits for it on the device).
  persistent   True | False (default): run the grid engine's step as one
               cooperative persistent kernel with grid-wide barriers (fast
               spiking networks).
  device       CUDA device index.
"""
from __future__ import annotations

import math
import time
import weakref

import numpy as np

from .monitor import Monitor
from .population import Population
from .projection import Projection

_NETWORK_IDS = [0]


class Network:
    def __init__(self, dt: float = 1.0, seed: int | None = None):
        _NETWORK_IDS[0] += 1
        self.id = _NETWORK_IDS[0]
        self.dt = float(dt)
        self.seed = seed
        self._rng = np.random.default_rng(seed)
        self._rng_state = self._rng.bit_generator.state
        self.populations: list[Population] = []
        self.projections: list[Projection] = []
        self.monitors: list[Monitor] = []
        self._config = {"precision": "double", "weight_dtype": None, "engine": "auto",
                        "graph_steps": 32, "device": 0}
        self._compiled = False
        self._backend = None
        self._t_python = 0
        # constants usable in equations: the global ones, then this network's
        self._constants: dict[str, Constant] = {}
        for c in GLOBAL_CONSTANTS.values():
            self._constants[c.name] = Constant(c.name, c.value, net=self)
        _LIVE.add(self)
        self._callbacks: list = []            # `every` decorators (Simulate.py:352-446)
        self._callbacks_enabled = True

    # ----------------------------------------------------------- construction
    def config(self, **kwargs):
        for key, val in kwargs.items():
            if key in ("dtype", "precision"):
                name = getattr(val, "__name__", str(val))
                val = {"float": "float", "float32": "float", "single": "float",
                       "double": "double", "float64": "double"}.get(name, name)
                key = "precision"
            if key == "paradigm" and val not in ("b200", "cuda"):
                raise ValueError("this backend only runs on the GPU (paradigm='b200')")
            if key in ("num_threads", "paradigm", "seed", "verbose", "sparse_matrix_format",
                       "method"):
                if key == "seed" and val is not None:
                    self.seed = val
                    self._rng = np.random.default_rng(val)
                    self._rng_state = self._rng.bit_generator.state
                if key == "sparse_matrix_format":
                    self._config["default_format"] = val
                continue
            self._config[key] = val
        return self

    def create(self, geometry=None, neuron=None, name: str | None = None, population=None,
               stop_condition: str | None = None, **kw) -> Population:
        """A population of `neuron`, or (as the reference's
        net.create(PoissonPopulation(...))) a population object built outside
        the network, which then joins it."""
        if self._compiled:
            raise RuntimeError("the network is already compiled")
        if population is not None:
            geometry = population
        if isinstance(geometry, Population):
            pop = geometry
            if pop.net is not None and pop.net is not self:
                raise ValueError("the population belongs to another network")
            object.__setattr__(pop, "net", self)
            object.__setattr__(pop, "id", len(self.populations))
            if name is not None or pop.__dict__.get("_auto_name", False):
                object.__setattr__(pop, "name", name or f"pop{pop.id}")
        else:
            if neuron is None:
                raise TypeError("create() needs a neuron type")
            pop = Population(geometry, neuron, name=name, net=self, pop_id=len(self.populations),
                             stop_condition=stop_condition)
        if stop_condition is not None and isinstance(geometry, Population):
            object.__setattr__(pop, "stop_condition", stop_condition)
        self.populations.append(pop)
        return pop

    def connect(self, pre, post, target: str = "exc", synapse=None, name: str | None = None,
                **kw) -> Projection:
        if self._compiled:
            raise RuntimeError("the network is already compiled")
        proj = Projection(pre, post, target, synapse=synapse, name=name, net=self,
                          proj_id=len(self.projections))
        if "default_format" in self._config:
            proj._storage_format = self._config["default_format"]
        self.projections.append(proj)
        return proj

    def monitor(self, obj, variables=None, period: float | None = None,
                period_offset: float | None = None, start: bool = True,
                name: str | None = None) -> Monitor:
        if self._compiled:
            raise RuntimeError("monitors must be created before compile() in this backend")
        mon = Monitor(obj, variables, period=period, period_offset=period_offset, start=start,
                      name=name, net=self, mon_id=len(self.monitors))
        self.monitors.append(mon)
        return mon

    # ------------------------------------------------------------ compilation
    def compile(self, directory: str | None = None, clean: bool = False, silent: bool = True,
                **kwargs):
        """Generate, compile (NVRTC, sm_100a) and load the network's kernels,
        and copy every population and projection to the device."""
        from .backend import CompiledNetwork
        if self._compiled:
            return
        if not self.populations:
            raise RuntimeError("the network has no population")
        backend = CompiledNetwork(self)
        backend.build()
        self._backend = backend
        self._compiled = True

    def generate_code(self):
        """Generate the network's CUDA module without a device (for
        inspection and compile-only checks); returns the codegen Module."""
        from .backend import CompiledNetwork
        backend = CompiledNetwork(self, dry=True)
        backend.build()
        return backend.module

    @property
    def compiled(self) -> bool:
        return self._compiled

    @property
    def engine(self) -> str | None:
        return self._backend.engine if self._backend else None

    # ------------------------------------------------------------- simulation
    def _steps(self, duration: float) -> int:
        return int(math.ceil(float(duration) / self.dt))

    def simulate(self, duration: float, measure_time: bool = False, callbacks: bool = True):
        if not self._compiled:
            raise RuntimeError("simulate(): the network is not compiled yet")
        n = self._steps(duration)
        t0 = time.time()
        if callbacks and self._callbacks_enabled and self._callbacks:
            self._simulate_with_callbacks(duration)
        else:
            self._backend.run(n)
        if measure_time:
            print(f"Simulating {duration / 1000.0} seconds of the network took "
                  f"{time.time() - t0} seconds.")

    # -- constants (ANNarchy/core/Network.py:482-510, core/Constant.py) -------------------
    def constant(self, name: str, value: float) -> "Constant":
        """A constant usable by name in every equation of this network."""
        if self._compiled:
            raise RuntimeError("constants must be added before compile() in this backend")
        c = Constant(name, value, net=self)
        self._constants[name] = c
        return c

    def get_constant(self, name: str) -> "Constant":
        return self._constants[name]

    def get_constants(self) -> list:
        return list(self._constants.values())

    # -- accessors (ANNarchy/core/Network.py) -------------------------------------------
    def get_population(self, name: str) -> Population:
        for pop in self.populations:
            if pop.name == name:
                return pop
        raise ValueError(f"get_population(): no population named {name!r}")

    def get_projection(self, name: str) -> Projection:
        for proj in self.projections:
            if proj.name == name:
                return proj
        raise ValueError(f"get_projection(): no projection named {name!r}")

    def get_monitor(self, name: str) -> Monitor:
        for mon in self.monitors:
            if mon.name == name:
                return mon
        raise ValueError(f"get_monitor(): no monitor named {name!r}")

    def get_populations(self) -> list:
        return list(self.populations)

    def get_projections(self, post=None, pre=None, target=None, suppress_error: bool = False) -> list:
        """Projections, optionally only those onto `post`, from `pre` or with
        `target`."""
        res = [p for p in self.projections
               if (post is None or p.post_pop is _pop_of(post))
               and (pre is None or p.pre_pop is _pop_of(pre))
               and (target is None or p.target == target)]
        if not res and not suppress_error and (post is not None or pre is not None or target is not None):
            raise ValueError("get_projections(): no matching projection")
        return res

    def get_monitors(self) -> list:
        return list(self.monitors)

    @property
    def time(self) -> float:
        """Current simulated time in ms."""
        return self.get_time()

    @time.setter
    def time(self, value: float):
        self.set_time(value)

    def enable_learning(self, projections=None, period: float | None = None,
                        offset: float | None = None):
        """Learning on for the given projections (default: all)."""
        for proj in projections or self.projections:
            proj.enable_learning(period=period, offset=offset)

    def disable_learning(self, projections=None):
        """Learning off for the given projections (default: all)."""
        for proj in projections or self.projections:
            proj.disable_learning()

    def simulate_until(self, max_duration: float, population, operator: str = "and",
                       measure_time: bool = False) -> float:
        """Simulate at most max_duration ms and stop after the first step at
        which the stop conditions of `population` (one or a list) hold: all
        of them (operator "and") or any ("or") (ANNarchy/core/Simulate.py:
        174-242, Network.simulate_until). Returns the simulated duration in
        ms."""
        if not self._compiled:
            raise RuntimeError("simulate_until(): the network is not compiled yet")
        import math
        n = int(math.ceil(float(max_duration) / self.dt))
        pops = population if isinstance(population, (list, tuple)) else [population]
        t0 = time.time()
        done = self._backend.run_until(n, list(pops), operator == "and")
        if measure_time:
            print(f"Simulating {done * self.dt / 1000.0} seconds of the network took "
                  f"{time.time() - t0} seconds.")
        return done * self.dt

    # -- callbacks (ANNarchy/core/Simulate.py:314-446) -------------------------------
    def callback_times(self, t_start: int, duration: float) -> list:
        """(step, callback, n) of every call during a simulation of
        `duration` ms from step t_start, in time order (declaration order at
        equal steps)."""
        length = int(duration / self.dt)
        times = []
        for c in self._callbacks:
            period = int(c.period / self.dt)
            offset = int(c.offset / self.dt) % period
            wait = int(c.wait / self.dt)
            for n, m in enumerate(range(t_start + wait + offset, t_start + length, period)):
                times.append((m, c, n))
        return sorted(times, key=lambda x: x[0])

    def _simulate_with_callbacks(self, duration: float):
        t_start = self.current_step
        length = int(duration / self.dt)
        for step, cb, n in self.callback_times(t_start, duration):
            if step != self.current_step:
                self._backend.run(step - self.current_step)
            cb.func(n)
        if self.current_step < t_start + length:
            self._backend.run(t_start + length - self.current_step)

    def callbacks_enabled(self) -> bool:
        return self._callbacks_enabled

    def enable_callbacks(self):
        self._callbacks_enabled = True

    def disable_callbacks(self):
        self._callbacks_enabled = False

    def clear_all_callbacks(self):
        self._callbacks.clear()

    def simulate_steps(self, nsteps: int):
        if not self._compiled:
            raise RuntimeError("the network is not compiled yet")
        self._backend.run(int(nsteps))

    def step(self):
        self.simulate_steps(1)

    @property
    def current_step(self) -> int:
        return self._backend.native.get_time() if self._compiled else 0

    def get_current_step(self) -> int:
        return self.current_step

    def get_time(self) -> float:
        return self.current_step * self.dt

    def set_current_step(self, t: int):
        nat = self._backend.native
        nat.set_time(int(t))
        # the spike lists are indexed by step parity: a new time starts them empty
        for pop in self.populations:
            if f"pop{pop.id}__spn" in nat.arrays:
                nat.zero(f"pop{pop.id}__spn")

    def set_time(self, t: float):
        self.set_current_step(int(round(t / self.dt)))

    def save(self, filename: str, populations: bool = True, projections: bool = True):
        """Network state into a file in the reference's layout
        (ANNarchy/core/IO.py:398-431): .npz, .gz, .mat (not loadable) or pickle."""
        from .io import network_description, save_data
        save_data(filename, network_description(self, populations, projections))

    def load(self, filename: str, populations: bool = True, projections: bool = True,
             pickle_encoding: str | None = None):
        """State saved by save() (or by the reference's save()); before
        compile() it also gives the projections their connectivity."""
        from .io import load_data, load_network
        load_network(self, load_data(filename, pickle_encoding), populations, projections)

    def reset(self, populations: bool = True, projections: bool = False, synapses: bool = False,
              monitors: bool = True, reseed_rng: bool = True):
        """Back to the state after compile() (ANNarchy/core/Network.py:628-675):
        time 0; with `populations`, every neural attribute at its initial
        value, no spikes in flight, the delay queues refilled with the
        initial rates; with `projections`, the synaptic variables (not the
        weights) at their initial values; with `monitors`, the recordings
        emptied; with `reseed_rng`, the network's generator back to its seed."""
        if synapses:
            raise NotImplementedError("reset(synapses=True): recreating the connectivity is not "
                                      "supported by this backend")
        if self._compiled:
            self.set_current_step(0)
            if populations:
                for pop in self.populations:
                    pop.reset()
            if projections:
                for proj in self.projections:
                    self._backend.reset_projection(proj)
        if monitors:
            for mon in self.monitors:
                mon.reset()
        if reseed_rng:
            self._rng.bit_generator.state = self._rng_state

    # ---------------------------------------------------------------- access
    def get_population(self, name: str) -> Population:
        for p in self.populations:
            if p.name == name:
                return p
        raise KeyError(name)

    def get_projection(self, name: str) -> Projection:
        for p in self.projections:
            if p.name == name:
                return p
        raise KeyError(name)

    def get_monitors(self):
        return list(self.monitors)

    def close(self):
        if self._backend is not None:
            self._backend.native.close()
            self._backend = None
        self._compiled = False

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _pop_of(obj):
    return obj.population if hasattr(obj, "population") and not isinstance(obj, Population) else obj


GLOBAL_CONSTANTS: dict[str, "Constant"] = {}


class Constant(float):
    """A named value usable in the equations of every neuron and synapse
    (ANNarchy/core/Constant.py): `Constant(name, value)` at the module level
    is seen by the networks created afterwards, `net.constant(name, value)`
    by one network. An attribute of the same name hides it. `set()` changes
    the value, also after compile(); a constant built from others keeps the
    value it had."""

    def __new__(cls, name: str, value: float, net=None):
        return float.__new__(cls, value)

    def __init__(self, name: str, value: float, net=None):
        self.name = name
        self.value = float(value)
        self.net = net
        if net is None:
            GLOBAL_CONSTANTS[name] = self

    def set(self, value: float):
        """New value (for the networks created from a global constant: in each)."""
        self.value = float(value)
        nets = [self.net] if self.net is not None else [n for n in _LIVE if name_in(n, self.name)]
        for n in nets:
            c = n._constants.get(self.name)
            if c is not None and c is not self:
                c.value = float(value)
            if n._compiled:
                n._backend.native.set_constant(self.name, float(value))

    def __repr__(self):
        return f"Constant({self.name!r}, {self.value})"


def name_in(net, name: str) -> bool:
    return name in getattr(net, "_constants", {})


_LIVE = weakref.WeakSet()             # networks that see the global constants


class every:
    """Decorator of a function called periodically during simulate()
    (ANNarchy/core/Simulate.py:352-406): every `period` ms (at least dt),
    `offset` ms into the period (negative: from its end), after `wait` ms,
    counted from the start of each simulate() call; the function receives
    the call count n.

        @every(network=net, period=100.0, offset=-10.0)
        def step_input(n):
            pop.I = float(n) / 100.0
    """

    def __init__(self, network=None, period: float = 1.0, offset: float = 0.0, wait: float = 0.0):
        if network is None:
            raise ValueError("every(): pass the network (this backend has no default network)")
        self.network = network
        network._callbacks.append(self)
        self.period = max(float(period), network.dt)
        self.offset = min(float(offset), self.period)
        self.wait = max(float(wait), 0.0)
        self.func = None

    def __call__(self, f):
        self.func = f
        return f
