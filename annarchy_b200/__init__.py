"""annarchy_b200 — a B200-native simulation backend with the Python API of
the ANNarchy neural simulator.

    import annarchy_b200 as ann
    net = ann.Network(dt=0.1, seed=42)
    pop = net.create(4000, ann.Neuron(parameters=..., equations=..., spike=..., reset=...))
    proj = net.connect(pop[:3200], pop, "exc")
    proj.from_sparse(W)
    m = net.monitor(pop, "spike")
    net.compile()
    net.simulate(1000.0)
    spikes = m.get("spike")
"""
from .core.models import (IF_cond_exp, LeakyIntegrator, Neuron, Parameter, STDP, Synapse, Variable,
                          add_function, functions)
from .core.inputs import PoissonPopulation, TimedArray
from .core.monitor import Monitor
from .core.network import Constant, Network, every
from .core.population import Population, PopulationView
from .core.projection import LILConnectivity, Projection
from .core.rate_batch import RateBatch
from .core.random import (DiscreteUniform, Exponential, LogNormal, Normal, RandomDistribution,
                          Uniform)

float32 = "float"
float64 = "double"
__version__ = "0.1.0"

__all__ = ["Network", "Neuron", "Synapse", "Population", "PopulationView", "Projection",
           "Monitor", "PoissonPopulation", "TimedArray", "Uniform", "Normal", "LogNormal", "Exponential", "DiscreteUniform",
           "RandomDistribution", "LeakyIntegrator", "IF_cond_exp", "STDP", "float32", "float64",
           "Constant", "every", "RateBatch", "Parameter", "Variable", "LILConnectivity",
           "add_function", "functions"]
