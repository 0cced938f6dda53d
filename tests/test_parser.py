"""The parser restatement against the reference parser's output for a
catalogue of models (tests/golden/parser_strings.json)."""
import json
import os
import sys

import pytest

from annarchy_b200.core.models import Neuron, Synapse
from annarchy_b200.parser.analysis import analyse_neuron, analyse_synapse
from annarchy_b200.parser.text import ParserError

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from models_catalog import NEURONS, SYNAPSES  # noqa: E402

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "parser_strings.json")))


def _cmp_vars(d, g):
    assert len(d["variables"]) == len(g["variables"])
    for v, gv in zip(d["variables"], g["variables"]):
        for f in ("name", "cpp", "switch", "bounds", "init", "locality", "method"):
            assert v.get(f) == gv.get(f), (v["name"], f)


@pytest.mark.parametrize("key", sorted(NEURONS))
def test_neuron_strings(key):
    d = analyse_neuron(Neuron(**NEURONS[key]))
    g = GOLD["neurons"][key]
    _cmp_vars(d, g)
    assert d["local"] == g["local"] and d["global"] == g["global"]
    assert d["targets"] == g["targets"]
    if "spike_cond" in g:
        assert d["spike"]["spike_cond"] == g["spike_cond"]
        assert [r["cpp"] for r in d["spike"]["spike_reset"]] == g["spike_reset"]
    for p, gp in zip(d["parameters"], g["parameters"]):
        assert (p["name"], p["init"], p["locality"]) == (gp["name"], gp["init"], gp["locality"])


@pytest.mark.parametrize("key", sorted(SYNAPSES))
def test_synapse_strings(key):
    d = analyse_synapse(Synapse(**SYNAPSES[key]))
    g = GOLD["synapses"][key]
    _cmp_vars(d, g)
    for f in ("pre_spike", "post_spike"):
        if f in g:
            assert [v["cpp"] for v in d[f]] == g[f]


def test_rate_neuron_needs_r():
    with pytest.raises(ParserError):
        analyse_neuron(Neuron(parameters="tau = 10.0", equations="tau * dv/dt = -v"))


def test_conditional_statement_errors():
    """Malformed conditionals are refused as the reference refuses them
    (ANNarchy/parser/ITE.py:150-170)."""
    with pytest.raises(ParserError):
        analyse_neuron(Neuron(equations="r = 1.0 + if t > 1: 1.0 else: 0.0"))
    with pytest.raises(ParserError):
        analyse_neuron(Neuron(equations="r = if t > 1: 1.0"))


def test_unsupported_constructs_rejected():
    # a reduction of something that is not a local attribute
    with pytest.raises(ParserError):
        analyse_neuron(Neuron(equations="r = mean(w)\n dv/dt = -v"))
    # coupled implicit systems
    with pytest.raises(ParserError):
        analyse_neuron(Neuron(equations="""
            dv/dt = -v + u : implicit
            du/dt = -u + v : implicit
        """))
