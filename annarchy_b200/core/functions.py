"""User functions of models evaluated on the host: the callables that
`Population.<function>(...)`, `Projection.<function>(...)` and
`functions(name)` return (the reference compiles them into its wrapper
module). The body is parsed by sympy into one expression per branch, and
branches are chosen elementwise with numpy.where; the device code uses the
C expressions of the same parse."""
from __future__ import annotations

import numpy as np
import sympy as sp
from sympy.parsing.sympy_parser import convert_xor, parse_expr, standard_transformations

from ..parser.equation import logical_operators

# the parser's C names of the built-in functions, as numpy functions
_NUMPY = {
    "positive": lambda x: np.maximum(x, 0.0), "pos": lambda x: np.maximum(x, 0.0),
    "negative": lambda x: np.minimum(x, 0.0), "neg": lambda x: np.minimum(x, 0.0),
    "clip": lambda x, a, b: np.where(x < a, a, np.where(x > b, b, x)),
    "modulo": lambda a, b: np.fmod(np.trunc(a), np.trunc(b)),
    "power": lambda x, a: np.power(x, np.trunc(a)),
    "fabs": np.abs, "ite": lambda c, a, b: np.where(c, a, b),
}


def _lambdify(args, text, table):
    expr = parse_expr(logical_operators(" " + text + " "), local_dict=table,
                      transformations=(standard_transformations + (convert_xor,)))
    return sp.lambdify([table[a] for a in args], expr, modules=[_NUMPY, "numpy"])


def evaluator(fdesc: dict, others: dict | None = None):
    """Host callable of a parsed user function (analyse_functions)."""
    args = fdesc["args"]
    table = {a: sp.Symbol(a) for a in args}
    for name, f in (others or {}).items():
        table[name] = sp.Function(name)
        _NUMPY.setdefault(name, evaluator(f))
    for name in ("pos", "positive", "neg", "negative", "clip", "modulo", "power", "ite"):
        table.setdefault(name, sp.Function(name))

    def branch(b):
        if isinstance(b, list):
            cond, then, other = _lambdify(args, b[0], table), branch(b[1]), branch(b[2])
            return lambda *v: np.where(cond(*v), then(*v), other(*v))
        return _lambdify(args, b, table)

    if fdesc["conditions"]:
        body = branch(fdesc["conditions"][0])
    else:
        body = _lambdify(args, fdesc["eq"], table)

    def call(*values):
        vals = [np.asarray(v, dtype=np.float64) for v in values]
        if len(vals) != len(args):
            raise TypeError(f"{fdesc['name']}() takes {len(args)} arguments")
        return np.asarray(body(*vals), dtype=np.float64) * np.ones(np.broadcast(*vals).shape)

    call.__name__ = fdesc["name"]
    return call
