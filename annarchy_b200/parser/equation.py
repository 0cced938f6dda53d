"""Translation of one model statement into a C expression string.

The translation goes through sympy exactly as the reference parser does
(ANNarchy/parser/Equation.py): statements are parsed with
``parse_expr(..., evaluate=False)`` against a symbol table whose symbols
carry index placeholders (``v%(local_index)s``, ``tau%(global_index)s``),
ODEs are solved for the derivative and simplified with ``ratio=1.0``, and
the result is printed by ``sympy.ccode(precision=8)``. Going through the
same sympy calls gives the same term order in every sum and product, which
is what makes a double-precision run of the generated kernels reproduce the
reference bit for bit.

Supported numerical methods: explicit Euler (Equation.py:276-307),
exponential Euler (Equation.py:559-604) and the closed-form event-driven
decay of synaptic traces (Equation.py:606-660).
"""
from __future__ import annotations

import contextvars
import re

import sympy as sp
from sympy.parsing.sympy_parser import convert_xor, parse_expr, standard_transformations

from .text import ParserError

# Built-in symbols (ANNarchy/parser/ParserTemplate.py:12-21)
BUILTIN_SYMBOLS = {
    "dt": sp.Symbol("dt"),
    "t": sp.Symbol("(double(t)*dt)"),
    "w": sp.Symbol("w%(local_index)s"),
    "g_target": sp.Symbol("sum"),
    "t_last": sp.Symbol("((double)(last_spike%(local_index)s)*dt)"),
    "t_pre": sp.Symbol("((double)(%(pre_prefix)slast_spike%(pre_index)s)*dt)"),
    "t_post": sp.Symbol("((double)(%(post_prefix)slast_spike%(post_index)s)*dt)"),
}

# Built-in functions (ParserTemplate.py:23-48)
BUILTIN_FUNCTIONS = {
    "pos": sp.Function("positive"),
    "positive": sp.Function("positive"),
    "neg": sp.Function("negative"),
    "negative": sp.Function("negative"),
    "modulo": sp.Function("modulo"),
    "fabs": sp.Function("fabs"),
    "ite": sp.Function("ite", nargs=3),
    "clip": sp.Function("clip"),
    "True": sp.Symbol("true"),
    "False": sp.Symbol("false"),
    "power": sp.Function("power", nargs=2),
    "round": sp.Function("round"),
}

C_FUNCTION_NAMES = {
    "pos": "positive", "positive": "positive", "neg": "negative", "negative": "negative",
    "modulo": "modulo", "fabs": "fabs", "clip": "clip", "ite": "ite", "power": "power",
    "isfinite": "isfinite", "isnan": "isnan",
}


# user functions visible to the statements being parsed: the global ones
# (add_function) and those of the model under analysis
GLOBAL_FUNCTIONS: dict = {}
_SCOPE_FUNCTIONS = contextvars.ContextVar("anb_scope_functions", default=())


def user_function_names() -> tuple:
    return tuple(GLOBAL_FUNCTIONS) + tuple(_SCOPE_FUNCTIONS.get())


def symbol_table(local, semiglobal, global_, untouched, functions=(), constants=()):
    """Symbols of a model's attributes with their index placeholders
    (ParserTemplate.py:51-105)."""
    table = dict(BUILTIN_SYMBOLS)
    table.update(BUILTIN_FUNCTIONS)
    for name in local:
        table[name] = sp.Symbol(name + "%(local_index)s")
    for name in semiglobal:
        table[name] = sp.Symbol(name + "%(semiglobal_index)s")
    for name in global_:
        table[name] = sp.Symbol(name + "%(global_index)s")
    for name in constants:
        table.setdefault(name, sp.Symbol(name))
    for name in untouched:
        table[name] = sp.Symbol(name)
    for name in functions:
        table[name] = sp.Function(name)
    return table


def logical_operators(expr: str) -> str:
    """Python logical words -> sympy operators (Equation.py:16-27)."""
    for a, b in ((" and ", " & "), (" or ", " | "), (" is not ", " != "), (" not ", " Not "),
                 (" not(", " Not("), (" is ", " == ")):
        expr = expr.replace(a, b)
    return expr


class Statement:
    """One statement of a model (an ODE, an assignment, an increment or a
    condition) and its C translation."""

    def __init__(self, name, expression, desc, untouched=(), method="explicit", kind=None,
                 functions=(), constants=()):
        self.name = name
        self.expression = logical_operators(expression)
        self.method = method
        self.desc = desc
        self.attributes = list(desc["attributes"])
        self.functions = dict(C_FUNCTION_NAMES)
        functions = tuple(functions) + user_function_names()
        for f in functions:
            self.functions[f] = f
        self.table = symbol_table(desc["local"], desc["semiglobal"], desc["global"],
                                  untouched, functions, constants)
        self.kind = kind or self._kind()
        self.analysed = None

    # -- classification (Equation.py:109-147) -------------------------------
    def _kind(self):
        e = self.expression.replace(" ", "")
        for op in ("+=", "-=", "*=", "/="):
            if op in e:
                return "inc"
        if "d" + self.name + "/dt" in e:
            return "ODE"
        parts = e.split("=")
        if len(parts) == 1:
            return "cond"
        if parts[1] == "":
            return "cond"
        if parts[0] and parts[0][-1] in "<>!":
            return "cond"
        return "simple"

    # -- helpers -------------------------------------------------------------
    def ccode(self, expr) -> str:
        """sympy -> C with 8 significant digits (Equation.py:153-197, double precision)."""
        try:
            return sp.ccode(expr, precision=8, strict=False, user_functions=self.functions)
        except TypeError:
            return sp.ccode(expr, precision=8, user_functions=self.functions)

    def parse_expr(self, text):
        try:
            return parse_expr(text, local_dict=self.table,
                              transformations=(standard_transformations + (convert_xor,)),
                              evaluate=False)
        except Exception as exc:  # sympy raises many exception types
            raise ParserError("cannot analyse the expression: " + str(text)) from exc

    def dependencies(self):
        if self.analysed is None:
            return []
        atoms = self.analysed.atoms()
        return [a for a in self.attributes if a in self.table and self.table[a] in atoms]

    # -- entry point ---------------------------------------------------------
    def parse(self):
        if self.kind == "ODE":
            return self._ode(self.expression)
        if self.kind == "cond":
            return self._condition(self.expression)
        if self.kind == "inc":
            return self._increment(self.expression)
        if self.kind == "return":
            self.analysed = self.parse_expr(self.expression)
            return self.ccode(self.analysed) + ";"
        return self._assignment(self.expression)

    # -- ODEs (Equation.py:254-275) -------------------------------------------
    def _ode(self, expression):
        if "=" in expression:
            expression = expression.replace("=", "- (") + ")"
        expression = expression.replace(" ", "")
        if self.method == "explicit":
            return self._explicit(expression)
        if self.method == "exponential":
            return self._exponential(expression)
        if self.method == "event-driven":
            return self._event_driven(expression)
        raise ParserError(f"numerical method {self.method!r} is not supported by this backend")

    def _explicit(self, expression):
        expression = expression.replace("d" + self.name + "/dt", "_grad_var_")
        grad = sp.Symbol("_grad_var_")
        self.table["_grad_var_"] = grad
        self.analysed = self.parse_expr(expression)
        rhs = sp.solve(self.analysed, grad, check=False, rational=False)[0]
        rhs = sp.simplify(rhs, ratio=1.0)
        code = "double _" + self.name + " = " + self.ccode(rhs) + ";"
        switch = self.ccode(self.table[self.name]) + " += dt*_" + self.name + " ;"
        return [{}, code, switch]

    def _standard_form(self, expression):
        """tau*dx/dt + x = S  ->  (tau, dt/tau, S) (Equation.py:662-742)."""
        expression = expression.replace("d" + self.name + "/dt", "_gradvar_")
        grad = sp.Symbol("_gradvar_")
        self.table["_gradvar_"] = grad
        analysed = self.parse_expr(expression)
        self.analysed = analysed
        var = self.table[self.name]
        expanded = analysed.expand(modulus=None, power_base=False, power_exp=False, mul=True,
                                   log=False, multinomial=False)
        coll = sp.collect(expanded, var, evaluate=False, exact=False)
        if var not in coll or len(coll) > 2:
            coll = sp.collect(sp.simplify(expanded), var, evaluate=False, exact=False)
            if var not in coll or len(coll) > 2:
                return None, None, None
        factor_var = coll[var]
        coll_grad = sp.collect(sp.expand(analysed, grad), grad, evaluate=False, exact=False)
        factor_grad = coll_grad[grad] if grad in coll_grad else sp.S(1.0)
        tau = factor_grad / factor_var
        normalized = analysed / factor_var
        steady = sp.simplify(sp.together(tau * grad + var - normalized))
        step = sp.simplify(sp.together(self.table["dt"] / tau))
        return tau, step, steady

    def _exponential(self, expression):
        tau, step, steady = self._standard_form(expression)
        if tau is None:
            return self._explicit(expression)
        local_step = any(self.table[a] in step.atoms() for a in self.attributes
                         if a in self.desc["local"])
        pre_loop = {}
        step_code = "(1.0 - exp(" + self.ccode(-step) + "))"
        if not local_step:
            pre_loop = {"name": "__stepsize_" + self.name,
                        "value": "1.0 - exp( " + self.ccode(-step) + ")"}
            step_code = "__stepsize_" + self.name
        var = self.ccode(self.table[self.name])
        code = ("double _" + self.name + " =  " + step_code + "*(" + self.ccode(steady) + " - "
                + var + ");")
        return [pre_loop, code, var + " += _" + self.name + " ;"]

    def _event_driven(self, expression):
        tau, _, steady = self._standard_form(expression)
        if tau is None:
            raise ParserError("event-driven equations must be linear first-order ODEs: "
                              + self.expression)
        var = self.ccode(self.table[self.name])
        s = self.ccode(steady)
        if s == "0":
            return (var + " *= exp(dt*(_last_event%(local_index)s - (t))/("
                    + self.ccode(tau) + "));")
        return (var + " = " + s + " + (" + var + " - " + s
                + ")*exp(dt*(_last_event%(local_index)s - (t))/(" + self.ccode(tau) + "));")

    # -- other statements (Equation.py:744-880) --------------------------------
    def _condition(self, expression):
        expression = expression.strip()
        if "==" in expression:
            if "&" in expression or "|" in expression:
                expression = re.sub(r"([\w\s.]+)==([\w\s.]+)", r"Equality(\1, \2)", expression)
            else:
                if expression[0] == "(" and expression[-1] == ")":
                    expression = expression[1:-1]
                a, b = expression.split("==")
                expression = "Equality(" + a + ", " + b + ")"
        if "!=" in expression:
            if "&" in expression or "|" in expression:
                expression = re.sub(r"([\w\s.]+)!=([\w\s.]+)", r"Not(Equality(\1, \2))",
                                    expression)
            else:
                if expression[0] == "(" and expression[-1] == ")":
                    expression = expression[1:-1]
                a, b = expression.split("!=")
                expression = "Not(Equality(" + a + ", " + b + "))"
        self.analysed = self.parse_expr(expression)
        return self.ccode(self.analysed)

    def _increment(self, expression):
        for op in ("+=", "-=", "*=", "/="):
            if op in expression:
                pos = expression.find(op)
                name = expression[:pos].strip()
                expression = expression[pos + 2:]
                break
        self.analysed = self.parse_expr(expression)
        return (self.ccode(self.table[name]) + " " + op + " "
                + self.ccode(sp.simplify(self.analysed, ratio=1.0)) + ";")

    def _assignment(self, expression):
        pos = expression.find("=")
        name = expression[:pos].strip()
        self.analysed = self.parse_expr(expression[pos + 1:])
        return self.ccode(self.table[name]) + " = " + self.ccode(self.analysed) + ";"
