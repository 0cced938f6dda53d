"""Splitting of the multi-line model strings into statements and flags.

Behaviour follows the reference's string handling
(ANNarchy/parser/StringManipulation.py:44-237): ';' and newlines separate
statements, '#' starts a comment, the text after the last ':' is a list of
flags only if it contains a known keyword, ``key = value`` flags are bounds
(init, min, max) and the others are plain flags (population, event-driven...).
"""
from __future__ import annotations

import re

FLAG_KEYWORDS = (
    "init", "min", "max", "population", "postsynaptic", "projection",
    "explicit", "implicit", "semiimplicit", "exponential", "midpoint", "rk4",
    "runge-kutta4", "exact", "event-driven", "unless_refractory", "int", "bool",
    "float", "unless_post",
)


class ParserError(ValueError):
    """Raised for model strings this parser cannot analyse."""


def statements(text: str) -> list[str]:
    """Split a multi-line definition into single statements without comments
    and with runs of white space collapsed (StringManipulation.py:66-81)."""
    out = []
    for line in text.replace(";", "\n").split("\n"):
        line = re.sub(r"\#[\s\S]+", " ", line)
        line = re.sub(r"\s+", " ", line)
        if line.strip():
            out.append(line)
    return out


def split_flags(definition: str) -> tuple[str, str | None]:
    """'eq : flags' -> (eq, flags) when the tail holds a keyword
    (StringManipulation.py:44-63)."""
    if ":" not in definition:
        return definition.strip(), None
    eq, tail = definition.rsplit(":", 1)
    if any(k in tail for k in FLAG_KEYWORDS):
        return eq.strip(), tail.strip()
    return definition.strip(), None


def parse_flags(tail: str | None) -> tuple[dict, list]:
    """'init=0.1, min=0.0, population' -> ({'init': '0.1', 'min': '0.0'},
    ['population']) (StringManipulation.py:125-150)."""
    bounds, flags = {}, []
    if not tail:
        return bounds, flags
    for item in re.findall(r"(?:[^,()]+|\([^()]*\))+", tail):
        item = item.strip()
        parts = item.split("=")
        if len(parts) == 2:
            bounds[parts[0].strip()] = parts[1].strip()
        else:
            flags.append(item)
    return bounds, flags


def lhs_name(equation: str, left: bool = False) -> str:
    """Name of the variable an equation defines: 'x' for 'x = ...', 'x += ...'
    and 'tau*dx/dt = ...' (StringManipulation.py:84-122)."""
    eq = equation.replace(" ", "")
    if not left:
        name = eq.split("=")[0]
        for op in ("+=", "-=", "*=", "/=", ">=", "<="):
            if op in eq:
                return eq.split(op)[0]
    else:
        name = eq.strip()
        for op in ("+", "-", "*", "/"):
            if eq.endswith(op):
                return eq.split(op)[0]
    if not name.strip():
        raise ParserError("no variable name in " + equation)
    if not any(op in name for op in "+-*/"):
        return name
    found = re.findall(r"d([\w]+)/dt", name)
    return found[0].strip() if len(found) == 1 else "_undefined"


def _is_flag_list(tail: str) -> bool:
    tail = "," + tail.replace(" ", "") + ","
    return any(re.match("([,]+)" + k + "([=,]+)", tail) for k in FLAG_KEYWORDS)


def equation_list(text) -> list[dict]:
    """Equations block -> [{'name', 'eq', 'constraint'}]; a line without an
    assignment continues the previous equation (StringManipulation.py:153-237)."""
    out: list[dict] = []
    if text is None:
        return out
    if isinstance(text, (list, tuple)):
        text = "\n".join("\n" + str(t) for t in text)
    for line in text.replace(";", "\n").split("\n"):
        d = line.strip()
        if not d:
            continue
        if "#" in d:
            d = d.split("#")[0]
            if not d.strip():
                continue
        if ":" in d:
            eq, tail = d.rsplit(":", 1)
            if _is_flag_list(tail):
                eq, tail = eq.strip(), tail.strip()
            else:
                eq, tail = d.strip(), ""
        else:
            eq, tail = d, ""
        ops = re.findall(r"([\s\w\+\-\*\/\)]+)=([^=])", eq)
        if len(ops) == 1:
            lhs = ops[0][0]
            if not lhs.strip():
                raise ParserError("cannot analyse " + eq)
            name = lhs_name(lhs, left=True)
            if name in ("_undefined", ""):
                raise ParserError("no variable name in " + eq)
            out.append({"name": name, "eq": eq.strip(), "constraint": tail.strip()})
        elif not ops:
            if not out:
                raise ParserError("cannot analyse " + eq)
            out[-1]["eq"] += " " + eq.strip()
            out[-1]["constraint"] += tail
        else:
            raise ParserError("only one assignment per equation: " + eq)
    return out
