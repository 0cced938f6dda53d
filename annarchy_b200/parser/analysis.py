"""Neuron and synapse analysis: model definition -> description dict.

The description has the same keys as the reference's
(ANNarchy/parser/AnalyseNeuron.py:27-392, AnalyseSynapse.py:34-590):
``parameters``, ``variables`` (each with ``cpp``, ``switch``, ``bounds``,
``init``, ``locality``, ``method``), ``local``/``semiglobal``/``global``,
``targets``, ``spike`` (``spike_cond``, ``spike_reset``) and, for synapses,
``pre_spike``/``post_spike``/``psp``. C strings keep the reference's index
placeholders (``%(local_index)s`` ...); the code generator fills them.

Random distributions inside neuron and synapse equations
(``p = Uniform(0.0, 1.0)``) become per-step draws ``rand_<k>`` listed in
``random_distributions``, as the reference's parser extracts them
(ANNarchy/parser/Extraction.py, extract_randomdist); the code generator draws
them on the device. If-then-else statements (``x = if c: a else: b``, nested)
become C conditionals as in ANNarchy/parser/ITE.py; ``ite(c, a, b)`` is a
function of the device header.

Not supported by this backend (an error names them): global operations
(``mean(pre.r)`` in synapses), coupled implicit/midpoint/rk4 systems.
"""
from __future__ import annotations

import re

from . import equation as _eq
from .equation import BUILTIN_FUNCTIONS, Statement
from .text import ParserError, equation_list, lhs_name, parse_flags, split_flags, statements


# ---------------------------------------------------------------------------
# parameters and variables (Extraction.py:251-536)
# ---------------------------------------------------------------------------

def _flags_to_locality(flags):
    for f in ("population", "postsynaptic", "projection"):
        if f in flags:
            return "semiglobal" if f == "postsynaptic" else "global"
    return "local"


def _typed_init(bounds, flags, equation=""):
    ctype = "int" if "int" in flags else ("bool" if "bool" in flags else "double")
    if "init" in bounds:
        init = bounds["init"]
        if ctype == "bool":
            init = init in ("true", "True", "1")
        else:
            try:
                init = int(init) if ctype == "int" else float(init)
            except ValueError:
                init = str(init)
    elif "=" in equation:
        init = equation.split("=")[1].strip()
        if init in ("false", "False", "true", "True"):
            ctype, init = "bool", init in ("true", "True")
        elif ctype == "int":
            init = int(eval(init, {}, {}))  # numeric literal, possibly an expression like 2*3
        else:
            try:
                init = float(eval(init, {}, {}))
            except Exception as exc:
                raise ParserError("the value of the parameter is not a float: " + equation) from exc
    else:
        init = False if ctype == "bool" else (0 if ctype == "int" else 0.0)
    return ctype, init


def extract_parameters(parameters, object_type):
    out = []
    if parameters is None:
        return out
    if isinstance(parameters, dict):
        for key, val in parameters.items():
            locality, ctype, value = "global", "double", val
            if hasattr(val, "locality") and hasattr(val, "value"):   # Parameter(...) objects
                locality = {"population": "global", "projection": "global",
                            "postsynaptic": "semiglobal"}.get(val.locality, val.locality)
                value = val.value
                ctype = {float: "double", int: "int", bool: "bool", "float": "double"}.get(
                    getattr(val, "type", float), str(getattr(val, "type", "double")))
            if locality == "global":
                flags = "population" if object_type == "neuron" else "projection"
            elif locality == "semiglobal":
                flags = "postsynaptic"
            else:
                flags = ""
            out.append(dict(name=key, locality=locality, eq=f"{key} = {value}", bounds={},
                            flags=flags, ctype=ctype, init=value))
        return out
    lines = statements(parameters) if isinstance(parameters, str) else list(parameters)
    for definition in lines:
        equation, tail = split_flags(definition)
        name = lhs_name(equation)
        if name in ("_undefined", ""):
            raise ParserError("definition can not be analysed: " + equation)
        bounds, flags = parse_flags(tail)
        ctype, init = _typed_init(bounds, flags, equation)
        out.append(dict(name=name, locality=_flags_to_locality(flags), eq=equation,
                        bounds=bounds, flags=flags, ctype=ctype, init=init))
    return out


def extract_variables(equations):
    out = []
    for d in equation_list(equations):
        eq = d["eq"]
        if eq.count("(") != eq.count(")"):
            raise ParserError("the number of parentheses does not match: " + eq)
        bounds, flags = parse_flags(d["constraint"])
        ctype, init = _typed_init(bounds, flags)
        out.append(dict(name=d["name"], locality=_flags_to_locality(flags), eq=eq, bounds=bounds,
                        flags=flags, ctype=ctype, init=init))
    return out


def _method(var, default="explicit"):
    for f, m in (("implicit", "implicit"), ("semiimplicit", "semiimplicit"),
                 ("exponential", "exponential"), ("midpoint", "midpoint"),
                 ("runge-kutta4", "rk4"), ("rk4", "rk4"), ("explicit", "explicit"),
                 ("exact", "event-driven"), ("event-driven", "event-driven")):
        if f in var["flags"]:
            return m
    return default


def _split_locality(items, neuron):
    attributes, local, global_, semiglobal = [], [], [], []
    for p in items:
        attributes.append(p["name"])
        flags = p["flags"]
        if "population" in flags:
            if not neuron:
                raise ParserError(f"{p['name']}: 'population' is a neuron flag")
            global_.append(p["name"])
        elif "projection" in flags:
            if neuron:
                raise ParserError(f"{p['name']}: 'projection' is a synapse flag")
            global_.append(p["name"])
        elif "postsynaptic" in flags:
            if neuron:
                raise ParserError(f"{p['name']}: 'postsynaptic' is a synapse flag")
            semiglobal.append(p["name"])
        else:
            local.append(p["name"])
    return attributes, local, global_, semiglobal


def _targets(variables):
    found = []
    for var in variables:
        for _, t in re.findall(r"(?P<pre>[^\w.])sum\(\s*([^()]+)\s*\)", var["eq"]):
            found.append(t.strip())
        if re.findall(r"([^\w.])sum\(\)", var["eq"]):
            found.append("__all__")
        for _, t in re.findall(r"([^\w.])g_([\w]+)", var["eq"]):
            found.append(t.strip())
    return sorted(set(found))


RANDOM_DISTRIBUTIONS = {"Uniform": 2, "Normal": 2, "LogNormal": 2, "Exponential": 1,
                        "DiscreteUniform": 2}
_RANDOM_RE = re.compile(r"\b(Uniform|Normal|LogNormal|Exponential|DiscreteUniform|Gamma|Binomial)"
                        r"\(([^()]*)\)")


def _extract_random(eq, var, found, untouched):
    """Replace every random distribution of `eq` by a placeholder of a
    per-step draw rand_<k> (one draw per neuron, or per population for a
    global variable) recorded in `found`."""
    def repl(m):
        dist, args = m.group(1), [a.strip() for a in m.group(2).split(",") if a.strip()]
        if dist not in RANDOM_DISTRIBUTIONS:
            raise ParserError(f"{var['name']}: the {dist} distribution is not supported in equations "
                              "by this backend")
        if len(args) != RANDOM_DISTRIBUTIONS[dist]:
            raise ParserError(f"{var['name']}: {dist} takes {RANDOM_DISTRIBUTIONS[dist]} arguments")
        k = len(found)
        found.append({"name": f"rand_{k}", "dist": dist, "args": args,
                      "locality": var.get("locality", "local")})
        untouched[f"__rand_{k}__"] = f"rand_{k}"
        return f" __rand_{k}__ "
    return _RANDOM_RE.sub(repl, eq)


GLOBAL_OPERATIONS = ("min", "max", "mean", "norm1", "norm2")


def _extract_globalops(eq, desc, where):
    """Population-wide reductions of a neuron's local variable in an
    equation (``mean(r)``, ``max(v)``...; ANNarchy/parser/Extraction.py:
    124-145): replaced by the scalar ``_<op>_<var>``, computed after every
    step's update and listed in desc["global_operations"]."""
    untouched = {}
    for op in GLOBAL_OPERATIONS:
        for _, var in re.findall(r"([^\w]*)" + op + r"\(([\s\w]*)\)", eq):
            if var.strip() not in desc["local"]:
                raise ParserError(f"{where}: there is no local attribute {var!r}")
            new = "_" + op + "_" + var.strip()
            eq = eq.replace(op + "(" + var + ")", new)
            untouched[new] = new
            item = {"function": op, "variable": var.strip()}
            if item not in desc["global_operations"]:
                desc["global_operations"].append(item)
    return eq, untouched


def _extract_globalops_synapse(eq, desc, where):
    """Reductions of the pre- or post-synaptic population in a synaptic
    equation (``mean(pre.r)``, ``max(post.v)``; ANNarchy/parser/
    Extraction.py:148-190): replaced by that population's scalar
    `%(pre_prefix)s_<op>_<var>` and listed in desc["pre_global_operations"] /
    desc["post_global_operations"]."""
    untouched = {}
    for op in GLOBAL_OPERATIONS:
        for side in ("pre", "post"):
            for var in re.findall(r"(?<![\w.])" + op + r"\(\s*" + side + r"\.([\w]+)\s*\)", eq):
                new = "__" + side + "_" + op + "_" + var
                eq = re.sub(op + r"\(\s*" + side + r"\." + var + r"\s*\)", new, eq)
                untouched[new] = "%(" + side + "_prefix)s_" + op + "_" + var
                item = {"function": op, "variable": var}
                lst = desc.setdefault(side + "_global_operations", [])
                if item not in lst:
                    lst.append(item)
    return eq, untouched


def _unsupported(eq, where, neuron=False):
    if not neuron and re.search(r"\b(mean|min|max|norm1|norm2)\(", eq):
        raise ParserError(f"{where}: global operations in synapses are not supported by this "
                          "backend")
    if re.search(r"\b(Uniform|Normal|LogNormal|Exponential|Gamma|Binomial|DiscreteUniform)\(", eq):
        raise ParserError(f"{where}: random distributions in equations are not supported by "
                          "this backend")


def _extract_ite(eq, split=True):
    """An if-then-else right-hand side (ANNarchy/parser/ITE.py:93-175):

        x = if cond: a else: b          (branches may nest)

    becomes `x = __conditional__0` and the nested [condition, then, else]
    structure; (eq, []) when the statement has no conditional."""
    if "if " not in eq:
        return eq, []
    left, right = eq.split("=", 1) if split else ("", eq)
    n_then, n_else = right.count(":"), len(re.findall("else", right))
    if n_then == 0:
        raise ParserError(f"{eq}: conditional statements must define then and else values "
                          "(var = if condition: a else: b)")
    if not right.strip().startswith("if"):
        raise ParserError(f"{eq}: the right term must directly start with an if statement")
    if n_then != 2 * n_else:
        raise ParserError(f"{eq}: conditional statements must use both : and else")
    lines = []
    for item in (x.strip() for x in right.split(":")):
        if item.startswith("if "):
            lines.append(item)
        elif item.endswith("else"):
            lines.append(item.split("else")[0].strip())
            lines.append("else")
        else:
            lines.append(item)

    def nest(rest):
        out = []
        while rest:
            if rest[0].startswith("if"):
                block = [rest.pop(0).split("if")[1], nest(rest)]
                if rest and rest[0].startswith("else"):
                    rest.pop(0)
                    block.append(nest(rest))
                out.append(block)
            elif not rest[0].startswith("else"):
                out.append(rest.pop(0))
            else:
                break
        return out[0]

    condition = nest(lines)
    right = " __conditional__0 "
    return (left + "=" + right if split else right), [condition]


def _ite_statement(name, eq, conditions, desc, untouched, method="explicit", kind=None):
    """The C code of a statement with conditionals (ANNarchy/parser/ITE.py:
    13-90): the statement with its placeholders, each replaced by
    (cond ? then : else), conditions parsed as conditions and branches as
    expressions, nested branches recursively. Returns (code, Statement)."""
    keys = list(untouched)

    def branch(b):
        if isinstance(b, list):
            return conditional(b)
        return Statement(name, b, desc, untouched=keys, kind="return").parse().split(";")[0]

    def conditional(c):
        cond = Statement(name, c[0], desc, untouched=keys, kind="cond").parse()
        return "(" + cond + " ? " + branch(c[1]) + " : " + branch(c[2]) + ")"

    st = Statement(name, eq, desc, untouched=keys + [f"__conditional__{i}" for i in
                                                   range(len(conditions))],
                   method=method, kind=kind)
    code = st.parse()
    for i, c in enumerate(conditions):
        ite = conditional(c)
        if isinstance(code, str):
            code = code.replace(f"__conditional__{i}", ite)
        else:
            code = list(code)
            code[1] = code[1].replace(f"__conditional__{i}", ite)
    return code, st


def _bound_code(name, value, desc, untouched):
    if isinstance(value, str):
        try:
            float(value)
        except ValueError:
            st = Statement(name, value, desc, untouched=untouched, kind="return")
            return st.parse().replace(";", "")
    return value


# ---------------------------------------------------------------------------
# neurons
# ---------------------------------------------------------------------------

def analyse_functions(text) -> list:
    """User functions ``name(a, b) = expression`` (one per line, branches
    with if/else allowed; ANNarchy/parser/Function.py and the reference's
    add_function): the arguments are plain symbols, the body a C
    expression; the description keeps what a host evaluator needs."""
    out = []
    if not text:
        return out
    empty = {"attributes": [], "local": [], "semiglobal": [], "global": []}
    for line in (x.strip() for x in str(text).split("\n")):
        if not line or line.startswith("#"):
            continue
        m = re.match(r"^(\w+)\s*\(([^()]*)\)\s*=(.*)$", line)
        if not m:
            raise ParserError("a function must be defined as name(arguments) = expression: " + line)
        name, rhs = m.group(1), m.group(3).strip()
        args = [a.strip() for a in m.group(2).split(",") if a.strip()]
        eq, conditions = _extract_ite(rhs, split=False)
        code, _ = _ite_statement(name, eq, conditions, empty, {a: a for a in args},
                                 kind="return")
        out.append({"name": name, "args": args, "cpp": code.strip().rstrip(";").strip(),
                    "eq": eq, "conditions": conditions})
    return out


def _with_functions(analyse):
    """Run a model's analysis with its own functions visible to the
    parser; the description lists them under "functions"."""
    def run(model):
        funcs = analyse_functions(getattr(model, "functions", None))
        token = _eq._SCOPE_FUNCTIONS.set(tuple(f["name"] for f in funcs))
        try:
            desc = analyse(model)
        finally:
            _eq._SCOPE_FUNCTIONS.reset(token)
        desc["functions"] = funcs
        return desc
    run.__doc__ = analyse.__doc__
    return run


@_with_functions
def analyse_neuron(neuron) -> dict:
    """Description dict of a neuron type (AnalyseNeuron.py:27-392)."""
    desc = {"object": "neuron", "type": neuron.type, "raw_parameters": neuron.parameters,
            "raw_equations": neuron.equations}
    if neuron.type == "spike":
        desc["raw_reset"] = neuron.reset
        desc["raw_spike"] = neuron.spike
        desc["refractory"] = neuron.refractory
    params = extract_parameters(neuron.parameters, "neuron")
    variables = extract_variables(neuron.equations)
    desc["parameters"], desc["variables"] = params, variables
    names = [v["name"] for v in params + variables]
    if neuron.type == "rate":
        if "r" not in names:
            raise ParserError('rate-coded neurons must define the variable "r"')
    else:
        if "r" in names:
            raise ParserError('spiking neurons use "r" for the mean firing rate; use another name')
        variables.append(dict(name="r", locality="local", bounds={}, ctype="double", init=0.0,
                              flags=[], eq="", cpp=""))
    attributes, local, global_, _ = _split_locality(params + variables, neuron=True)
    if len(attributes) != len(set(attributes)):
        raise ParserError("attributes must be declared only once: " + str(attributes))
    desc.update(attributes=attributes, local=local, semiglobal=[], global_=None)
    desc["global"] = global_
    del desc["global_"]
    targets = _targets(variables)
    desc["targets"] = targets
    if neuron.type == "spike":
        for t in targets:
            if not any(v["name"] == "g_" + t for v in variables):
                variables.append(dict(name="g_" + t, locality="local", bounds={}, ctype="double",
                                      init=0.0, flags=[], eq="g_" + t + " = 0.0"))
                desc["attributes"].append("g_" + t)
                desc["local"].append("g_" + t)
        desc["spike"] = _spike(desc)
    randoms = []
    desc["random_distributions"] = randoms
    desc["global_operations"] = []
    for var in variables:
        eq = var.get("transformed_eq", var["eq"])
        if eq.strip() == "":
            continue
        untouched = {}
        eq = _extract_random(eq, var, randoms, untouched)
        eq, glob_untouched = _extract_globalops(eq, desc, var["name"])
        untouched.update(glob_untouched)
        _unsupported(eq, var["name"], neuron=True)
        for t in targets:
            eq = re.sub(r"(?P<pre>[^\w.])sum\(\)", r"\1sum(__all__)", eq)
            eq = re.sub(r"sum\(\s*" + t + r"\s*\)", "__sum_" + t + "__", eq)
            untouched["__sum_" + t + "__"] = "_sum_" + t + "%(local_index)s"
        method = _method(var)
        for b in ("min", "max"):
            if b in var["bounds"]:
                var["bounds"][b] = _bound_code(var["name"], var["bounds"][b], desc, untouched)
        eq, conditions = _extract_ite(eq)
        code, st = _ite_statement(var["name"], eq, conditions, desc, untouched, method)
        if isinstance(code, str):
            pre_loop, cpp, switch = {}, code, None
        else:
            pre_loop, cpp, switch = code
        for prev, new in sorted(untouched.items(), key=lambda kv: len(kv[0]), reverse=True):
            cpp = re.sub(prev, new, cpp)
            if pre_loop:
                pre_loop["value"] = re.sub(prev, new, pre_loop["value"])
            if switch:
                switch = re.sub(prev, new, switch)
        var.update(pre_loop=pre_loop, cpp=cpp, switch=switch, transformed_eq=eq,
                   untouched=untouched, method=method, dependencies=sorted(set(st.dependencies())))
        if method in ("implicit", "semiimplicit", "midpoint", "rk4") and switch is not None:
            raise ParserError(f"{var['name']}: method {method!r} is not supported by this backend")
    return desc


def _spike(desc):
    cond = statements(desc["raw_spike"])
    if len(cond) != 1:
        raise ParserError("the spike condition must be a single expression")
    st = Statement("raw_spike_cond", cond[0].strip(), desc)
    spike_cond = st.parse()
    resets = []
    raw = desc.get("raw_reset")
    if raw:
        for var in equation_list(raw):
            rs = Statement(var["name"], var["eq"], desc)
            var["cpp"] = rs.parse()
            var["dependencies"] = rs.dependencies()
            resets.append(var)
    return {"spike_cond": spike_cond, "spike_cond_dependencies": st.dependencies(),
            "spike_reset": resets}


# ---------------------------------------------------------------------------
# synapses
# ---------------------------------------------------------------------------

def _prepost(eq):
    """pre.x / post.x -> placeholders (Extraction.py:189-248)."""
    untouched = {}
    for var in sorted(set(re.findall(r"pre\.([\w]+)", eq))):
        if var == "sum":
            def rep(m):
                t = m.group(1).strip()
                untouched["_pre_sum_" + t] = "%(pre_prefix)s_sum_" + t + "%(pre_index)s"
                return "_pre_sum_" + t
            eq = re.sub(r"pre\.sum\(([\s\w]+)\)", rep, eq)
        else:
            eq = re.sub(r"pre." + var + r"([^_\w]+)", "_pre_" + var + r"__\g<1>", eq + " ")
            untouched["_pre_" + var + "__"] = "%(pre_prefix)s" + var + "%(pre_index)s"
    for var in sorted(set(re.findall(r"post\.([\w]+)", eq))):
        if var == "sum":
            def rep(m):
                t = m.group(1).strip()
                untouched["_post_sum_" + t] = "%(post_prefix)s_sum_" + t + "%(post_index)s"
                return "_post_sum_" + t
            eq = re.sub(r"post\.sum\(([\s\w]+)\)", rep, eq)
        else:
            eq = re.sub(r"post." + var + r"([^_\w]+)", "_post_" + var + r"__\g<1>", eq + " ")
            untouched["_post_" + var + "__"] = "%(post_prefix)s" + var + "%(post_index)s"
    return eq, untouched


def _event_statements(raw):
    out = []
    if not raw:
        return out
    for var in equation_list(raw):
        bounds, flags = parse_flags(var["constraint"])
        ctype, init = _typed_init(bounds, flags)
        out.append(dict(name=var["name"], eq=var["eq"], locality="local", bounds=bounds,
                        flags=flags, ctype=ctype, init=init))
    return out


@_with_functions
def analyse_synapse(synapse) -> dict:
    """Description dict of a synapse type (AnalyseSynapse.py:34-590)."""
    desc = {"object": "synapse", "type": synapse.type, "raw_parameters": synapse.parameters,
            "raw_equations": synapse.equations}
    if synapse.psp:
        desc["raw_psp"] = synapse.psp
    elif synapse.type == "rate":
        desc["raw_psp"] = "w*pre.r"
    params = extract_parameters(synapse.parameters, "synapse")
    variables = extract_variables(synapse.equations)
    if not any(v["name"] == "w" for v in params + variables):
        params.append(dict(name="w", bounds={}, ctype="double", init=0.0, flags=[], eq="w=0.0",
                           locality="local"))
    desc["plasticity"] = any(v["name"] == "w" for v in variables)
    attributes, local, global_, semiglobal = _split_locality(params + variables, neuron=False)
    if len(attributes) != len(set(attributes)):
        raise ParserError("attributes must be declared only once: " + str(attributes))
    desc.update(parameters=params, variables=variables, attributes=attributes, local=local,
                semiglobal=semiglobal)
    desc["global"] = global_
    if synapse.type == "spike":
        desc["pre_spike"] = _event_statements(synapse.pre_spike)
        desc["post_spike"] = _event_statements(synapse.post_spike)
        for group, skip in (("pre_spike", ("g_target",)), ("post_spike", ("g_target", "w"))):
            for var in desc[group]:
                if var["name"] in skip or any(v["name"] == var["name"] for v in variables):
                    continue
                variables.append(dict(name=var["name"], bounds=var["bounds"], ctype=var["ctype"],
                                      init=var["init"], locality=var["locality"], flags=[],
                                      transformed_eq="", eq="", cpp="", switch="",
                                      untouched="", method="explicit"))
                desc["local"].append(var["name"])
                desc["attributes"].append(var["name"])
    untouched_all = {}
    randoms = []
    desc["random_distributions"] = randoms
    for var in variables:
        eq = var.get("transformed_eq", var["eq"])
        if eq.strip() == "":
            continue
        # per-step draws (one per synapse, dendrite or projection by the
        # variable's locality)
        rand_untouched = {}
        eq = _extract_random(" " + eq + " ", var, randoms, rand_untouched)
        untouched_all.update(rand_untouched)
        eq, glob_untouched = _extract_globalops_synapse(eq, desc, var["name"])
        untouched_all.update(glob_untouched)
        _unsupported(eq, var["name"])
        eq, untouched = _prepost(eq)
        for k, v in untouched.items():
            untouched_all.setdefault(k, v)
        method = _method(var)
        for b in ("min", "max"):
            if b in var["bounds"]:
                var["bounds"][b] = _bound_code(var["name"], var["bounds"][b], desc,
                                               list(untouched_all))
        eq, conditions = _extract_ite(eq)
        code, st = _ite_statement(var["name"], eq, conditions, desc, untouched_all, method)
        if isinstance(code, str):
            pre_loop, cpp, switch = {}, code, None
        else:
            pre_loop, cpp, switch = code
        for prev, new in sorted(untouched_all.items(), key=lambda kv: len(kv[0]), reverse=True):
            cpp = cpp.replace(prev, new)
        var.update(pre_loop=pre_loop, cpp=cpp, switch=switch, transformed_eq=eq,
                   untouched=dict(untouched_all), method=method,
                   dependencies=st.dependencies())
        if method in ("implicit", "semiimplicit", "midpoint", "rk4") and switch is not None:
            raise ParserError(f"{var['name']}: method {method!r} is not supported by this backend")
    if "raw_psp" in desc:
        eq, glob_untouched = _extract_globalops_synapse(" " + desc["raw_psp"].strip() + " ", desc,
                                                        "psp")
        untouched_all.update(glob_untouched)
        eq, untouched = _prepost(eq)
        for k, v in untouched.items():
            untouched_all.setdefault(k, v)
        eq, conditions = _extract_ite(eq, split=False)
        code, st = _ite_statement("psp", eq, conditions, desc, untouched_all, kind="return")
        for prev, new in sorted(untouched_all.items(), key=lambda kv: len(kv[0]), reverse=True):
            code = code.replace(prev, new)
        desc["psp"] = {"eq": desc["raw_psp"].strip(), "cpp": code}
    if synapse.type == "spike":
        for var in desc["pre_spike"] + desc["post_spike"]:
            if var["name"] == "w":
                desc["plasticity"] = True
            _unsupported(var["eq"], var["name"])
            eq, untouched = _prepost(var["eq"])
            st = Statement(var["name"], eq, desc, untouched=untouched, method="explicit")
            code = st.parse()
            if isinstance(code, list):
                raise ParserError("ODEs are not allowed in pre_spike/post_spike: " + var["eq"])
            for prev, new in sorted(untouched.items(), key=lambda kv: len(kv[0]), reverse=True):
                code = code.replace(prev, new)
            for b in ("min", "max"):
                if b in var["bounds"]:
                    var["bounds"][b] = _bound_code(var["name"], var["bounds"][b], desc, untouched)
            var["cpp"] = code
            var["dependencies"] = st.dependencies()
    return desc


__all__ = ["analyse_neuron", "analyse_synapse", "ParserError", "BUILTIN_FUNCTIONS"]
