"""Model files of the reference: SBML level 2 with Inchman annotations (the editor's
output, as in doc/examples/*.xml) -> DiffusionModel.

Follows InchmanDiffusionModel.cpp:
  document annotation <im:sbml>  solver, runs, steps, time, outputInterval, init and
                                 events scripts, driftDiffusivity method (:120-210)
  model annotation <im:model>    gridWidth, gridHeight, physicalWidth (:212-219)
  parameters                     value; domain "single" or "field" (:283-297)
  compartments                   x, y, width, height (:300-313)
  species                        diffusionConstant, initial amount per compartment,
                                 individual flag (:316-358)
  reactions                      reactant/product stoichiometry, kinetic law,
                                 compartment localisation (:361-439)
Numbers are MathML (<cn>, <ci> of a parameter, <apply>).

Kinetic laws: a law that is a product of constants and the falling factorials of the
reactants, k A (A-1) ... B ... (the reference's mass-action hazard,
Reaction.cpp:119-138), becomes a built-in mass-action reaction; any other law is kept
as a C expression and compiled into the SSA kernel at run time (custom_laws).  The
drift/diffusivity method is C code; it is compiled at run time as well (DRIFT_CODE),
with the parameters as defines and every species id bound to SP(i).

Individual species (<im:individual/>) become individual species of the solver, with the
newIndividualsMethod compiled at run time; their properties start at zero, as the
reference's do without an init script.

A nonlinear drift method (nonLinear="true", or computeMoments="true") that reads the
state, the time or MeanX is evaluated again after every sweep (GPGMP_FLAG_NONLINEAR,
GPGMP_FLAG_COMPUTE_MOMENTS; one realisation per solver).

Field parameters (domain "field") are per-cell values, zero until set (the reference's
init scripts fill them): the model code reads them by name (F(f)), and the setField
method, compiled at run time, updates them every step.

Reactions localised to compartments fire only inside them (the reaction mask of
Solver.cpp:352-390).

Not supported (raises Unsupported): init and event scripts (Python run by the
reference's executable).
"""
from __future__ import annotations

import math
import re
import xml.etree.ElementTree as ET
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np

from . import _lib
from .model import Compartment, DiffusionModel

SB = "{http://www.sbml.org/sbml/level2}"
IM = "{http://www.csse.monash.edu.au/~berndm/inchman}"
MM = "{http://www.w3.org/1998/Math/MathML}"

# DiffusionModel::setSolver (DiffusionModel.cpp:250-263)
SOLVERS = {
    "stochastic_homogeneous": _lib.STOCHASTIC_HOMOGENEOUS,
    "stochastic_inhomogeneous": _lib.STOCHASTIC_INHOMOGENEOUS,
    "stochastic_inhomogeneous_fpe": _lib.STOCHASTIC_INHOMOGENEOUS_FPE,
    "deterministic_homogeneous": _lib.DETERMINISTIC_RK4,
    "deterministic_homogeneous_RK4": _lib.DETERMINISTIC_RK4,
    "deterministic_homogeneous_aqss": _lib.DETERMINISTIC_AQSS,
    "deterministic_inhomogeneous_RK4": _lib.DETERMINISTIC_INHOMOGENEOUS_RK4,
    "deterministic_inhomogeneous_aqss": _lib.DETERMINISTIC_INHOMOGENEOUS_AQSS,
}

# identifiers a drift method may use besides parameters and species (the reference's
# generated kernel, Solver.cpp:684-700, and helpers.cl)
DRIFT_NAMES = {"All", "Real", "GridX", "GridY", "PhysicalX", "PhysicalY", "PhysicalModelWidth",
               "PhysicalModelHeight", "PhysicalCellWidth", "PhysicalCellHeight", "GridModelWidth",
               "GridModelHeight", "PhysicalSimTime", "DiffusivityX", "DiffusivityY", "DriftX", "DriftY", "State",
               "MeanX", "SpeciesState", "getCentralDifferenceX", "getCentralDifferenceY", "getPhysicalX",
               "getPhysicalY"}
C_MATH = {"sin", "cos", "tan", "exp", "log", "sqrt", "pow", "fabs", "tanh", "sinh", "cosh", "atan", "atan2",
          "floor", "ceil", "fmin", "fmax", "asin", "acos", "if", "else", "return", "float", "int", "double",
          "sinf", "cosf", "expf", "logf", "sqrtf", "powf", "fabsf", "fminf", "fmaxf", "true", "false"}


class Unsupported(ValueError):
    """The model uses a feature of the reference this build does not run."""


# ---- MathML -------------------------------------------------------------------------
# expression tree: ("num", value) | ("id", name) | (op, [args])

def mathml(e: ET.Element):
    tag = e.tag.replace(MM, "")
    if tag == "math":
        kids = list(e)
        if len(kids) != 1:
            raise ValueError("MathML <math> with %d children" % len(kids))
        return mathml(kids[0])
    if tag == "cn":
        t = (e.get("type") or "real").lower()
        if t == "e-notation":
            parts = [p for p in (e.text or "").split() if p]
            sep = e.find(MM + "sep")
            mant = float((e.text or "").strip())
            ex = float((sep.tail or "").strip()) if sep is not None else 0.0
            return ("num", mant * 10.0 ** ex)
        return ("num", float((e.text or "").strip()))
    if tag == "ci":
        name = (e.text or "").strip()
        try:
            return ("num", float(name))          # editors write some numbers as <ci>
        except ValueError:
            return ("id", name)
    if tag in ("true", "false"):
        return ("num", 1.0 if tag == "true" else 0.0)
    if tag in ("exponentiale",):
        return ("num", math.e)
    if tag in ("pi",):
        return ("num", math.pi)
    if tag == "apply":
        kids = list(e)
        op = kids[0].tag.replace(MM, "")
        args = [mathml(k) for k in kids[1:] if k.tag.replace(MM, "") not in ("logbase", "degree")]
        if op == "log":
            base = kids[1].find(MM + "cn") if len(kids) > 1 and kids[1].tag == MM + "logbase" else None
            if base is not None:
                return ("divide", [("ln", args), ("ln", [mathml(base)])])
            return ("log10", args)
        if op == "root":
            return ("sqrt", args)
        return (op, args)
    raise ValueError(f"unsupported MathML element <{tag}>")


def ids_in(t) -> set:
    if t[0] == "id":
        return {t[1]}
    if t[0] == "num":
        return set()
    out = set()
    for a in t[1]:
        out |= ids_in(a)
    return out


def evaluate(t, env: Dict[str, float]) -> float:
    k = t[0]
    if k == "num":
        return t[1]
    if k == "id":
        if t[1] in ("true", "false"):
            return 1.0 if t[1] == "true" else 0.0
        if t[1] not in env:
            raise Unsupported(f"unknown identifier {t[1]!r} in a constant expression")
        return env[t[1]]
    a = [evaluate(x, env) for x in t[1]]
    if k == "times":
        return float(np.prod(a)) if a else 1.0
    if k == "plus":
        return float(sum(a))
    if k == "minus":
        return -a[0] if len(a) == 1 else a[0] - a[1]
    if k == "divide":
        return a[0] / a[1]
    if k == "power":
        return a[0] ** a[1]
    fn = {"exp": math.exp, "ln": math.log, "log10": math.log10, "sqrt": math.sqrt, "abs": abs,
          "floor": math.floor, "ceiling": math.ceil, "sin": math.sin, "cos": math.cos, "tanh": math.tanh}
    if k in fn:
        return fn[k](a[0])
    raise Unsupported(f"MathML operator {k!r}")


def c_float(v: float) -> str:
    return repr(float(np.float32(v))) + "f" if np.isfinite(v) else ("(1.0f/0.0f)" if v > 0 else "(-1.0f/0.0f)")


def to_c(t, names: Dict[str, str]) -> str:
    """C expression of the tree; names maps identifiers to C text."""
    k = t[0]
    if k == "num":
        return c_float(t[1])
    if k == "id":
        if t[1] not in names:
            raise Unsupported(f"unknown identifier {t[1]!r} in a kinetic law")
        return names[t[1]]
    a = [to_c(x, names) for x in t[1]]
    if k == "times":
        return "(" + " * ".join(a) + ")"
    if k == "plus":
        return "(" + " + ".join(a) + ")"
    if k == "minus":
        return f"(-{a[0]})" if len(a) == 1 else f"({a[0]} - {a[1]})"
    if k == "divide":
        return f"({a[0]} / {a[1]})"
    if k == "power":
        return f"powf({a[0]}, {a[1]})"
    fn = {"exp": "expf", "ln": "logf", "log10": "log10f", "sqrt": "sqrtf", "abs": "fabsf", "floor": "floorf",
          "ceiling": "ceilf", "sin": "sinf", "cos": "cosf", "tanh": "tanhf"}
    if k in fn:
        return f"{fn[k]}({a[0]})"
    raise Unsupported(f"MathML operator {k!r} in a kinetic law")


def _flatten_times(t) -> List:
    if t[0] == "times":
        out = []
        for a in t[1]:
            out += _flatten_times(a)
        return out
    return [t]


def mass_action_rate(t, reactants: Dict[str, int], species: set, env: Dict[str, float]) -> Optional[float]:
    """The rate constant when the law is rate * prod_s s (s-1) ... (s-nu_s+1) over the
    reactants (the built-in hazard), else None."""
    const = 1.0
    falling: Dict[str, List[int]] = {}
    for f in _flatten_times(t):
        used = ids_in(f) & species
        if not used:
            try:
                const *= evaluate(f, env)
            except (Unsupported, ZeroDivisionError, OverflowError, ValueError):
                return None
            continue
        if f[0] == "id":
            falling.setdefault(f[1], []).append(0)
        elif f[0] == "minus" and len(f[1]) == 2 and f[1][0][0] == "id" and f[1][0][1] in species \
                and not (ids_in(f[1][1]) & species):
            off = evaluate(f[1][1], env)
            if off != int(off) or off < 0:
                return None
            falling.setdefault(f[1][0][1], []).append(int(off))
        else:
            return None
    if set(falling) != {s for s, n in reactants.items() if n > 0}:
        return None
    for s, offs in falling.items():
        if sorted(offs) != list(range(reactants[s])):
            return None
    return const


# ---- drift/diffusivity method -------------------------------------------------------

_COMMENT = re.compile(r"//[^\n]*|/\*.*?\*/", re.S)
_IDENT = re.compile(r"[A-Za-z_][A-Za-z0-9_]*")


def drift_identifiers(code: str) -> set:
    c = _COMMENT.sub(" ", code)
    c = re.sub(r"(?<![A-Za-z_0-9])\.?\d+\.?\d*([eE][-+]?\d+)?[fF]?", " ", c)   # numbers, not B00's digits
    return set(_IDENT.findall(c))


# ---- the loader ---------------------------------------------------------------------

@dataclass
class LoadedModel:
    model: DiffusionModel
    runs: int = 1
    parameters: Dict[str, float] = field(default_factory=dict)
    notes: List[str] = field(default_factory=list)
    # named compartments as inclusive rectangles (x0, y0, x1, y1), in file order
    compartments: Dict[str, Tuple[int, int, int, int]] = field(default_factory=dict)
    source: str = ""          # the model file's text


def _text(e: Optional[ET.Element]) -> str:
    return (e.text or "").strip() if e is not None else ""


def _num(parent: Optional[ET.Element], name: str, env: Dict[str, float]) -> Optional[float]:
    if parent is None:
        return None
    c = parent.find(IM + name)
    if c is None:
        return None
    m = c.find(MM + "math")
    if m is None:
        t = _text(c)
        return float(t) if t else None
    return evaluate(mathml(m), env)


def load(source: str, *, ignore_scripts: bool = False, overrides: Optional[Dict[str, float]] = None) -> LoadedModel:
    """source: a file path or the XML text.  ignore_scripts: load a model whose init
    or event scripts are non-empty without them (the reference runs them as Python).
    overrides: parameter values that replace (or add to) the file's, before any
    expression is evaluated (the executable's --p name=value,
    InchmanDiffusionModel.cpp:100-118)."""
    text = source if source.lstrip().startswith("<") else open(source, encoding="utf-8").read()
    root = ET.fromstring(text)
    model_e = root.find(SB + "model")
    if model_e is None:
        raise ValueError("no <model> element")
    notes: List[str] = []
    # parameters first: every MathML expression may refer to them
    params: Dict[str, float] = {}
    fields: List[str] = []
    for p in model_e.iter(SB + "parameter"):
        a = p.find(f"{SB}annotation/{IM}parameter")
        domain = a.get("domain", "single") if a is not None else "single"
        if domain == "field":
            # a per-cell value, zero until set (DiffusionModel.cpp:402-404, 778)
            fields.append(p.get("id"))
            continue
        if domain != "single":
            raise Unsupported(f"parameter domain {domain!r}")
        params[p.get("id")] = float(p.get("value", "0"))
    fields.sort()      # the reference keeps them in a std::map: offsets in name order
    for k, v in (overrides or {}).items():
        params[k] = float(v)
    sb = root.find(f"{SB}annotation/{IM}sbml")
    m = DiffusionModel()
    runs = 1
    method = ""
    nonlinear = False
    moments = False
    set_field = ""
    if sb is not None:
        solver = _text(sb.find(IM + "solver")) or "stochastic_inhomogeneous"
        if solver not in SOLVERS:
            raise Unsupported(f"solver {solver!r}")
        m.solver = SOLVERS[solver]
        v = _num(sb, "runs", params)
        runs = int(v) if v is not None else 1
        v = _num(sb, "steps", params)
        if v is not None:
            m.max_steps = int(v)
        v = _num(sb, "time", params)
        if v is not None:
            m.max_time = float(v)
        v = _num(sb, "outputInterval", params)
        if v is not None:
            m.output_interval = float(v)
        for kind in ("init", "events"):
            sc = sb.find(f"{IM}{kind}/{IM}script")
            if sc is not None and _text(sc):
                if not ignore_scripts:
                    raise Unsupported(f"the model's {kind} script (Python run by the reference's executable)")
                notes.append(f"{kind} script ignored")
        dd = sb.find(IM + "driftDiffusivity")
        if dd is not None:
            method = _text(dd.find(IM + "method"))
            nonlinear = dd.get("nonLinear", "false") == "true"
            moments = dd.get("computeMoments", "") == "true"
        sf = sb.find(f"{IM}setField/{IM}method")
        set_field = _text(sf) if sf is not None else ""
        ni = sb.find(f"{IM}newIndividualsMethod/{IM}method")
        newind = _text(ni) if ni is not None else ""
    ma = model_e.find(f"{SB}annotation/{IM}model")
    if ma is not None:
        for name, attr in (("gridWidth", "width"), ("gridHeight", "height")):
            v = _num(ma, name, params)
            if v is not None:
                setattr(m, attr, int(v))
        v = _num(ma, "physicalWidth", params)
        if v is not None:
            m.physical_length = float(v)
    W, H = m.width, m.height
    # constants the reference's generated code defines (Solver.cpp:499-504)
    env = dict(params)
    env.update(PhysicalModelWidth=m.physical_length, PhysicalModelHeight=m.physical_length,
               PhysicalCellWidth=float(np.float32(m.physical_length) / np.float32(W)),
               PhysicalCellHeight=float(np.float32(m.physical_length) / np.float32(H)),
               GridModelWidth=float(W), GridModelHeight=float(H))
    # compartments: inclusive rectangles
    comps: Dict[str, Tuple[int, int, int, int]] = {}
    for c in model_e.iter(SB + "compartment"):
        a = c.find(f"{SB}annotation/{IM}compartment")
        x0 = int(_num(a, "x", env) or 0)
        y0 = int(_num(a, "y", env) or 0)
        w = int(_num(a, "width", env) or W)
        h = int(_num(a, "height", env) or H)
        comps[c.get("id")] = (x0, y0, x0 + w - 1, y0 + h - 1)
    # species
    for s in model_e.iter(SB + "species"):
        sid = s.get("id")
        a = s.find(f"{SB}annotation/{IM}species")
        D = _num(a, "diffusionConstant", env) if a is not None else None
        m.add_species(sid, float(D or 0.0))
        if a is not None:
            if a.find(IM + "individual") is not None:
                # InchmanDiffusionModel.cpp:345-350: the molecules become individuals
                m.species[-1].individual = True
            lst = a.find(IM + "listOfCompartmentParameters")
            for cp in (lst if lst is not None else []):
                cid = cp.get("compartment")
                amount = _num(cp, "initialAmount", env)
                if cid in comps and amount:
                    x0, y0, x1, y1 = comps[cid]
                    m.add_compartment(Compartment(sid, x0, y0, x1, y1, int(amount), "homogeneous"))
    species_ids = [s.id for s in m.species]
    spset = set(species_ids)
    # reactions
    laws: List[Optional[str]] = []
    names = {sid: f"X({i})" for i, sid in enumerate(species_ids)}
    names.update({k: c_float(v) for k, v in env.items()})
    for r in model_e.iter(SB + "reaction"):
        rid = r.get("id")

        def refs(tag):
            out: Dict[str, int] = {}
            for sr in r.findall(f"{SB}{tag}/{SB}speciesReference"):
                out[sr.get("species")] = out.get(sr.get("species"), 0) + int(float(sr.get("stoichiometry", "1")))
            return out

        reactants, products = refs("listOfReactants"), refs("listOfProducts")
        # localisation (InchmanDiffusionModel.cpp:410-435): every compartment whose
        # isAllowed is non-zero; a reaction with none fires everywhere
        regions = []
        loc = r.find(f"{SB}annotation/{IM}reaction/{IM}listOfCompartmentParameters")
        if loc is not None:
            for cp in loc:
                if cp.tag != IM + "compartmentParameters":
                    continue
                v = _num(cp, "isAllowed", env)
                cid = cp.get("compartment")
                if v and cid in comps:
                    regions.append(comps[cid])
        kl = r.find(f"{SB}kineticLaw/{MM}math")
        if kl is None:
            raise Unsupported(f"reaction {rid!r} has no kinetic law")
        tree = mathml(kl)
        rate = mass_action_rate(tree, reactants, spset, env)
        if rate is not None:
            m.add_reaction(rid, reactants, products, float(rate), regions)
            laws.append(None)
        else:
            m.add_reaction(rid, reactants, products, 0.0, regions)
            laws.append(to_c(tree, names))
    if any(l is not None for l in laws):
        m.custom_laws = laws
        notes.append("custom kinetic laws compiled at run time")
    # drift / diffusivity method (inhomogeneous solvers)
    if m.solver in _lib.INHOMOGENEOUS_TYPES:
        used = drift_identifiers(method)
        dynamic = used & {"PhysicalSimTime", "State", "SpeciesState", "MeanX", "getCentralDifferenceX",
                          "getCentralDifferenceY"}
        if (nonlinear or moments) and dynamic:
            # evaluated again after every sweep (InhomogeneousSolver.cpp:288-335)
            if m.solver not in (_lib.STOCHASTIC_INHOMOGENEOUS, _lib.STOCHASTIC_INHOMOGENEOUS_FPE):
                raise Unsupported(f"a nonlinear drift method that reads {sorted(dynamic)} with a deterministic solver")
            m.flags |= _lib.FLAG_NONLINEAR | (_lib.FLAG_COMPUTE_MOMENTS if moments else 0)
            notes.append("nonlinear drift method: one realisation per solver")
        unknown = used - DRIFT_NAMES - set(params) - set(fields) - spset - C_MATH
        declared = set(re.findall(r"\bReal\s+([A-Za-z_]\w*)", _COMMENT.sub(" ", method)))
        unknown -= declared
        if unknown:
            raise Unsupported(f"drift method uses {sorted(unknown)}")
        m.drift_method = _lib.DRIFT_CODE
        m.drift_code = method
    field_defines = [f"#define {f} F({i})" for i, f in enumerate(fields)]
    if m.solver in _lib.INHOMOGENEOUS_TYPES:
        defines = [f"#define {k} {c_float(v)}" for k, v in params.items()] + field_defines
        defines += [f"#define {sid} SP({i})" for i, sid in enumerate(species_ids)]
        m.code_defines = "\n".join(defines)
    elif m.custom_laws is not None or fields:
        m.code_defines = "\n".join([f"#define {k} {c_float(v)}" for k, v in params.items()] + field_defines)
    if fields:
        m.field_names = list(fields)
        if set_field and _COMMENT.sub(" ", set_field).strip():
            # in the setField method a species name is its count (Solver.cpp:606-612)
            pre = "".join(f"#undef {sid}\n#define {sid} X({i})\n" for i, sid in enumerate(species_ids))
            m.set_field_code = pre + set_field
        notes.append("field parameters: " + ", ".join(fields) + " (zero until set)")
    if any(sp.individual for sp in m.species):
        if m.solver not in (_lib.STOCHASTIC_INHOMOGENEOUS, _lib.STOCHASTIC_INHOMOGENEOUS_FPE):
            raise Unsupported("individual species with a solver other than stochastic_inhomogeneous(_fpe)")
        if newind and _COMMENT.sub(" ", newind).strip():
            m.new_individuals_code = newind
        notes.append("individual species: " + ", ".join(sp.id for sp in m.species if sp.individual))
    return LoadedModel(model=m, runs=runs, parameters=params, notes=notes, compartments=comps, source=text)
