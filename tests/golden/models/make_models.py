"""Writes the annotated-SBML model fixtures of tests/golden/models/ (our own small
models in the file format of the reference's editor: SBML level 2 with Inchman
annotations, as InchmanDiffusionModel.cpp reads it).  Run from the repository root:
    python tests/golden/models/make_models.py
"""
import os

HERE = os.path.dirname(os.path.abspath(__file__))
IMNS = "http://www.csse.monash.edu.au/~berndm/inchman"
MML = "http://www.w3.org/1998/Math/MathML"


def num(v):
    return f'<math:math xmlns:math="{MML}"><math:cn>{v}</math:cn></math:math>'


def document(name, solver, W, L, time, out, params, comps, species, reactions, method="", newind=None,
             individual=(), nonlinear=False, moments=False, fields=(), set_field=None):
    ps = "\n".join(f'      <parameter id="{k}" value="{v}"><annotation><im:parameter xmlns:im="{IMNS}" '
                   f'type="float" domain="single"/></annotation></parameter>' for k, v in params.items())
    if fields:
        ps += "\n" + "\n".join(f'      <parameter id="{f}" value="0"><annotation><im:parameter xmlns:im="{IMNS}" '
                                f'type="float" domain="field"/></annotation></parameter>' for f in fields)
    cs = "\n".join(f'      <compartment id="{cid}"><annotation><im:compartment xmlns:im="{IMNS}">'
                   f'<im:x>{num(x)}</im:x><im:y>{num(y)}</im:y><im:width>{num(w)}</im:width>'
                   f'<im:height>{num(h)}</im:height></im:compartment></annotation></compartment>'
                   for cid, (x, y, w, h) in comps.items())
    ss = []
    for sid, (D, amounts) in species.items():
        cp = "".join(f'<im:compartmentParameters compartment="{c}"><im:initialAmount>{num(a)}</im:initialAmount>'
                     f'</im:compartmentParameters>' for c, a in amounts.items())
        ss.append(f'      <species id="{sid}" compartment="World"><annotation><im:species xmlns:im="{IMNS}">'
                  f'<im:diffusionConstant>{num(D)}</im:diffusionConstant>'
                  f'<im:listOfCompartmentParameters>{cp}</im:listOfCompartmentParameters>'
                  + ('<im:individual/>' if sid in individual else '') +
                  f'</im:species></annotation></species>')
    rs = []
    for rid, spec in reactions.items():
        # (reactants, products, law[, {compartment: allowed}]): without the fourth entry
        # the reaction is allowed in World, as the editor writes a global reaction
        re_, pr, law = spec[:3]
        allowed = spec[3] if len(spec) > 3 else {"World": True}
        rl = "".join(f'<speciesReference species="{s}" stoichiometry="{n}"/>' for s, n in re_.items())
        pl = "".join(f'<speciesReference species="{s}" stoichiometry="{n}"/>' for s, n in pr.items())
        cps = "".join(f'<im:compartmentParameters compartment="{c}"><im:isAllowed>'
                      f'<math xmlns="{MML}"><ci>{"true" if ok else "false"}</ci></math></im:isAllowed>'
                      f'</im:compartmentParameters>' for c, ok in allowed.items())
        rs.append(f'      <reaction id="{rid}"><annotation><im:reaction xmlns:im="{IMNS}">'
                  f'<im:listOfCompartmentParameters>{cps}'
                  f'</im:listOfCompartmentParameters></im:reaction></annotation>'
                  f'<listOfReactants>{rl}</listOfReactants><listOfProducts>{pl}</listOfProducts>'
                  f'<kineticLaw><math xmlns="{MML}">{law}</math></kineticLaw></reaction>')
    return f'''<?xml version="1.0" encoding="UTF-8"?>
<sbml xmlns="http://www.sbml.org/sbml/level2" level="2" version="1">
<annotation><im:sbml xmlns:im="{IMNS}">
  <im:solver>{solver}</im:solver>
  <im:runs>{num(1)}</im:runs>
  <im:time>{num(time)}</im:time>
  <im:outputInterval>{num(out)}</im:outputInterval>
  <im:init type="python"><im:script><![CDATA[]]></im:script></im:init>
  <im:events type="python"><im:script><![CDATA[]]></im:script><im:listOfTimeStamps/></im:events>
  <im:driftDiffusivity nonLinear="{"true" if nonlinear else "false"}" computeMoments="{"true" if moments else ""}"><im:method><![CDATA[{method}]]></im:method></im:driftDiffusivity>
{"" if newind is None else f"  <im:newIndividualsMethod><im:method><![CDATA[{newind}]]></im:method></im:newIndividualsMethod>" + chr(10)}{"" if set_field is None else f"  <im:setField><im:method><![CDATA[{set_field}]]></im:method></im:setField>" + chr(10)}</im:sbml></annotation>
  <model name="{name}">
<annotation><im:model xmlns:im="{IMNS}"><im:gridWidth>{num(W)}</im:gridWidth><im:gridHeight>{num(W)}</im:gridHeight>
<im:physicalWidth>{num(L)}</im:physicalWidth><im:physicalHeight>{num(L)}</im:physicalHeight></im:model></annotation>
    <listOfCompartments>
{cs}
    </listOfCompartments>
    <listOfSpecies>
{chr(10).join(ss)}
    </listOfSpecies>
    <listOfParameters>
{ps}
    </listOfParameters>
    <listOfReactions>
{chr(10).join(rs)}
    </listOfReactions>
  </model>
</sbml>
'''


def times(*xs):
    return "<apply><times/>" + "".join(xs) + "</apply>"


def ci(n):
    return f"<ci>{n}</ci>"


def cn(v):
    return f"<cn>{v}</cn>"


def minus(a, b):
    return f"<apply><minus/>{a}{b}</apply>"


def plus(a, b):
    return f"<apply><plus/>{a}{b}</apply>"


def divide(a, b):
    return f"<apply><divide/>{a}{b}</apply>"


def main():
    # A+B annihilation with drift, 2A annihilation, sources; mass-action laws
    ab = document(
        "AB drift", "stochastic_inhomogeneous", 24, 12.0, 0.3, 0.1, {"k1": 0.002, "k2": 0.02, "k3": 1.5},
        {"World": (0, 0, 24, 24), "Left": (0, 0, 8, 24)},
        {"A": (1.0, {"World": 24 * 24 * 20 + 7}), "B": (0.5, {"Left": 3000})},
        {"AA": ({"A": 2}, {}, times(times(ci("k1"), ci("A")), minus(ci("A"), cn("1.0")))),
         "AB": ({"A": 1, "B": 1}, {}, times(times(ci("k2"), ci("A")), ci("B"))),
         "Asrc": ({}, {"A": 1}, ci("k3"))},
        method="All->DiffusivityX = 1.;\nAll->DiffusivityY = 0.5;\nAll->DriftX = 0.4;\nB->DriftX = -0.2;\n"
               "All->DriftY = -0.1;")
    # saturating production (a custom law): 0 -> P at vmax S / (km + S), S -> 0
    mm = document(
        "Saturating production", "stochastic_homogeneous", 8, 8.0, 0.5, 0.25, {"vmax": 40.0, "km": 25.0, "kd": 0.3},
        {"World": (0, 0, 8, 8)},
        {"S": (0.5, {"World": 64 * 30}), "P": (0.2, {})},
        {"prod": ({}, {"P": 1}, divide(times(ci("vmax"), ci("S")), plus(ci("km"), ci("S")))),
         "deg": ({"S": 1}, {}, times(ci("kd"), ci("S")))})
    # individual species: A tracked one by one (decays, made from B), drift per
    # individual, new individuals with a random drift
    ind = document(
        "Individual A", "stochastic_inhomogeneous", 16, 16.0, 0.6, 0.2, {"kd": 0.5, "km": 0.2},
        {"World": (0, 0, 16, 16)},
        {"A": (0.0, {"World": 16 * 16 * 6}), "B": (0.5, {"World": 16 * 16 * 3})},
        {"decay": ({"A": 1}, {}, times(ci("kd"), ci("A"))),
         "make": ({"B": 1}, {"A": 1, "B": 1}, times(ci("km"), ci("B")))},
        method="A->DiffusivityX = 0.8;\nA->DiffusivityY = 0.6;\nA->DriftX = A->DriftX + 0.1;\nA->DriftY = 0.0;\n"
               "B->DiffusivityX = 0.5;\nB->DiffusivityY = 0.5;\nB->DriftX = 0.0;\nB->DriftY = 0.0;",
        newind="All->DriftX = 0.2 * RANDOM;", individual=("A",))
    # a nonlinear method: drift towards the species' mean x (moments), diffusivity
    # growing with the local count
    nl = document(
        "Nonlinear pull", "stochastic_inhomogeneous", 16, 16.0, 0.5, 0.25, {"pull": 0.4},
        {"World": (0, 0, 16, 16), "Left": (0, 0, 5, 16)},
        {"A": (0.0, {"Left": 5 * 16 * 12})}, {},
        method="All->DiffusivityX = 0.3 + 0.02 * All->State;\nAll->DiffusivityY = 0.3;\n"
               "All->DriftX = -pull * (PhysicalX - All->MeanX);\nAll->DriftY = 0.0;",
        nonlinear=True, moments=True)
    # a field parameter: the setField method accumulates where A is, the drift method
    # reads it
    fd = document(
        "Trace field", "stochastic_inhomogeneous", 12, 12.0, 0.4, 0.2, {"rate": 0.5},
        {"World": (0, 0, 12, 12)},
        {"A": (0.0, {"World": 12 * 12 * 8})}, {},
        method="All->DiffusivityX = 0.4 + 0.0 * trace;\nAll->DiffusivityY = 0.4;\nAll->DriftX = 0.0;\n"
               "All->DriftY = 0.0;",
        fields=("trace",), set_field="trace = trace + rate * deltat * A;")
    # localised reactions: A made only in a spot, A + B -> C only in the left part, C
    # decays everywhere, B made by a saturating (custom) law only in the right part
    loc = document(
        "Localised reactions", "stochastic_homogeneous", 16, 16.0, 0.6, 0.2,
        {"ks": 30.0, "kb": 0.02, "kd": 0.4, "vm": 12.0, "km": 10.0},
        {"World": (0, 0, 16, 16), "Left": (0, 0, 6, 16), "Right": (10, 0, 6, 16), "Spot": (7, 7, 2, 2)},
        {"A": (1.0, {"World": 16 * 16 * 10}), "B": (0.8, {"World": 16 * 16 * 10}), "C": (0.3, {})},
        {"make": ({}, {"A": 1}, ci("ks"), {"World": False, "Spot": True}),
         "bind": ({"A": 1, "B": 1}, {"C": 1}, times(times(ci("kb"), ci("A")), ci("B")), {"Left": True}),
         "decay": ({"C": 1}, {}, times(ci("kd"), ci("C"))),
         "bmake": ({}, {"B": 1}, divide(times(ci("vm"), ci("B")), plus(ci("km"), ci("B"))), {"Right": True})})
    for name, text in (("ab_drift.xml", ab), ("saturating.xml", mm), ("individual_a.xml", ind),
                       ("nonlinear.xml", nl), ("field_trace.xml", fd), ("localised.xml", loc)):
        with open(os.path.join(HERE, name), "w") as f:
            f.write(text)


if __name__ == "__main__":
    main()
