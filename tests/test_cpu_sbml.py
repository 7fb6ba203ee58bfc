"""Model files in the reference's format (SBML level 2 with Inchman annotations,
read as InchmanDiffusionModel.cpp does): our fixtures under tests/golden/models/ and,
where the reference tree is present, its own doc/examples."""
import glob
import os

import numpy as np
import pytest

from inchman_b200 import _lib, sbml
from inchman_b200.sbml import Unsupported

HERE = os.path.dirname(os.path.abspath(__file__))
MODELS = os.path.join(HERE, "golden", "models")
# the reference checkout, when present: INCHMAN_REFERENCE names its root
REF_EXAMPLES = os.path.join(os.environ.get("INCHMAN_REFERENCE", ""), "doc", "examples")


def test_fixture_ab_drift():
    lm = sbml.load(os.path.join(MODELS, "ab_drift.xml"))
    m = lm.model
    assert m.solver == _lib.STOCHASTIC_INHOMOGENEOUS and (m.width, m.height) == (24, 24)
    assert m.physical_length == 12.0 and m.max_time == pytest.approx(0.3) and m.output_interval == pytest.approx(0.1)
    assert [r.id for r in m.reactions] == ["AA", "AB", "Asrc"]
    assert [r.rate for r in m.reactions] == pytest.approx([0.002, 0.02, 1.5])
    assert m.reactions[0].reactants == {"A": 2} and m.reactions[2].products == {"A": 1}
    assert m.custom_laws is None                       # all three are mass action
    assert m.drift_method == _lib.DRIFT_CODE and "All->DriftX = 0.4" in m.drift_code
    assert "#define A SP(0)" in m.code_defines and "#define k3 1.5f" in m.code_defines
    # initial amounts: the reference's homogeneous rule (amount // area per cell, one more
    # in the cells whose grid offset is below amount % area)
    st = m.initial_state(np.random.default_rng(0))
    a = st[0, 0]
    assert a.sum() == 24 * 24 * 20 + 7 and a.flat[:7].tolist() == [21] * 7 and (a.flat[7:] == 20).all()
    # the rule's offset is the grid offset, not the offset inside the compartment, so in
    # an 8 x 24 compartment only 40 of the 120 remainder cells get their extra particle:
    # 192 * 15 + 40 = 2920 of 3000 (the reference places the same)
    b = st[0, 1]
    assert b.sum() == 192 * 15 + 40 and (b[:, 8:] == 0).all()


def test_fixture_custom_law_becomes_code():
    lm = sbml.load(os.path.join(MODELS, "saturating.xml"))
    m = lm.model
    assert m.solver == _lib.STOCHASTIC_HOMOGENEOUS
    assert m.custom_laws == ["((40.0f * X(0)) / (25.0f + X(0)))", None]
    assert m.reactions[1].rate == pytest.approx(0.3)


@pytest.mark.parametrize("law,reactants,rate", [
    ("k*A*(A-1)", {"A": 2}, 0.5), ("k*A*B", {"A": 1, "B": 1}, 0.5), ("k", {}, 0.5), ("A", {"A": 1}, 1.0),
    ("k*A*A", {"A": 2}, None), ("k*A/(1+A)", {"A": 1}, None), ("k*B", {"A": 1}, None),
])
def test_mass_action_recognition(law, reactants, rate):
    import xml.etree.ElementTree as ET

    def tree(s):
        # tiny infix -> tree for the test cases above
        s = s.replace(" ", "")
        import ast
        node = ast.parse(s, mode="eval").body

        def conv(n):
            if isinstance(n, ast.BinOp):
                op = {ast.Mult: "times", ast.Add: "plus", ast.Sub: "minus", ast.Div: "divide"}[type(n.op)]
                return (op, [conv(n.left), conv(n.right)])
            if isinstance(n, ast.Name):
                return ("id", n.id)
            return ("num", float(n.value))
        return conv(node)

    got = sbml.mass_action_rate(tree(law), reactants, {"A", "B"}, {"k": 0.5})
    assert got == (pytest.approx(rate) if rate is not None else None)


def test_unsupported_features_are_named():
    text = open(os.path.join(MODELS, "saturating.xml")).read()
    with pytest.raises(Unsupported, match="init script"):
        sbml.load(text.replace("<im:script><![CDATA[]]></im:script></im:init>",
                               "<im:script><![CDATA[x = 1]]></im:script></im:init>"))
    lm = sbml.load(text.replace("<im:script><![CDATA[]]></im:script></im:init>",
                                "<im:script><![CDATA[x = 1]]></im:script></im:init>"), ignore_scripts=True)
    assert lm.notes and "init script ignored" in lm.notes[0]


@pytest.mark.skipif(not os.path.isdir(REF_EXAMPLES), reason="reference examples not present")
def test_reference_examples_load_or_name_what_is_missing():
    ok, unsupported = {}, {}
    for f in sorted(glob.glob(os.path.join(REF_EXAMPLES, "*.xml"))):
        name = os.path.basename(f)
        try:
            ok[name] = sbml.load(f).model
        except Unsupported as e:
            unsupported[name] = str(e)
    assert {"ABReaction.xml", "HomogeneousDiffusion.xml", "HomogeneousDrift.xml", "OrnsteinUhlenbeck.xml",
            "MultiplicativeNoise.xml", "ABAnnihilationDrift.xml"} <= set(ok)
    ab = ok["ABReaction.xml"]
    assert [r.rate for r in ab.reactions] == pytest.approx([1e-3, 1e-2, 1.2, 1.0])
    assert ab.reactions[0].reactants == {"SpeciesA": 2}
    ind = ok["ABReactionIndividual.xml"]
    assert [sp.individual for sp in ind.species][:2] == [True, True]
    # what still needs its Python script is named; without the scripts all load
    assert all("script" in why for why in unsupported.values()), unsupported
    for name in unsupported:
        sbml.load(os.path.join(REF_EXAMPLES, name), ignore_scripts=True)
    slit = sbml.load(os.path.join(REF_EXAMPLES, "Slit.xml"), ignore_scripts=True).model
    assert slit.field_names and slit.flags & 1          # field parameters, nonlinear method
    # without its (Python 2) init script the Calcium model loads, with custom laws
    ca = sbml.load(os.path.join(REF_EXAMPLES, "Calcium.xml"), ignore_scripts=True).model
    assert ca.custom_laws is not None and sum(l is not None for l in ca.custom_laws) >= 3


def test_fixture_localised_reactions():
    """localised.xml: reactions allowed in some compartments (isAllowed true), others
    (isAllowed false) left out; the mask is the union of the allowed rectangles, and a
    reaction allowed in World fires everywhere (InchmanDiffusionModel.cpp:410-435,
    Reaction.cpp:216-235)."""
    m = sbml.load(os.path.join(MODELS, "localised.xml")).model
    assert [r.id for r in m.reactions] == ["make", "bind", "decay", "bmake"]
    assert m.reactions[0].regions == [(7, 7, 8, 8)]
    assert m.reactions[1].regions == [(0, 0, 5, 15)]
    assert m.reactions[2].regions == [(0, 0, 15, 15)]
    assert m.reactions[3].regions == [(10, 0, 15, 15)]
    mask = m.reaction_mask()
    assert mask.shape == (4, 16, 16) and mask.dtype == np.uint8
    assert mask[0].sum() == 4 and mask[0, 7:9, 7:9].all()
    assert mask[1, :, :6].all() and not mask[1, :, 6:].any()
    assert mask[2].all()
    assert mask[3, :, 10:].all() and not mask[3, :, :10].any()
    assert m.custom_laws[3] is not None and m.custom_laws[0] is None
    desc, keep = m.to_desc()
    assert bool(desc.reaction_mask)
    # without localised reactions the descriptor carries no mask
    m2 = sbml.load(os.path.join(MODELS, "saturating.xml")).model
    assert m2.reaction_mask() is None and not bool(m2.to_desc()[0].reaction_mask)
