"""TEST INFRASTRUCTURE ONLY: builds the reference checker's model-specific kernels.

The reference's SSA and deterministic reaction kernels are templates
(Gillespie.cl, Deterministic.cl) whose marker comments ("// <<<! ... !>>>") the
reference's host replaces with code generated from the model at run time
(Solver::oclGenerateProgram, Solver.cpp:778-959; kinetic laws Reaction.cpp:119-162).
This script does that replacement for a few fixed test models, the way those lines
do it, and writes the programs as C files into oracle/_ref/gen/ (never into the
repository: they are derived from the reference's sources), plus one driver that
runs a kernel over every cell of the grid the way the reference enqueues it (local
size 1).  The templates themselves are read unchanged from the reference checkout.

Beyond the marker text, two OpenCL constructs are mapped to C here, as the shim
(cl_shim.h) maps the built-ins: vector literals "(int4)(a, b, c, d)" become
shim_int4(a, b, c, d), and "inline" functions become "static inline" (OpenCL C's
inline functions have no external definition).  <tgmath.h> gives C the overloads
OpenCL's math functions have (log of a float is the float logarithm).

    python oracle/ref/gen_models.py <reference gpgmp/src dir> <output dir>
"""
from __future__ import annotations

import os
import re
import sys

# The test models.  Species in creation order (the reference's reactant and product
# maps are keyed by Species*, i.e. allocation order, which is creation order here);
# reactions as (id, {reactant: stoich}, {product: stoich}, rate, localised).
MODELS = {
    # config 1's network
    "abc": (["A", "B", "C"], [("bind", {"A": 1, "B": 1}, {"C": 1}, 0.01, False),
                              ("unbind", {"C": 1}, {"A": 1, "B": 1}, 0.1, False)]),
    # second-order reactant, zero-order source, product stoichiometry 2
    "dimer": (["A", "B"], [("dim", {"A": 2}, {"B": 1}, 0.005, False),
                           ("split", {"B": 1}, {"A": 2}, 0.2, False),
                           ("src", {}, {"A": 1}, 3.0, False)]),
    # config 1's network with both reactions localised (reaction mask image)
    "abcloc": (["A", "B", "C"], [("bind", {"A": 1, "B": 1}, {"C": 1}, 0.01, True),
                                 ("unbind", {"C": 1}, {"A": 1, "B": 1}, 0.1, False),
                                 ("make", {}, {"C": 1}, 2.5, True)]),
    # Gray-Scott network of exec/src/tests/GrayScottModel.cpp:14-60 (F = 0.04, k = 0.06)
    "gs": (["U", "V"], [("r1", {"U": 1, "V": 2}, {"V": 3}, 1.0, False),
                        ("r2", {"U": 1}, {}, 0.04, False),
                        ("r3", {"V": 1}, {}, 0.1, False),
                        ("r4", {}, {"U": 1}, 0.04, False)]),
    "gsloc": (["U", "V"], [("r1", {"U": 1, "V": 2}, {"V": 3}, 1.0, True),
                           ("r2", {"U": 1}, {}, 0.04, False),
                           ("r3", {"V": 1}, {}, 0.1, True),
                           ("r4", {}, {"U": 1}, 0.04, False)]),
}
SSA_MODELS = ["abc", "dimer", "abcloc"]
DET_MODELS = ["gs", "gsloc"]


def fmt_rate(r: float) -> str:
    """`ss << m_reactionRate` (Reaction.cpp:122): a float printed with the default
    stream format, six significant digits (%g)."""
    return "%g" % r


def kinetic_law(species, re_, rate):
    """Reaction::generateKineticLaw (Reaction.cpp:119-138)."""
    s = fmt_rate(rate)
    for sp in species:
        if sp in re_:
            s += " * " + sp
            for k in range(1, re_[sp]):
                s += " * (%s-%d)" % (sp, k)
    return s


def deterministic_law(species, re_, rate):
    """Reaction::generateDeterministicLaw (Reaction.cpp:145-162)."""
    s = fmt_rate(rate)
    for sp in species:
        if sp in re_:
            s += " * " + sp
            for _ in range(1, re_[sp]):
                s += " * " + sp
    return s


def mask_term(j):
    return " read_imagef(_reactionMask, _reactionMaskSampler, (int4)(GridX, GridY, %d, 0)).x * " % j


def markers(species, reactions):
    """The replacement text of each marker, as Solver.cpp:778-959 builds it."""
    out = {}
    to_local, to_state, define, define_rk4 = [], [], [], []
    for i, sp in enumerate(species):
        to_local.append("    _localState[_localId + %d * _speciesOffsetLocal] = _globalState[_globalId + %d * "
                        "_speciesOffsetGlobal]; // species %s\n" % (i, i, sp))
        to_local.append("#define %s _localState[_localId + %d * _speciesOffsetLocal]\n" % (sp, i))
        to_state.append("    _globalState[_globalId + %d * _speciesOffsetGlobal] = _localState[_localId + %d * "
                        "_speciesOffsetLocal]; // species %s\n" % (i, i, sp))
        to_state.append("#undef %s\n" % sp)
        define.append("#define %s _localState[_localId + %d * _speciesOffsetLocal]\n" % (sp, i))
        define_rk4.append("#define %s _localState[ %d ]\n" % (sp, i))
    out["copyStateToLocal"] = "".join(to_local)
    out["copyLocalToState"] = "".join(to_state)
    out["defineSpeciesFromLocal"] = "".join(define)
    out["defineSpeciesFromLocalRK4"] = "".join(define_rk4)
    # Solver.cpp:820-824 writes the #undef lines into the define stream, so the
    # undefSpeciesFromLocal marker is replaced by an empty string
    out["undefSpeciesFromLocal"] = ""
    out["defineUserParameters"] = ""          # the test models have no parameters
    # Solver.cpp:843-858
    h = ["      _h[0] = 0.;\n"]
    for i, (rid, re_, pr, rate, loc) in enumerate(reactions):
        h.append("      // Reaction '%s'\n" % rid)
        h.append("      _h[%d] = _h[0] + " % (i + 1) + (mask_term(i) if loc else "") +
                 kinetic_law(species, re_, rate) + ";\n")
        h.append("      _h[0] = _h[%d];\n" % (i + 1))
    out["computeReactionHazards"] = "".join(h)
    # Solver.cpp:860-905 (without the debug-kernel lines)
    p = ["        // perform reactions\n", "        int _index;\n\n"]
    n = len(reactions)
    for i, (rid, re_, pr, rate, loc) in enumerate(reactions):
        p.append("        // Reaction '%s'\n" % rid)
        if i == 0:
            p.append("        _index = isless(_r2, _h[1]);\n")
        else:
            p.append("        _index = isgreaterequal(_r2, _h[%d]) * isless(_r2, _h[%d]);\n" % (i, i + 1))
        body = ""
        for sp in species:
            if sp in re_:
                body += "        %s = %s - %d * _index; \n" % (sp, sp, re_[sp])
        for sp in species:
            if sp in pr:
                body += "        %s = %s + %d * _index; \n" % (sp, sp, pr[sp])
        p.append(body + "\n")
    out["performReactions"] = "".join(p)
    # Solver.cpp:922-959
    rhs = []
    for i, sp in enumerate(species):
        line = "    _deriv[%d] = 0." % i
        for j, (rid, re_, pr, rate, loc) in enumerate(reactions):
            tot = pr.get(sp, 0) - re_.get(sp, 0)
            if tot != 0:
                line += (" + %d. * " % abs(tot)) if tot > 0 else (" - %d. * " % abs(tot))
                if loc:
                    line += mask_term(j)
                line += deterministic_law(species, re_, rate)
        rhs.append(line + ";\n")
    out["computeODERHS"] = "".join(rhs)
    # Solver.cpp:961-1004
    aq = []
    for i, sp in enumerate(species):
        aq.append("    // Species '%s'\n" % sp)
        prod, dest = "    _q[%d] = 0." % i, "    _d[%d] = 0." % i
        for j, (rid, re_, pr, rate, loc) in enumerate(reactions):
            tot = pr.get(sp, 0) - re_.get(sp, 0)
            if tot == 0:
                continue
            term = " + %d. * " % abs(tot) + (mask_term(j) if loc else "") + deterministic_law(species, re_, rate)
            if tot > 0:
                prod += term
            else:
                dest += term
        aq.append(prod + ";\n" + dest + ";\n\n")
    out["computeODERHSaqss"] = "".join(aq)
    out["updateFields"] = ""
    out["deterministicStoreDiffusionConstants"] = ""
    out["computeDriftDiffusivity"] = ""
    return out


def substitute(text, repl):
    for name, code in repl.items():
        text = text.replace("// <<<! %s !>>>" % name, code)
    left = re.findall(r"// <<<! (\w+) !>>>", text)
    if left:
        raise SystemExit("unreplaced markers: %s" % left)
    return text


def to_c(text):
    """OpenCL vector literals and inline functions in C form (see the module note)."""
    text = re.sub(r"\(int4\)\(([^()]*)\)", r"shim_int4(\1)", text)
    text = re.sub(r"(?m)^inline\s", "static inline ", text)
    return text


PRELUDE = """/* Generated by oracle/ref/gen_models.py from the reference's %(src)s for the test
 * model '%(model)s' (markers filled as Solver.cpp:778-959 fills them).  TEST
 * INFRASTRUCTURE ONLY; not part of the repository. */
#include "cl_shim.h"
#include <tgmath.h>
#undef GPGMP_NUM_REACTIONS
#define GPGMP_NUM_REACTIONS %(nr)d
%(loc)s
typedef struct { const float* data; int w, h; } image3d_t;
static inline int4 shim_int4(int a, int b, int c, int d) { int4 v = {a, b, c, d}; return v; }
static inline float4 read_imagef(image3d_t img, int sampler, int4 c) {
    (void)sampler;
    float4 r = {img.data[((size_t)c.z * img.h + c.y) * img.w + c.x], 0.f, 0.f, 0.f};
    return r;
}
#define _reactionMaskSampler 0
"""


def gen_ssa(model, src_text):
    species, reactions = MODELS[model]
    loc = any(r[4] for r in reactions)
    head = PRELUDE % {"src": "Gillespie.cl", "model": model, "nr": len(reactions),
                      "loc": "#define GPGMP_HAS_LOCALIZED_REACTIONS" if loc else ""}
    head += "#define performGillespie gref_ssa_kernel_%s\n#define updateFields gref_ssa_fields_%s\n" % (model, model)
    body = to_c(substitute(src_text, markers(species, reactions)))
    drv = """
/* one enqueue of performGillespie over the W x H grid, local size 1 (the reference
 * enqueues work-groups of the grid; each work-item reads and writes only its cell) */
void gref_ssa_%(m)s(int* state, int seed, float deltat, const float* mask) {
    int local[64];
    image3d_t img = {mask, (int)GridModelWidth, (int)GridModelHeight};
    (void)img;
    for (size_t y = 0; y < GridModelHeight; ++y)
        for (size_t x = 0; x < GridModelWidth; ++x) {
            shim_gid[0] = x; shim_gid[1] = y; shim_gsize[0] = GridModelWidth; shim_gsize[1] = GridModelHeight;
            shim_lid[0] = shim_lid[1] = 0; shim_lsize[0] = shim_lsize[1] = 1;
            shim_group[0] = x; shim_group[1] = y; shim_ngroups[0] = GridModelWidth; shim_ngroups[1] = GridModelHeight;
            gref_ssa_kernel_%(m)s(state, seed, deltat, %(imgarg)slocal);
        }
}
""" % {"m": model, "imgarg": "img, " if loc else ""}
    return head + body + drv


def gen_det(model, src_text):
    species, reactions = MODELS[model]
    loc = any(r[4] for r in reactions)
    head = PRELUDE % {"src": "Deterministic.cl", "model": model, "nr": len(reactions),
                      "loc": "#define GPGMP_HAS_LOCALIZED_REACTIONS" if loc else ""}
    head += "#define GPGMP_SOLVER_DETERMINISTIC_RK4\n"
    # OpenCL's min / max built-ins, used by the alpha-QSS kernel of the same file
    head += "#define min(a, b) fminf((a), (b))\n#define max(a, b) fmaxf((a), (b))\n"
    for k in ("homogeneous_deterministic_diffuse", "inhomogeneous_deterministic_diffuseX",
              "inhomogeneous_deterministic_diffuseY", "deterministic_rhs_ode_rk4", "deterministic_rhs_ode_aqss",
              "deterministic_performReaction_aqss"):
        head += "#define %s gref_%s_%s\n" % (k, k, model)
    head += "#define deterministic_performReaction_rk4 gref_rk4_kernel_%s\n" % model
    body = to_c(substitute(src_text, markers(species, reactions)))
    drv = """
/* one enqueue of deterministic_performReaction_rk4 over the grid, local size 1 */
void gref_rk4_%(m)s(float* state, float deltat, const float* mask) {
    float local[5 * 64];
    image3d_t img = {mask, (int)GridModelWidth, (int)GridModelHeight};
    (void)img;
    for (size_t y = 0; y < GridModelHeight; ++y)
        for (size_t x = 0; x < GridModelWidth; ++x) {
            shim_gid[0] = x; shim_gid[1] = y; shim_gsize[0] = GridModelWidth; shim_gsize[1] = GridModelHeight;
            shim_lid[0] = shim_lid[1] = 0; shim_lsize[0] = shim_lsize[1] = 1;
            shim_group[0] = x; shim_group[1] = y; shim_ngroups[0] = GridModelWidth; shim_ngroups[1] = GridModelHeight;
            gref_rk4_kernel_%(m)s(state, deltat, %(imgarg)slocal);
        }
}
""" % {"m": model, "imgarg": "img, " if loc else ""}
    return head + body + drv


def main(argv):
    if len(argv) != 3:
        raise SystemExit(__doc__)
    src, out = argv[1], argv[2]
    os.makedirs(out, exist_ok=True)
    gil = open(os.path.join(src, "Gillespie.cl")).read()
    det = open(os.path.join(src, "Deterministic.cl")).read()
    files = []
    for m in SSA_MODELS:
        files.append(("ssa_%s.c" % m, gen_ssa(m, gil)))
    for m in DET_MODELS:
        files.append(("det_%s.c" % m, gen_det(m, det)))
    for name, text in files:
        path = os.path.join(out, name)
        if not os.path.exists(path) or open(path).read() != text:
            with open(path, "w") as f:
                f.write(text)
    print(" ".join(os.path.join(out, n) for n, _ in files))


if __name__ == "__main__":
    main(sys.argv)
