"""The reference's executable end to end (exec/src/inchman/main.cpp:67-160): a model
file in, the reference's HDF5 layout out (inchman_b200.cli), with the same numbers as
the solver run directly on the same model, seed and initial state."""
import os

import numpy as np
import pytest

from inchman_b200 import _lib, cli, h5, sbml
from inchman_b200.solver import Solver

MODELS = os.path.join(os.path.dirname(__file__), "golden", "models")


def _variant(tmp_path, name, runs=None, solver=None):
    text = open(os.path.join(MODELS, name), encoding="utf-8").read()
    if runs is not None:
        old = '<im:runs><math:math xmlns:math="http://www.w3.org/1998/Math/MathML"><math:cn>1</math:cn>'
        assert old in text, name
        text = text.replace(old, old.replace("<math:cn>1</math:cn>", f"<math:cn>{runs}</math:cn>"))
    if solver is not None:
        a = text.index("<im:solver>") + len("<im:solver>")
        b = text.index("</im:solver>")
        text = text[:a] + solver + text[b:]
    p = tmp_path / name
    p.write_text(text, encoding="utf-8")
    return str(p)


@pytest.mark.gpu
@pytest.mark.parametrize("name,runs,solver,override", [
    ("saturating.xml", 3, None, None),
    ("ab_drift.xml", 2, None, ("k2", 0.02)),
    ("ab_drift.xml", 1, "deterministic_inhomogeneous_RK4", None),
])
def test_cli_writes_the_solver_results(gpgmp, tmp_path, name, runs, solver, override):
    path = _variant(tmp_path, name, runs, solver)
    out = str(tmp_path / "out.h5")
    args = [path, "--output", out, "--seed", "11"]
    overrides = {}
    if override:
        args += ["--p", f"{override[0]}={override[1]}"]
        overrides[override[0]] = override[1]
    assert cli.main(args) == 0
    # the same model run directly
    lm = sbml.load(path, overrides=overrides)
    m = lm.model
    det = m.solver in _lib.DETERMINISTIC_TYPES
    R = 1 if det else runs
    init = m.initial_state(np.random.default_rng(11), R)
    with Solver(m, realisations=R, seed=11) as s:
        s.set_state(init.astype(np.float32) if det else init)
        snaps, times, _ = s.solve(max_snapshots=64)
    f = h5.read(out)
    assert f["Model"].attrs["numRuns"].tolist() == [R]
    assert f["Model/Species"].value == [sp.id for sp in m.species]
    assert f["Model/InchmanFile"].value == open(path, encoding="utf-8").read()
    if override:
        assert f["Parameters"].attrs[override[0]].tolist() == [np.float32(override[1])]
    names = []
    for t in times:
        if cli.dump_name(t) not in names:
            names.append(cli.dump_name(t))
    assert sorted(names) == list(f["Runs/0"]) and "Dump_0" in names
    for r in range(R):
        seen = set()
        for k, t in enumerate(times):
            nm = cli.dump_name(t)
            if nm in seen:
                continue                       # a repeated name keeps the first dump
            seen.add(nm)
            d = f[f"Runs/{r}/{nm}"]
            assert d.attrs["time"].tolist() == [t]
            for si, sp in enumerate(m.species):
                v = d[sp.id].value
                assert v.dtype == (np.float32 if det else np.int32)
                assert np.array_equal(v.reshape(-1), snaps[k, r, si].reshape(-1))


@pytest.mark.gpu
def test_cli_writes_individuals(gpgmp, tmp_path):
    """A model file with an individual species: every dump holds the species' list
    (cell | id << 32, the reference's getPositionList) whose cells count exactly the
    dump's counts, with the properties of each listed individual."""
    path = _variant(tmp_path, "individual_a.xml", runs=2)
    out = str(tmp_path / "ind.h5")
    assert cli.main([path, "--output", out, "--seed", "5"]) == 0
    f = h5.read(out)
    lm = sbml.load(path)
    W, H = lm.model.width, lm.model.height
    saw_new = False
    for r in ("0", "1"):
        for name in f[f"Runs/{r}"]:
            d = f[f"Runs/{r}/{name}"]
            counts = d["A"].value.reshape(-1)
            ig = d["Individuals"]
            if counts.sum() == 0:
                assert "A" not in ig
                continue
            pairs = ig["A"].value
            assert pairs.dtype == np.uint64 and len(pairs) == counts.sum()
            cells = (pairs & np.uint64(0xFFFFFFFF)).astype(np.int64)
            ids = (pairs >> np.uint64(32)).astype(np.int64)
            assert np.array_equal(np.bincount(cells, minlength=W * H), counts)
            assert np.all(np.diff(cells) >= 0) and len(np.unique(ids)) == len(ids)
            drift = ig["A.DriftX"].value
            assert len(drift) == len(pairs) and ig["A.DiffusivityY"].value.dtype == np.float32
            assert np.all((drift >= 0) & (drift < 0.2))
            saw_new = saw_new or bool((drift > 0).any())
    assert saw_new                                       # the new-individuals method ran


@pytest.mark.gpu
def test_cli_runs_a_nonlinear_model_one_solver_per_run(gpgmp, tmp_path):
    """A nonlinear drift method (fields recomputed from each run's state after every
    sweep) runs each run in its own solver; the file still holds every run, and
    reflecting walls without reactions keep each run's total."""
    path = _variant(tmp_path, "nonlinear.xml", runs=2)
    out = str(tmp_path / "nl.h5")
    assert cli.main([path, "--output", out, "--seed", "3"]) == 0
    f = h5.read(out)
    assert f["Model"].attrs["numRuns"].tolist() == [2]
    total = 5 * 16 * 12
    finals = []
    for r in ("0", "1"):
        names = list(f[f"Runs/{r}"])
        assert "Dump_0" in names and len(names) >= 3
        for nm in names:
            assert int(f[f"Runs/{r}/{nm}/A"].value.sum()) == total
        last = max(names, key=lambda nm: float(f[f"Runs/{r}/{nm}"].attrs["time"][0]))
        finals.append(f[f"Runs/{r}/{last}/A"].value)
    assert not np.array_equal(finals[0], finals[1])          # two different runs
    # mass left the strip x < 5 it started in (the datasets hold the [y][x] buffer)
    assert finals[0].reshape(16, 16)[:, 5:].sum() > 0


@pytest.mark.gpu
def test_cli_writes_field_parameters(gpgmp, tmp_path):
    """A model with a field parameter that its setField method accumulates: every dump
    has a Fields group; the field starts at zero and grows where A is."""
    path = _variant(tmp_path, "field_trace.xml", runs=2)
    out = str(tmp_path / "f.h5")
    assert cli.main([path, "--output", out, "--seed", "9"]) == 0
    f = h5.read(out)
    for r in ("0", "1"):
        by_time = sorted(f[f"Runs/{r}"], key=lambda nm: float(f[f"Runs/{r}/{nm}"].attrs["time"][0]))
        tr = [f[f"Runs/{r}/{nm}/Fields/trace"].value for nm in by_time]
        assert tr[0].dtype == np.float32 and tr[0].shape == (12, 12)
        assert np.all(tr[0] == 0)
        assert np.all(np.diff(np.stack(tr).reshape(len(tr), -1), axis=0) >= 0)
        assert tr[-1].sum() > 0
