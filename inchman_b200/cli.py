"""The reference's executable (exec/src/inchman/main.cpp:67-160) on the B200 solvers:

    python -m inchman_b200.cli [--output FILE] [--p NAME=VALUE]... [--seed N] model.xml

loads an annotated-SBML model file (inchman_b200.sbml), runs it -- every run of a
stochastic model as one realisation of one wide solver, a deterministic model once --
and writes the reference's HDF5 layout (DiffusionModel.cpp:934-1296,
InchmanDiffusionModel.cpp:240-274, doc/source/hdf5.rst) with inchman_b200.h5:

  /Model                      attributes numSpecies, numRuns (int32[1])
  /Model/Species              variable-length strings, the species ids in order
  /Model/InchmanFile          the model file's text (fixed-length string)
  /Model/Compartments/<id>    int32[4]: x0, y0, x1, y1 (inclusive)
  /Parameters                 one float32[1] attribute per parameter (after --p)
  /Runs/<run>/Dump_<time>     attribute time (float32[1]); one dataset per species,
                              dims [gridWidth, gridHeight] over the state buffer
                              (int32 counts, float32 for deterministic solvers);
                              a Fields group with the field parameters (when the
                              model has them); an Individuals group: per individual
                              species its
                              (cell | id << 32) uint64 list and four float32
                              property lists (empty without individual species)

Dumps are named by the time printed with 9 significant digits (the reference's
boost::lexical_cast of a float): Dump_0, Dump_1, Dump_0.100000001, ...  They are taken
where the reference writes them: the initial state, every output interval, and the
final state (a dump whose name exists already is not written again, as
H5Gcreate2 fails on it).

Options as the reference's: --output (default output.h5), --p name=value (repeatable),
--cl-source and --wait-on-exit (accepted; there are no OpenCL sources to point at).
Added: --seed (the reference seeds from the clock; default here too) and
--ignore-scripts (run a model whose Python init/event scripts are not supported,
without them).
"""
from __future__ import annotations

import argparse
import sys
import time
from typing import Dict, Optional

import numpy as np

from . import _lib, h5, sbml


def dump_name(t: float) -> str:
    return "Dump_" + ("%.9g" % float(np.float32(t)))


PROPERTY_NAMES = ("DiffusivityX", "DiffusivityY", "DriftX", "DriftY")


def output_tree(lm: sbml.LoadedModel, snaps: np.ndarray, times: np.ndarray, individuals=None,
                fields=None) -> h5.Group:
    """The reference's file layout for snapshots [n][runs][S][H][W] at times [n].
    individuals[k][species] = (keys, ids, props [4][n]) of dump k (keys r * area + cell):
    written per run as /Individuals/<species> (uint64 cell | id << 32, the reference's
    getPositionList) and <species>.DiffusivityX/Y, .DriftX/Y (float32, in the same
    order as the positions).  fields[k] = [runs][F][H][W] field parameters of dump k,
    written as /Fields/<name> (float32, dims [gridWidth, gridHeight])."""
    m = lm.model
    S, H, W = m.num_species, m.height, m.width
    runs = snaps.shape[1]
    root = h5.Group()
    model_g = root.create_group("Model")
    model_g.attrs["numSpecies"] = np.array([S], np.int32)
    model_g.attrs["numRuns"] = np.array([runs], np.int32)
    model_g.create_dataset("Species", [s.id for s in m.species])
    comp_g = model_g.create_group("Compartments")
    for cid, (x0, y0, x1, y1) in lm.compartments.items():
        comp_g.create_dataset(cid, np.array([x0, y0, x1, y1], np.int32))
    model_g.create_dataset("InchmanFile", lm.source)
    par_g = root.create_group("Parameters")
    for k in sorted(lm.parameters):
        par_g.attrs[k] = np.array([lm.parameters[k]], np.float32)
    runs_g = root.create_group("Runs")
    for r in range(runs):
        run_g = runs_g.create_group(str(r))
        for k in range(snaps.shape[0]):
            name = dump_name(times[k])
            if name in run_g:
                continue
            d = run_g.create_group(name)
            d.attrs["time"] = np.array([times[k]], np.float32)
            for s, sp in enumerate(m.species):
                # the state buffer of one species as the reference hands it to HDF5:
                # dims [gridWidth, gridHeight] over the bytes of the [H][W] plane
                d.create_dataset(sp.id, np.ascontiguousarray(snaps[k, r, s]).reshape(W, H))
            if fields is not None and m.field_names:
                fg = d.create_group("Fields")
                for f, fname in enumerate(m.field_names):
                    fg.create_dataset(fname, np.ascontiguousarray(fields[k][r][f]).reshape(W, H))
            ig = d.create_group("Individuals")
            if individuals is None:
                continue
            area = W * H
            for s_idx, (keys, ids, props) in individuals[k].items():
                sel = (keys // area) == r
                if not sel.any():
                    continue
                sid = m.species[s_idx].id
                pairs = (keys[sel] % area).astype(np.uint64) | (ids[sel].astype(np.uint64) << np.uint64(32))
                ig.create_dataset(sid, pairs)
                for q, pname in enumerate(PROPERTY_NAMES):
                    ig.create_dataset(f"{sid}.{pname}", np.ascontiguousarray(props[q][sel], dtype=np.float32))
    return root


def run(lm: sbml.LoadedModel, seed: int):
    """Runs the model; returns (snapshots [n][runs][S][H][W], times [n], steps,
    individuals per dump or None, fields per dump [runs][F][H][W] or None)."""
    from .solver import Solver
    m = lm.model
    det = m.solver in _lib.DETERMINISTIC_TYPES
    R = 1 if det else max(1, int(lm.runs))
    state = m.initial_state(np.random.default_rng(seed), R)
    if det:
        state = state.astype(np.float32)
    if m.output_interval > 0:
        nmax = int(np.floor(m.max_time / m.output_interval)) + 4
    else:
        nmax = 4
    if R > 1 and ((m.flags & _lib.FLAG_NONLINEAR) or m.set_field_code):
        # a nonlinear method's fields follow each run's state: one solver per run
        parts = []
        for r in range(R):
            one = sbml.LoadedModel(model=m, runs=1, parameters=lm.parameters, notes=lm.notes,
                                   compartments=lm.compartments, source=lm.source)
            parts.append(run(one, seed + r))
        n = min(len(p[1]) for p in parts)
        snaps = np.concatenate([p[0][:n] for p in parts], axis=1)
        inds = None
        if parts[0][3] is not None:
            area = m.width * m.height
            inds = []
            for k in range(n):
                merged = {}
                for r, p in enumerate(parts):
                    for sp, (keys, ids, props) in p[3][k].items():
                        prev = merged.get(sp)
                        kk = keys + np.uint32(r * area)
                        merged[sp] = (kk, ids, props) if prev is None else (
                            np.concatenate([prev[0], kk]), np.concatenate([prev[1], ids]),
                            np.concatenate([prev[2], props], axis=1))
                inds.append(merged)
        flds = None
        if parts[0][4] is not None:
            flds = [np.concatenate([p[4][k] for p in parts], axis=0) for k in range(n)]
        return snaps, parts[0][1][:n], sum(p[2] for p in parts), inds, flds
    ind_species = [i for i, sp in enumerate(m.species) if sp.individual]
    individuals, fields = [], []
    with Solver(m, realisations=R, seed=seed) as s:
        s.set_state(state)
        if ind_species or m.field_names:
            def on_dump(index, t):
                if ind_species:
                    individuals.append({i: s.get_individuals(i) for i in ind_species})
                if m.field_names:   # shared by the solver's realisations (no setField with R > 1)
                    fields.append(np.repeat(s.get_fields()[None], R, axis=0))
            snaps, times, steps = s.solve(max_snapshots=nmax, on_dump=on_dump)
        else:
            snaps, times, steps = s.solve(max_snapshots=nmax)
    return (snaps, times, steps, (individuals[:len(times)] if ind_species else None),
            (fields[:len(times)] if m.field_names else None))


def main(argv: Optional[list] = None) -> int:
    ap = argparse.ArgumentParser(prog="inchman", description="Run an Inchman model file on the GPU.")
    ap.add_argument("model_file")
    ap.add_argument("--output", default="output.h5", help='output filename (default: "output.h5")')
    ap.add_argument("--p", action="append", default=[], metavar="NAME=VALUE", help="override a parameter value")
    ap.add_argument("--cl-source", default=None, help="accepted for compatibility; unused")
    ap.add_argument("--wait-on-exit", action="store_true", help="accepted for compatibility; unused")
    ap.add_argument("--seed", type=int, default=None, help="random seed (default: from the clock)")
    ap.add_argument("--ignore-scripts", action="store_true", help="run without the model's init/event scripts")
    args = ap.parse_args(argv)
    overrides: Dict[str, float] = {}
    for kv in args.p:
        if "=" not in kv:
            ap.error(f"--p expects NAME=VALUE, got {kv!r}")
        k, v = kv.split("=", 1)
        overrides[k.strip()] = float(v)
    seed = args.seed if args.seed is not None else int(time.time())
    try:
        lm = sbml.load(args.model_file, ignore_scripts=args.ignore_scripts, overrides=overrides)
    except sbml.Unsupported as e:
        print(f"Error: {e}", file=sys.stderr)
        return 1
    for n in lm.notes:
        print(f"note: {n}", file=sys.stderr)
    t0 = time.perf_counter()
    snaps, times, steps, individuals, fields = run(lm, seed)
    t1 = time.perf_counter()
    h5.write(args.output, output_tree(lm, snaps, times, individuals, fields))
    print(f"{args.model_file}: {snaps.shape[1]} run(s), {len(times)} dumps, {steps} steps in {t1 - t0:.3f} s "
          f"-> {args.output}", file=sys.stderr)
    return 0


if __name__ == "__main__":
    sys.exit(main())
