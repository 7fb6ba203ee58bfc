"""Model description of the hot path's input (species, mass-action reactions,
compartments, diffusion and drift fields).

Mirrors the reference's model classes and builders:
  Species            exec/src/gpgmp/src/Species.h:23 (id, diffusion constant)
  Reaction           Reaction.h:31-211 (reactant/product stoichiometry maps, rate)
  Compartment        Compartment.h:29-43 (inclusive rectangle, initial amount and
                     distribution Homogeneous / Random / LinearX)
  DiffusionModel     DiffusionModel.h: grid, physical length, p0, boundary and
                     source masks, solver type, drift/diffusivity method,
                     addSpecies/addReaction/addCompartment (DiffusionModel.cpp:426-493)
and turns it into the gpgmp_model_desc of the C ABI.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from . import _lib


@dataclass
class Species:
    id: str
    diffusion: float = 0.0
    initial: float = 0.0          # mean initial count per cell (Poisson) or amount
    individual: bool = False      # molecules tracked one by one (IndividualSolver)


@dataclass
class Reaction:
    id: str
    reactants: Dict[str, int]
    products: Dict[str, int]
    rate: float
    # localisation (Reaction::addCompartment, Reaction.cpp:209-235): inclusive
    # rectangles (x0, y0, x1, y1); the reaction fires only in cells inside one of them.
    # Empty: everywhere.
    regions: List[tuple] = field(default_factory=list)


@dataclass
class Compartment:
    """Inclusive rectangle [x0, x1] x [y0, y1] with an initial amount of one species.

    distribution (DiffusionModel.cpp:568-723): "homogeneous" spreads the amount
    evenly, amount // area per cell plus one more in the cells whose grid offset
    y*width + x is below amount % area (the reference's rule); "random" places each
    particle in a uniformly chosen cell; "linearx" a ramp in x with slope
    2 amount / ((nx - 1) nx ny), nx = x1 - x0, ny = y1 - y0, rounded half away from 0."""
    species: str
    x0: int
    y0: int
    x1: int
    y1: int
    amount: float
    distribution: str = "homogeneous"


@dataclass
class DiffusionModel:
    width: int = 32
    height: int = 32
    physical_length: float = 40.0
    p0: float = 0.1
    max_time: float = 1.0
    output_interval: float = 1.0
    max_steps: int = -1
    boundary_mask: tuple = (0, 0, 0, 0)
    source_mask: tuple = (0, 0, 0, 0)
    solver: int = _lib.STOCHASTIC_HOMOGENEOUS
    drift_method: int = _lib.DRIFT_HOMOGENEOUS
    drift_params: tuple = (0.0,) * 8
    flags: int = 0
    species: List[Species] = field(default_factory=list)
    reactions: List[Reaction] = field(default_factory=list)
    compartments: List[Compartment] = field(default_factory=list)
    field_dx: Optional[np.ndarray] = None
    field_dy: Optional[np.ndarray] = None
    field_rx: Optional[np.ndarray] = None
    field_ry: Optional[np.ndarray] = None
    # model code compiled at run time (gpgmp_model_desc.code_defines / drift_code /
    # custom_laws): parameter defines, the drift/diffusivity method for
    # DRIFT_CODE, and per reaction a C propensity expression in X(i) or None
    code_defines: Optional[str] = None
    drift_code: Optional[str] = None
    custom_laws: Optional[List[Optional[str]]] = None
    # individual species (gpgmp_model_desc.individual_capacity / new_individuals_code)
    individual_capacity: int = 0
    new_individuals_code: Optional[str] = None
    # field parameters: names (code reads field f as F(f); code_defines name them),
    # initial values [F][H][W] (None: zeros) and the setField method
    field_names: List[str] = field(default_factory=list)
    field_values: Optional[np.ndarray] = None
    set_field_code: Optional[str] = None

    # -- builders (DiffusionModel.cpp:426-493) --------------------------------
    def add_species(self, id: str, diffusion: float = 0.0, initial: float = 0.0,
                    individual: bool = False) -> "DiffusionModel":
        self.species.append(Species(id, diffusion, initial, individual))
        return self

    def add_reaction(self, id: str, reactants: Dict[str, int], products: Dict[str, int], rate: float,
                     regions=None):
        """regions: inclusive rectangles (x0, y0, x1, y1) the reaction is localised to
        (its compartments), or None for everywhere."""
        self.reactions.append(Reaction(id, dict(reactants), dict(products), rate,
                                       [tuple(int(v) for v in r) for r in (regions or [])]))
        return self

    def reaction_mask(self) -> Optional[np.ndarray]:
        """[R][H][W] uint8, 1 where each reaction may fire (the reference's
        reactionMask: inside one of its compartments, or everywhere if it has none);
        None when every reaction may fire in every cell (no reaction localised, or
        localised to compartments that cover the grid)."""
        if not any(r.regions for r in self.reactions):
            return None
        mask = np.zeros((len(self.reactions), self.height, self.width), dtype=np.uint8)
        for k, r in enumerate(self.reactions):
            if not r.regions:
                mask[k] = 1
            for (x0, y0, x1, y1) in r.regions:
                mask[k, max(y0, 0):y1 + 1, max(x0, 0):x1 + 1] = 1
        return None if mask.all() else mask

    def add_compartment(self, comp: Compartment):
        self.compartments.append(comp)
        return self

    def species_index(self, sid: str) -> int:
        for i, s in enumerate(self.species):
            if s.id == sid:
                return i
        raise KeyError(sid)

    @property
    def num_species(self) -> int:
        return len(self.species)

    @property
    def area(self) -> int:
        return self.width * self.height

    def cell_width(self) -> float:
        return float(np.float32(self.physical_length) / np.float32(self.width))

    # -- C ABI ------------------------------------------------------------------
    def reaction_array(self):
        arr = (_lib.Reaction * max(1, len(self.reactions)))()
        for k, r in enumerate(self.reactions):
            rc = arr[k]
            rc.rate = r.rate
            if len(r.reactants) > 3 or len(r.products) > 4:
                raise ValueError(f"reaction {r.id}: at most 3 reactant and 4 product species")
            rc.num_reactants = len(r.reactants)
            for j, (sid, st) in enumerate(r.reactants.items()):
                rc.reactant_species[j] = self.species_index(sid)
                rc.reactant_stoich[j] = int(st)
            rc.num_products = len(r.products)
            for j, (sid, st) in enumerate(r.products.items()):
                rc.product_species[j] = self.species_index(sid)
                rc.product_stoich[j] = int(st)
        return arr

    def to_desc(self):
        """Returns (desc, keepalive): keepalive holds the arrays desc points into."""
        d = _lib.ModelDesc()
        d.width, d.height = self.width, self.height
        d.num_species, d.num_reactions = len(self.species), len(self.reactions)
        d.physical_length, d.p0 = self.physical_length, self.p0
        d.max_time, d.output_interval = self.max_time, self.output_interval
        d.max_steps = self.max_steps
        for i in range(4):
            d.boundary_mask[i] = int(self.boundary_mask[i])
            d.source_mask[i] = int(self.source_mask[i])
        d.solver_type = self.solver
        d.drift_method = self.drift_method
        d.flags = self.flags
        for i, v in enumerate(list(self.drift_params)[:8]):
            d.drift_params[i] = v
        diff = np.ascontiguousarray([s.diffusion for s in self.species], dtype=np.float32)
        rx = self.reaction_array()
        keep = [diff, rx]
        d.diffusion = diff.ctypes.data_as(C.POINTER(C.c_float))
        d.reactions = C.cast(rx, C.POINTER(_lib.Reaction))
        for name in ("field_dx", "field_dy", "field_rx", "field_ry"):
            arr = getattr(self, name)
            if arr is not None:
                a = np.ascontiguousarray(arr, dtype=np.float32).reshape(-1)
                if a.size != self.num_species * self.area:
                    raise ValueError(f"{name} must hold [species][height][width] values")
                keep.append(a)
                setattr(d, name, a.ctypes.data_as(C.POINTER(C.c_float)))
        if self.code_defines:
            b = self.code_defines.encode()
            keep.append(b)
            d.code_defines = b
        if self.drift_code is not None:
            b = self.drift_code.encode()
            keep.append(b)
            d.drift_code = b
        if any(sp.individual for sp in self.species):
            flags = np.ascontiguousarray([1 if sp.individual else 0 for sp in self.species], dtype=np.uint8)
            keep.append(flags)
            d.individual = flags.ctypes.data_as(C.POINTER(C.c_uint8))
            d.individual_capacity = int(self.individual_capacity)
            if self.new_individuals_code:
                b = self.new_individuals_code.encode()
                keep.append(b)
                d.new_individuals_code = b
        if self.field_names:
            d.num_fields = len(self.field_names)
            if self.field_values is not None:
                fv = np.ascontiguousarray(self.field_values, dtype=np.float32).reshape(-1)
                if fv.size != len(self.field_names) * self.area:
                    raise ValueError("field_values must hold [fields][height][width] values")
                keep.append(fv)
                d.field_values = fv.ctypes.data_as(C.POINTER(C.c_float))
            if self.set_field_code:
                b = self.set_field_code.encode()
                keep.append(b)
                d.set_field_code = b
        rm = self.reaction_mask()
        if rm is not None:
            rm = np.ascontiguousarray(rm).reshape(-1)
            keep.append(rm)
            d.reaction_mask = rm.ctypes.data_as(C.POINTER(C.c_uint8))
        if self.custom_laws is not None:
            if len(self.custom_laws) != len(self.reactions):
                raise ValueError("custom_laws needs one entry (or None) per reaction")
            laws = (C.c_char_p * max(1, len(self.reactions)))(*[(l.encode() if l else None) for l in self.custom_laws])
            keep.append(laws)
            d.custom_laws = C.cast(laws, C.POINTER(C.c_char_p))
        return d, keep

    # -- initial state (DiffusionModel.cpp:568-723) ------------------------------
    def initial_state(self, rng: np.random.Generator, realisations: int = 1) -> np.ndarray:
        """Host-side initial counts from the compartments, [R][S][H][W] int32."""
        S, H, W = self.num_species, self.height, self.width
        out = np.zeros((realisations, S, H, W), dtype=np.int32)
        for r in range(realisations):
            for comp in self.compartments:
                s = self.species_index(comp.species)
                ys, xs = slice(comp.y0, comp.y1 + 1), slice(comp.x0, comp.x1 + 1)
                ncell = (comp.y1 - comp.y0 + 1) * (comp.x1 - comp.x0 + 1)
                amount = int(comp.amount)
                if comp.distribution == "homogeneous":
                    per, rem = divmod(amount, ncell)
                    yy, xx = np.mgrid[comp.y0:comp.y1 + 1, comp.x0:comp.x1 + 1]
                    out[r, s, ys, xs] += (per + ((yy * W + xx) < rem)).astype(np.int32)
                elif comp.distribution == "random":
                    cells = rng.integers(0, ncell, size=amount)
                    counts = np.bincount(cells, minlength=ncell).reshape(comp.y1 - comp.y0 + 1, -1)
                    out[r, s, ys, xs] += counts.astype(np.int32)
                elif comp.distribution == "linearx":
                    nx, ny = comp.x1 - comp.x0, comp.y1 - comp.y0
                    if nx < 2 or ny < 1:
                        raise ValueError("linearx needs a compartment at least 3 wide and 2 high")
                    coeff = np.float32(2.0 * amount / ((nx - 1) * nx * ny))
                    v = coeff * np.arange(comp.x1 - comp.x0 + 1, dtype=np.float32)
                    ramp = (np.sign(v) * np.floor(np.abs(v) + 0.5)).astype(np.int32)
                    out[r, s, ys, xs] += ramp[None, :]
                else:
                    raise ValueError(comp.distribution)
        return out


# ---------------------------------------------------------------------------
# The benchmark workloads (synthetic, seeded).
# ---------------------------------------------------------------------------

def plain_ssa_model(width: int = 32, max_time: float = 10.0) -> DiffusionModel:
    """A+B->C (k1=0.01), C->A+B (k2=0.1) on a reflecting width x width grid,
    D = (1, 1, 0.5), h = 1, p0 = 0.1, snapshots every 1.0; A,B ~ Poisson(100)."""
    m = DiffusionModel(width=width, height=width, physical_length=float(width), p0=0.1, max_time=max_time,
                       output_interval=1.0, solver=_lib.STOCHASTIC_HOMOGENEOUS)
    m.add_species("A", 1.0, 100.0).add_species("B", 1.0, 100.0).add_species("C", 0.5, 0.0)
    m.add_reaction("bind", {"A": 1, "B": 1}, {"C": 1}, 0.01)
    m.add_reaction("unbind", {"C": 1}, {"A": 1, "B": 1}, 0.1)
    return m


def lotka_volterra_model(width: int = 512, max_time: float = 50.0, seed: int = 1234) -> DiffusionModel:
    """X->2X (1.0), X+Y->2Y (0.005), Y->0 (0.6) with per-cell lognormal(0, 0.5)
    diffusivity (shared by X and Y, isotropic) and drift
    r = 0.3 (sin(2 pi y / width), cos(2 pi x / width)); reflecting walls, h = 1.
    X, Y ~ Poisson(50)."""
    m = DiffusionModel(width=width, height=width, physical_length=float(width), p0=0.1, max_time=max_time,
                       output_interval=1.0, solver=_lib.STOCHASTIC_INHOMOGENEOUS, drift_method=_lib.DRIFT_FIELD)
    m.add_species("X", 1.0, 50.0).add_species("Y", 1.0, 50.0)
    m.add_reaction("birth", {"X": 1}, {"X": 2}, 1.0)
    m.add_reaction("predation", {"X": 1, "Y": 1}, {"Y": 2}, 0.005)
    m.add_reaction("death", {"Y": 1}, {}, 0.6)
    rng = np.random.Generator(np.random.PCG64(seed))
    D = rng.lognormal(0.0, 0.5, size=(width, width)).astype(np.float32)
    y, x = np.meshgrid(np.arange(width, dtype=np.float64), np.arange(width, dtype=np.float64), indexing="ij")
    rx = (0.3 * np.sin(2 * np.pi * y / width)).astype(np.float32)
    ry = (0.3 * np.cos(2 * np.pi * x / width)).astype(np.float32)
    m.field_dx = np.stack([D, D])
    m.field_dy = np.stack([D, D])
    m.field_rx = np.stack([rx, rx])
    m.field_ry = np.stack([ry, ry])
    return m
