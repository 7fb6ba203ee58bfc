"""Shared builders for the tests."""
import numpy as np

from inchman_b200 import _lib
from inchman_b200.model import DiffusionModel


def small_homog(W=12, H=10, max_time=0.5, bmask=(0, 0, 0, 0), source=(0, 0, 0, 0)):
    m = DiffusionModel(width=W, height=H, physical_length=float(W), p0=0.1, max_time=max_time, output_interval=0.2,
                       boundary_mask=bmask, source_mask=source, solver=_lib.STOCHASTIC_HOMOGENEOUS)
    m.add_species("A", 1.0, 60.0).add_species("B", 1.0, 40.0).add_species("C", 0.5, 5.0)
    m.add_reaction("bind", {"A": 1, "B": 1}, {"C": 1}, 0.01)
    m.add_reaction("unbind", {"C": 1}, {"A": 1, "B": 1}, 0.1)
    return m


def small_inhom(W=16, H=16, max_time=0.3, seed=7):
    m = DiffusionModel(width=W, height=H, physical_length=float(W), p0=0.1, max_time=max_time, output_interval=0.1,
                       solver=_lib.STOCHASTIC_INHOMOGENEOUS, drift_method=_lib.DRIFT_FIELD)
    m.add_species("X", 1.0, 50.0).add_species("Y", 1.0, 50.0)
    m.add_reaction("birth", {"X": 1}, {"X": 2}, 1.0)
    m.add_reaction("predation", {"X": 1, "Y": 1}, {"Y": 2}, 0.005)
    m.add_reaction("death", {"Y": 1}, {}, 0.6)
    rng = np.random.Generator(np.random.PCG64(seed))
    D = rng.lognormal(0.0, 0.5, size=(H, W)).astype(np.float32)
    y, x = np.meshgrid(np.arange(H, dtype=np.float64), np.arange(W, dtype=np.float64), indexing="ij")
    rx = (0.3 * np.sin(2 * np.pi * y / W)).astype(np.float32)
    ry = (0.3 * np.cos(2 * np.pi * x / W)).astype(np.float32)
    m.field_dx = np.stack([D, D]); m.field_dy = np.stack([D, D])
    m.field_rx = np.stack([rx, rx]); m.field_ry = np.stack([ry, ry])
    return m
