"""B200-native Trotter-Suzuki evolution, a drop-in for trotter-suzuki-mpi's evolution path.

High level (same names as the reference's Python package):
    Lattice1D, Lattice2D, State, GaussianState, ExponentialState, SinusoidState,
    Potential, HarmonicPotential, Hamiltonian, Solver, map_lattice_to_coordinate_space
    DevicePotential -- a time-dependent V(x, y, t) evaluated with torch on the GPU.
Low level: Kernel -- one lattice tile on the GPU through the C ABI of include/ts_b200.h;
Batch -- many Kernel tiles of uneven sizes advanced by one persistent launch per step.
"""
from ._capi import B200Error, Desc, EnergyParams  # noqa: F401
from .api import (DevicePotential, ExponentialState, GaussianState, Hamiltonian,  # noqa: F401
                  Hamiltonian2Component,
                  HarmonicPotential, Lattice1D, Lattice2D, Potential, SinusoidState, Solver,
                  SolverBatch, State, make_desc, map_lattice_to_coordinate_space)
from .kernel import FP32, FP64, Batch, Kernel, Pair, launch_count, version  # noqa: F401

__version__ = "1.6.2+b200"

__all__ = ["Lattice1D", "Lattice2D", "State", "ExponentialState", "GaussianState",
           "SinusoidState", "Potential", "DevicePotential", "HarmonicPotential", "Hamiltonian",
           "Hamiltonian2Component", "Solver", "SolverBatch", "map_lattice_to_coordinate_space",
           "Kernel", "Batch", "Pair",
           "B200Error"]
