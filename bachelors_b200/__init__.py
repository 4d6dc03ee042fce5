"""B200-native fast-multipole Biot-Savart solver (sm_100a), a drop-in for the FMM path of
iamwhoamianamy/bachelors. The compute path is libfmmcuda.so (include/fmmcuda.h); this package
is its Python host side."""
from . import geometry
from ._lib import FmmError, load as load_library
from .solver import (Device, FastMultipoleSolver, M2LAlg, M2MAlg, MultipoleSolver, Plan, Problem,
                     calcBioSavartLaplace)

__all__ = ["geometry", "FmmError", "load_library", "Device", "FastMultipoleSolver", "M2LAlg", "M2MAlg",
           "MultipoleSolver", "Plan", "Problem", "calcBioSavartLaplace"]
