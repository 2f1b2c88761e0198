"""maxwellfdtd_b200 -- B200-native time-stepper for the MaxwellFDTD finite-difference
time-domain method.

The Python API mirrors the reference's Julia API (Grid, Material, sources, CPML, monitors,
Model, solve!).  The time-step path itself runs in libmaxwellfdtd_b200.so, hand-written
CUDA for sm_100a behind the C ABI in include/maxwellfdtd.h.
"""
from .constants import C0, EPS0, HBAR, ME, MU0, QE
from .geometry import Ball, Box, Cylinder, Ellipsoid, Everywhere, HalfSpace, Shape
from .grids import Grid1D, Grid2D, Grid3D, make_grid as Grid
from .materials import (DebyeSusceptibility, DrudeSusceptibility, IonizationRate, LorentzSusceptibility,
                        Material, Plasma, PowerLawRate, susceptibility)
from .model import B200, Model, Solution, load_library, library_path, solve
from .monitors import FieldMonitor, SpectralMonitor
from .pml import CPML
from .sources import HardSource, SeparableWaveform, SoftSource, TFSFSource

solve_ = solve   # Julia's solve! spelling is not a Python identifier

__all__ = [
    "C0", "EPS0", "MU0", "QE", "ME", "HBAR",
    "Grid", "Grid1D", "Grid2D", "Grid3D",
    "Shape", "Ball", "Box", "Ellipsoid", "Cylinder", "HalfSpace", "Everywhere",
    "Material", "Plasma", "DebyeSusceptibility", "DrudeSusceptibility", "LorentzSusceptibility",
    "PowerLawRate", "IonizationRate", "susceptibility",
    "CPML", "SoftSource", "HardSource", "TFSFSource", "SeparableWaveform",
    "FieldMonitor", "SpectralMonitor",
    "Model", "solve", "Solution", "B200", "load_library", "library_path",
]
