"""Electromagnetism: the FDTD Maxwell solvers (2D and 3D) and waveguide
analysis under the reference's import path (``src/neurosim/em/__init__.py``).
The reference's point-charge N-body integrator (``ChargeSystem``,
``PointCharge``) is not part of this engine."""

from .fdtd import EMGrid, PlaneWave, Wall
from .fdtd3d import DielectricRegion, EMGrid3D, PointSource3D
from .waveguides import RectangularWaveguide

__all__ = [
    "EMGrid",
    "PlaneWave",
    "Wall",
    "EMGrid3D",
    "PointSource3D",
    "DielectricRegion",
    "RectangularWaveguide",
]
