"""Electromagnetism: the FDTD Maxwell solvers (2D TM and 3D), waveguide mode ports and
moving-charge current sources."""

from .fdtd import FDTD2D, EMGrid, PlaneWave, Wall
from .fdtd3d import FDTD3D, CPMLSpec, DielectricRegion, EMGrid3D, PointSource3D
from .waveguides import ModeSource3D, RectangularWaveguide, WaveguideMode
from .charges import MovingCharge3D, charges_from_trajectory

__all__ = [
    "EMGrid",
    "PlaneWave",
    "Wall",
    "FDTD2D",
    "EMGrid3D",
    "PointSource3D",
    "DielectricRegion",
    "CPMLSpec",
    "FDTD3D",
    "RectangularWaveguide",
    "WaveguideMode",
    "ModeSource3D",
    "MovingCharge3D",
    "charges_from_trajectory",
]
