"""B200-native FDTD Maxwell engine with the jaxphys (``neurosim``) FDTD API.

Import surface of the reference's FDTD path (``src/neurosim/__init__.py:60-62``,
``src/neurosim/em/__init__.py:6-21``): ``EMGrid``, ``PlaneWave``, ``Wall``,
``EMGrid3D``, ``PointSource3D``, ``DielectricRegion``, ``EMConfig``, the
exception classes and the history containers.  The solvers run as sm_100a
CUDA kernels behind the C ABI in ``include/jaxphys_fdtd.h``.
"""

from .config import EMConfig
from .em import (
    FDTD2D,
    FDTD3D,
    CPMLSpec,
    DielectricRegion,
    EMGrid,
    EMGrid3D,
    PlaneWave,
    PointSource3D,
    Wall,
)
from .exceptions import (
    ConfigurationError,
    ConvergenceError,
    DimensionError,
    NeurosimError,
    NumericalInstabilityError,
    PhysicsError,
    SimulationError,
    VisualizationError,
)
from .state import EMFieldHistory, EMFieldHistory3D

__version__ = "0.1.0"

__all__ = [
    "EMConfig",
    "EMGrid",
    "PlaneWave",
    "Wall",
    "FDTD2D",
    "EMGrid3D",
    "PointSource3D",
    "DielectricRegion",
    "CPMLSpec",
    "FDTD3D",
    "EMFieldHistory",
    "EMFieldHistory3D",
    "NeurosimError",
    "SimulationError",
    "NumericalInstabilityError",
    "ConfigurationError",
    "DimensionError",
    "PhysicsError",
    "ConvergenceError",
    "VisualizationError",
]
