"""``neurosim`` import surface of the FDTD path, served by the B200 engine.

The reference package ``neurosim`` (jaxphys) exposes its FDTD solvers as
``neurosim.EMGrid3D`` / ``neurosim.em.fdtd3d.EMGrid3D`` and so on
(``src/neurosim/__init__.py:60-62``, ``src/neurosim/em/__init__.py:6-21``).
This package keeps those import paths, so code written against the
reference runs unchanged on the CUDA engine in ``jaxphys_b200``:

    from neurosim.em.fdtd3d import EMGrid3D, PointSource3D

Differences from ``jaxphys_b200``: ``simulate()`` returns JAX arrays (through
DLPack) by default when JAX is importable, as the reference does, and torch
tensors otherwise.  Only the FDTD path and what is built around it are here
(solvers, results, exceptions, ``EMConfig``, waveguide analysis,
``optimize``/``sensitivity``, field viewers); the reference's mechanics,
fluids, quantum, statistical-mechanics and optics modules are not part of
this engine.
"""

from __future__ import annotations

try:  # the reference enables 64-bit JAX on import (src/neurosim/__init__.py:22-24)
    import jax as _jax

    _jax.config.update("jax_enable_x64", True)
except Exception:  # JAX is optional here
    _jax = None

from jaxphys_b200.config import EMConfig
from jaxphys_b200.exceptions import (
    ConfigurationError,
    ConvergenceError,
    DimensionError,
    NeurosimError,
    NumericalInstabilityError,
    PhysicsError,
    SimulationError,
    VisualizationError,
)
from jaxphys_b200.optimize import optimize, sensitivity
from jaxphys_b200.state import EMFieldHistory, EMFieldHistory3D

from .em import (
    DielectricRegion,
    EMGrid,
    EMGrid3D,
    PlaneWave,
    PointSource3D,
    RectangularWaveguide,
    Wall,
)

__version__ = "0.1.0"

__all__ = [
    "EMConfig",
    "EMGrid",
    "PlaneWave",
    "Wall",
    "EMGrid3D",
    "PointSource3D",
    "DielectricRegion",
    "RectangularWaveguide",
    "EMFieldHistory",
    "EMFieldHistory3D",
    "optimize",
    "sensitivity",
    "NeurosimError",
    "SimulationError",
    "NumericalInstabilityError",
    "ConfigurationError",
    "DimensionError",
    "PhysicsError",
    "ConvergenceError",
    "VisualizationError",
]
