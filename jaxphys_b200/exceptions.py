"""Exception hierarchy of the drop-in API.

Same classes, base classes and meaning as the reference's
``src/neurosim/exceptions.py:8-45``, so ``except ConfigurationError`` clauses
written against jaxphys keep working.
"""


class NeurosimError(Exception):
    """Base exception for all errors raised by this package."""


class SimulationError(NeurosimError):
    """A simulation failed: a device call returned an error status."""


class NumericalInstabilityError(SimulationError):
    """Fields became NaN / Inf (for example a time step above the CFL limit)."""


class ConfigurationError(NeurosimError):
    """Simulation parameters are invalid or inconsistent."""


class DimensionError(NeurosimError):
    """Array dimensions are incompatible."""


class PhysicsError(NeurosimError):
    """A physical constraint is violated."""


class ConvergenceError(SimulationError):
    """An iterative solver failed to converge."""


class VisualizationError(NeurosimError):
    """Visualisation failed."""
