"""Exception hierarchy under the reference's module path
(``src/neurosim/exceptions.py``)."""

from jaxphys_b200.exceptions import (  # noqa: F401
    ConfigurationError,
    ConvergenceError,
    DimensionError,
    NeurosimError,
    NumericalInstabilityError,
    PhysicsError,
    SimulationError,
    VisualizationError,
)
