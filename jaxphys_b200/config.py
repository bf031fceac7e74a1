"""EMConfig, the validated 2D FDTD configuration.

Same fields, defaults and validation as the reference's ``EMConfig``
(``src/neurosim/config.py:96-110``).  As in the reference, ``courant_number``
is validated and stored but the 2D time step is fixed by the CFL formula
``0.99*dx/(c*sqrt(2))`` (``src/neurosim/em/fdtd.py:214``).
"""

from typing import Literal

from pydantic import BaseModel, Field


class EMConfig(BaseModel):
    """Configuration for electromagnetic FDTD simulations.

    Attributes:
        resolution: Spatial grid resolution (cell size in meters).
        courant_number: Courant-Friedrichs-Lewy number, in (0, 1].
        boundary: Boundary condition type.
        pml_layers: Number of PML absorbing layers at boundaries.
    """

    resolution: float = Field(0.01, gt=0.0)
    courant_number: float = Field(0.5, gt=0.0, le=1.0)
    boundary: Literal["absorbing", "periodic", "reflecting"] = "absorbing"
    pml_layers: int = Field(10, ge=0)
