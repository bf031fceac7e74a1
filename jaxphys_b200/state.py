"""Result containers of the FDTD solvers.

Field-for-field the reference's ``EMFieldHistory`` (``src/neurosim/state.py:271-289``)
and ``EMFieldHistory3D`` (``src/neurosim/state.py:388-414``): time-major stacks of
saved frames plus the grid coordinates.  Arrays are torch tensors (fields on
the GPU, float32) unless ``simulate(..., output="numpy")`` asked for NumPy.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any


@dataclass(frozen=True)
class EMFieldHistory:
    """Time series of 2D TM field snapshots.

    Attributes:
        t: Time values, shape (n_snapshots,).
        ez: Ez snapshots, shape (n_snapshots, nx, ny).
        hx: Hx snapshots, shape (n_snapshots, nx, ny).
        hy: Hy snapshots, shape (n_snapshots, nx, ny).
        grid_x: Spatial x-coordinates.
        grid_y: Spatial y-coordinates.
    """

    t: Any
    ez: Any
    hx: Any
    hy: Any
    grid_x: Any
    grid_y: Any


@dataclass(frozen=True)
class EMFieldHistory3D:
    """Time series of 3D field snapshots.

    Attributes:
        t: Time values, shape (n_snapshots,).
        ex, ey, ez, hx, hy, hz: Snapshots, shape (n_snapshots, nx, ny, nz).
        grid_x, grid_y, grid_z: Spatial coordinates.
    """

    t: Any
    ex: Any
    ey: Any
    ez: Any
    hx: Any
    hy: Any
    hz: Any
    grid_x: Any
    grid_y: Any
    grid_z: Any
