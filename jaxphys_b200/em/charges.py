"""Moving point charges as sources of the 3D grid.

The reference's charge module (``src/neurosim/em/charges.py``) integrates
point charges under Coulomb and Lorentz forces and returns their
trajectories (``NBodyTrajectory``: ``t`` (S,), ``positions`` (S, n, 3)); it is
not coupled to a field solver.  Here a trajectory drives the Yee grid:
``MovingCharge3D`` deposits the charge's current on the E edges with
Esirkepov's charge-conserving scheme for a linear (cloud-in-cell) particle
shape (T. Zh. Esirkepov, Comput. Phys. Commun. 135, 144, 2001).  With node
weights S = S(t_n) and DS = S(t_n+1) - S(t_n) of the charge over step n
(a 4 x 4 x 4 node window around it),

    W_x = DS_x (S_y S_z + DS_y S_z / 2 + S_y DS_z / 2 + DS_y DS_z / 3)
    J_x(i + 1/2, j, k) = -q / (dx^2 dt) * sum over i' <= i of W_x(i', j, k)

(likewise y and z), and E += -dt / (eps0 eps_r) J on each edge after the E
update of step n, the same place as every soft source.  W_x + W_y + W_z =
S(t_n+1) - S(t_n) node by node, so the discrete continuity equation holds
exactly and, with the Yee identity div curl H = 0, so does Gauss's law
eps0 div(eps_r E) = rho(t) - rho(0) with rho = q S / dx^3 (checked on the
oracle in tests/test_charges.py).

The deposit is tabulated on the host: one per-step sample table per touched
(cell, component), fed through the grid's source tables, so the step kernels
are the ones of every other source.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Any

import numpy as np

from ..exceptions import ConfigurationError
from .fdtd3d import EPS0, PointSource3D
from .sources import SampleTable

_POL = "xyz"


def cic_weights(xi: float, base: int) -> np.ndarray:
    """Linear (cloud-in-cell) weights of nodes base .. base+3 for a charge at
    grid coordinate xi (node i sits at xi = i)."""
    return np.maximum(0.0, 1.0 - np.abs(xi - (base + np.arange(4))))


def deposit_step(xi0: np.ndarray, xi1: np.ndarray):
    """Esirkepov current weights of one step, in grid units.

    Returns (base, Fx, Fy, Fz): the window's low node (3,) and, on the window's
    edges, the flux sum_{i' <= i} W (so that J = -q / (dx^2 dt) * F).  Fx[i, j, k]
    belongs to the Ex edge of cell base + (i, j, k)."""
    xi0 = np.asarray(xi0, dtype=np.float64)
    xi1 = np.asarray(xi1, dtype=np.float64)
    if np.any(np.abs(xi1 - xi0) >= 1.0):
        raise ConfigurationError("the charge moves a cell or more in one step")
    base = np.floor(np.minimum(xi0, xi1)).astype(np.int64) - 1
    s0 = [cic_weights(xi0[a], base[a]) for a in range(3)]
    s1 = [cic_weights(xi1[a], base[a]) for a in range(3)]
    d = [s1[a] - s0[a] for a in range(3)]

    def w(a):
        b, c = (a + 1) % 3, (a + 2) % 3
        shape = [1, 1, 1]

        def ax(v, axis):
            sh = list(shape)
            sh[axis] = 4
            return v.reshape(sh)

        return ax(d[a], a) * (ax(s0[b], b) * ax(s0[c], c) + 0.5 * ax(d[b], b) * ax(s0[c], c)
                              + 0.5 * ax(s0[b], b) * ax(d[c], c)
                              + (1.0 / 3.0) * ax(d[b], b) * ax(d[c], c))

    return base, np.cumsum(w(0), axis=0), np.cumsum(w(1), axis=1), np.cumsum(w(2), axis=2)


def node_density(xi: np.ndarray, size) -> np.ndarray:
    """q = 1 charge density times dx^3 on the grid nodes (CIC weights)."""
    rho = np.zeros(size)
    base = np.floor(np.asarray(xi)).astype(np.int64) - 1
    wts = [cic_weights(xi[a], base[a]) for a in range(3)]
    for i in range(4):
        for j in range(4):
            for k in range(4):
                x, y, z = base + np.array([i, j, k])
                if 0 <= x < size[0] and 0 <= y < size[1] and 0 <= z < size[2]:
                    rho[x, y, z] += wts[0][i] * wts[1][j] * wts[2][k]
    return rho


@dataclass(frozen=True)
class MovingCharge3D:
    """A point charge following a prescribed path, as a current source.

    Attributes:
        charge: Charge in coulombs.
        times: Sample times (s) of the path, increasing, shape (S,).
        positions: Positions (m) at those times, shape (S, 3); the grid's cell
            (i, j, k) node sits at (i, j, k) * resolution.  Between samples the
            path is linear; after the last sample the charge rests.
    """

    charge: float
    times: Any
    positions: Any

    def grid_path(self, resolution: float, dt: float, t_start: float) -> np.ndarray:
        """Positions in grid units at t_start + n dt, n = 0 .. N (N = steps
        until the last sample time)."""
        t = np.asarray(self.times, dtype=np.float64)
        p = np.asarray(self.positions, dtype=np.float64)
        if t.ndim != 1 or p.shape != (len(t), 3) or len(t) < 2 or np.any(np.diff(t) <= 0):
            raise ConfigurationError("MovingCharge3D needs increasing times (S,) and positions "
                                     "(S, 3) with S >= 2")
        n_last = int(math.floor((t[-1] - t_start) / dt + 1e-9))
        if n_last < 1:
            raise ConfigurationError("the path ends before the first step")
        tn = t_start + dt * np.arange(n_last + 1)
        path = np.stack([np.interp(tn, t, p[:, a]) for a in range(3)], axis=1)
        return path / resolution

    def deposit_sources(self, size, resolution: float, dt: float, t_start: float = 0.0,
                        eps_r=None) -> list[PointSource3D]:
        """The deposit as point sources with per-step sample tables."""
        xi = self.grid_path(resolution, dt, t_start)
        n = np.asarray(size)
        if np.any(xi < 1.0) or np.any(xi > n - 3.0):
            raise ConfigurationError(
                f"MovingCharge3D path out of grid bounds {tuple(size)}: its current window "
                f"needs 1 <= x / resolution <= n - 3 on every axis")
        eps = None if eps_r is None else np.asarray(eps_r, dtype=np.float64)
        scale = self.charge / (EPS0 * resolution ** 2)  # -dt/eps0 * (-q/(dx^2 dt))
        rows: dict = {}
        n_steps = len(xi) - 1
        for step in range(n_steps):
            base, *flux = deposit_step(xi[step], xi[step + 1])
            for comp in range(3):
                f = flux[comp]
                for idx in zip(*np.nonzero(f)):
                    cell = tuple(int(v) for v in base + np.array(idx))
                    val = scale * f[idx]
                    if eps is not None:
                        val /= eps[cell]
                    key = (cell, comp)
                    if key not in rows:
                        rows[key] = np.zeros(n_steps)
                    rows[key][step] += val
        return [PointSource3D(frequency=0.0, position=cell, amplitude=1.0,
                              polarization=_POL[comp], waveform="table",
                              samples=SampleTable(v))
                for (cell, comp), v in sorted(rows.items())]


def charges_from_trajectory(t, positions, charges) -> list[MovingCharge3D]:
    """Sources for every charge of an N-body trajectory (the reference's
    ``NBodyTrajectory`` layout: ``t`` (S,), ``positions`` (S, n, 3))."""
    p = np.asarray(positions, dtype=np.float64)
    q = np.asarray(charges, dtype=np.float64).reshape(-1)
    if p.ndim != 3 or p.shape[2] != 3 or p.shape[1] != len(q):
        raise ConfigurationError("positions must be (S, n, 3) with one charge per body")
    return [MovingCharge3D(charge=float(q[i]), times=np.asarray(t, dtype=np.float64),
                           positions=p[:, i, :]) for i in range(len(q))]
