"""Rectangular waveguide modes, and mode ports that excite them in the 3D grid.

Analysis -- same classes, formulas, arguments and errors as the reference's
``src/neurosim/em/waveguides.py``:

* ``cutoff_frequency`` f_c = (c/2) sqrt((m/a)^2 + (n/b)^2)   (``:91-101``)
* ``propagation_constant`` beta = sqrt(k^2 - k_c^2), ``PhysicsError`` below
  cutoff (``:103-125``)
* ``compute_mode`` TE: Hz = cos(m pi x/a) cos(n pi y/b); TM: Ez = sin sin on
  an ``n_points`` x ``n_points`` linspace grid, ``ConfigurationError`` for
  TE00, TM with m or n < 1 and unknown mode types (``:127-188``)
* ``dispersion_relation`` beta(f), NaN below cutoff (``:190-212``)

Arrays are NumPy float64 (the reference returns JAX arrays).

Port excitation (extension): ``RectangularWaveguide.port`` returns a
``ModeSource3D``, a plane of soft E sources whose amplitudes follow the
transverse electric field of a TE_mn or TM_mn mode of the guide.  Guide
axis w, transverse axes (u, v) in cyclic order after w, walls at u = u0,
u0 + A and v = v0, v0 + B (cells).  On the Yee grid E_u sits at (i + 1/2, j)
and E_v at (i, j + 1/2) of the transverse plane, so

    TE_mn:  E_u = -(n/B) cos(m pi (i+1/2)/A) sin(n pi j/B)
            E_v =  (m/A) sin(m pi i/A) cos(n pi (j+1/2)/B)
    TM_mn:  E_u =  (m/A) cos(m pi (i+1/2)/A) sin(n pi j/B)
            E_v =  (n/B) sin(m pi i/A) cos(n pi (j+1/2)/B)

(i, j relative to the walls; the overall sign is chosen so that TE_m0 has a
positive E_v), scaled so the largest entry equals ``amplitude``.  Sources sit
on the cells strictly between the walls (1 <= i <= A-1, 1 <= j <= B-1), so
none lands on a wall cell made a conductor by ``walls``.  ``walls`` builds
the matching perfect-conductor tube for ``EMGrid3D.add_conductor``.  A soft
source on one plane radiates towards both ends of the guide.
"""

from __future__ import annotations

import logging
from dataclasses import dataclass
from typing import Literal

import numpy as np

from ..exceptions import ConfigurationError, PhysicsError
from .fdtd3d import PointSource3D

logger = logging.getLogger(__name__)

C0 = 299792458.0  # speed of light (m/s)
_AXIS = {"x": 0, "y": 1, "z": 2}
_POL = "xyz"


@dataclass(frozen=True)
class WaveguideMode:
    """A waveguide mode solution (``waveguides.py:35-54``).

    Attributes:
        mode_type: "TE" or "TM".
        m: Mode index along x.
        n: Mode index along y.
        cutoff_frequency: Cutoff frequency in Hz.
        field_pattern: 2D field pattern, shape (n_points, n_points).
        x: x-coordinates, shape (n_points,).
        y: y-coordinates, shape (n_points,).
    """

    mode_type: str
    m: int
    n: int
    cutoff_frequency: float
    field_pattern: np.ndarray
    x: np.ndarray
    y: np.ndarray


def _check_mode(mode_type: str, m: int, n: int) -> None:
    if mode_type not in ("TE", "TM"):
        raise ConfigurationError(f"mode_type must be 'TE' or 'TM', got '{mode_type}'")
    if mode_type == "TE" and m == 0 and n == 0:
        raise ConfigurationError("TE00 mode does not exist")
    if mode_type == "TM" and (m < 1 or n < 1):
        raise ConfigurationError(f"TM modes require m >= 1 and n >= 1, got ({m},{n})")
    if m < 0 or n < 0:
        raise ConfigurationError(f"mode indices must be >= 0, got ({m},{n})")


@dataclass(frozen=True)
class ModeSource3D:
    """A waveguide mode port: a plane of soft sources with the mode's
    transverse E profile (extension; see the module docstring).

    Attributes:
        mode_type, m, n: The mode.
        frequency: Source frequency in Hz (centre frequency for "gauss_sine").
        index: Cell index of the source plane along ``axis``.
        origin: (u0, v0), the cell indices of the low walls on the transverse
            axes (u, v) = the two axes after ``axis`` in cyclic order
            (z: (x, y); x: (y, z); y: (z, x)).
        extent: (A, B), wall-to-wall distance in cells (A, B >= 2).
        axis: Guide axis.
        amplitude: Largest source amplitude of the profile (V/m).
        waveform, width_steps, delay_steps: As for ``PointSource3D``.
    """

    mode_type: str
    m: int
    n: int
    frequency: float
    index: int
    origin: tuple[int, int]
    extent: tuple[int, int]
    axis: Literal["x", "y", "z"] = "z"
    amplitude: float = 1.0
    waveform: Literal["sine", "gauss_sine"] = "sine"
    width_steps: float = 30.0
    delay_steps: float | None = None

    def axes(self) -> tuple[int, int, int]:
        """(w, u, v) axis numbers."""
        if self.axis not in _AXIS:
            raise ConfigurationError(f"axis must be x, y or z, got {self.axis!r}")
        w = _AXIS[self.axis]
        return w, (w + 1) % 3, (w + 2) % 3

    def profile(self) -> tuple[np.ndarray, np.ndarray]:
        """(E_u, E_v) on the cells i = 0..A, j = 0..B of the aperture
        (relative to the walls), zero on the walls, largest |entry| = 1."""
        _check_mode(self.mode_type, self.m, self.n)
        A, B = (int(v) for v in self.extent)
        if A < 2 or B < 2:
            raise ConfigurationError(f"port extent must be at least 2x2 cells, got {self.extent}")
        m, n = self.m, self.n
        i = np.arange(A + 1, dtype=np.float64)[:, None]
        j = np.arange(B + 1, dtype=np.float64)[None, :]
        cu_ = np.cos(m * np.pi * (i + 0.5) / A) * np.sin(n * np.pi * j / B)
        sv_ = np.sin(m * np.pi * i / A) * np.cos(n * np.pi * (j + 0.5) / B)
        if self.mode_type == "TE":
            eu, ev = -(n / B) * cu_, (m / A) * sv_
        else:
            eu, ev = (m / A) * cu_, (n / B) * sv_
        inside = np.zeros((A + 1, B + 1), dtype=bool)
        inside[1:A, 1:B] = True
        eu = np.where(inside, eu, 0.0)
        ev = np.where(inside, ev, 0.0)
        peak = max(float(np.abs(eu).max()), float(np.abs(ev).max()))
        if peak == 0.0:
            raise ConfigurationError(
                f"{self.mode_type}{m}{n} has no transverse field on a {A}x{B}-cell aperture")
        return eu / peak, ev / peak

    def point_sources(self, size: tuple[int, int, int]) -> list[PointSource3D]:
        """The port as point sources of a grid of ``size`` (bounds checked)."""
        w, u, v = self.axes()
        A, B = (int(e) for e in self.extent)
        u0, v0 = (int(o) for o in self.origin)
        if not (0 <= self.index < size[w] and 0 <= u0 and u0 + A < size[u]
                and 0 <= v0 and v0 + B < size[v]):
            raise ConfigurationError(
                f"Port plane {self.axis}={self.index}, origin {self.origin}, extent "
                f"{self.extent} out of grid bounds {tuple(size)}")
        eu, ev = self.profile()
        tol = 1e-12
        out = []
        for comp, prof in ((u, eu), (v, ev)):
            for i, j in zip(*np.nonzero(np.abs(prof) > tol)):
                pos = [0, 0, 0]
                pos[w] = int(self.index)
                pos[u] = u0 + int(i)
                pos[v] = v0 + int(j)
                out.append(PointSource3D(
                    frequency=self.frequency, position=tuple(pos),
                    amplitude=float(self.amplitude * prof[i, j]), polarization=_POL[comp],
                    waveform=self.waveform, width_steps=self.width_steps,
                    delay_steps=self.delay_steps))
        return out


class RectangularWaveguide:
    """Rectangular metallic waveguide analyzer (``waveguides.py:57-212``).

    Example:
        >>> wg = RectangularWaveguide(a=0.02286, b=0.01016)  # WR-90
        >>> mode = wg.compute_mode("TE", 1, 0, n_points=100)
        >>> print(f"TE10 cutoff: {mode.cutoff_frequency/1e9:.3f} GHz")

    Args:
        a: Width (larger dimension) in meters.
        b: Height (smaller dimension) in meters.
    """

    def __init__(self, a: float, b: float) -> None:
        if a <= 0 or b <= 0:
            raise ConfigurationError(f"Waveguide dimensions must be positive: a={a}, b={b}")
        self._a = float(a)
        self._b = float(b)

    @property
    def a(self) -> float:
        """Waveguide width."""
        return self._a

    @property
    def b(self) -> float:
        """Waveguide height."""
        return self._b

    def cutoff_frequency(self, m: int, n: int) -> float:
        """Cutoff frequency (Hz) of mode (m, n)."""
        return float((C0 / 2.0) * np.sqrt((m / self._a) ** 2 + (n / self._b) ** 2))

    def propagation_constant(self, frequency: float, m: int, n: int) -> float:
        """Propagation constant beta (rad/m); ``PhysicsError`` below cutoff."""
        fc = self.cutoff_frequency(m, n)
        if frequency < fc:
            raise PhysicsError(
                f"Frequency {frequency:.3e} Hz is below cutoff "
                f"{fc:.3e} Hz for mode ({m},{n}). Mode is evanescent.")
        k = 2.0 * np.pi * frequency / C0
        kc = 2.0 * np.pi * fc / C0
        return float(np.sqrt(k ** 2 - kc ** 2))

    def compute_mode(self, mode_type: str, m: int, n: int, n_points: int = 100) -> WaveguideMode:
        """Transverse pattern of a mode: Hz (TE) or Ez (TM) on an n_points^2 grid."""
        _check_mode(mode_type, m, n)
        x = np.linspace(0.0, self._a, n_points)
        y = np.linspace(0.0, self._b, n_points)
        X, Y = np.meshgrid(x, y, indexing="ij")
        if mode_type == "TE":
            pattern = np.cos(m * np.pi * X / self._a) * np.cos(n * np.pi * Y / self._b)
        else:
            pattern = np.sin(m * np.pi * X / self._a) * np.sin(n * np.pi * Y / self._b)
        return WaveguideMode(mode_type=mode_type, m=m, n=n,
                             cutoff_frequency=self.cutoff_frequency(m, n),
                             field_pattern=pattern, x=x, y=y)

    def dispersion_relation(self, m: int, n: int, frequencies) -> np.ndarray:
        """beta(f) for an array of frequencies; NaN below cutoff."""
        f = np.asarray(frequencies, dtype=np.float64)
        fc = self.cutoff_frequency(m, n)
        k = 2.0 * np.pi * f / C0
        kc = 2.0 * np.pi * fc / C0
        beta_sq = k ** 2 - kc ** 2
        return np.where(beta_sq > 0, np.sqrt(np.maximum(beta_sq, 0.0)), np.nan)

    # ------------------------------------------------------------ FDTD ports
    def extent_cells(self, resolution: float) -> tuple[int, int]:
        """(A, B): the guide's width and height in cells of size ``resolution``."""
        A, B = int(round(self._a / resolution)), int(round(self._b / resolution))
        if A < 2 or B < 2:
            raise ConfigurationError(
                f"waveguide {self._a} x {self._b} m spans fewer than 2 cells at "
                f"resolution {resolution}")
        return A, B

    def port(self, mode_type: str, m: int, n: int, frequency: float, resolution: float,
             index: int, origin: tuple[int, int], axis: Literal["x", "y", "z"] = "z",
             amplitude: float = 1.0, waveform: Literal["sine", "gauss_sine"] = "sine",
             width_steps: float = 30.0, delay_steps: float | None = None) -> ModeSource3D:
        """A ``ModeSource3D`` exciting mode (m, n) of this guide in a grid of
        cell size ``resolution`` (the guide's a and b rounded to cells)."""
        _check_mode(mode_type, m, n)
        if frequency < self.cutoff_frequency(m, n):
            logger.warning("port frequency %.3e Hz is below the (%d,%d) cutoff %.3e Hz: "
                           "the mode is evanescent", frequency, m, n,
                           self.cutoff_frequency(m, n))
        return ModeSource3D(mode_type=mode_type, m=m, n=n, frequency=frequency, index=int(index),
                            origin=(int(origin[0]), int(origin[1])),
                            extent=self.extent_cells(resolution), axis=axis,
                            amplitude=amplitude, waveform=waveform, width_steps=width_steps,
                            delay_steps=delay_steps)

    def walls(self, size: tuple[int, int, int], resolution: float, origin: tuple[int, int],
              axis: Literal["x", "y", "z"] = "z", span: tuple[int, int] | None = None) -> np.ndarray:
        """Boolean mask of this guide's metal tube (one cell thick) in a grid
        of ``size``, walls at u0, u0 + A and v0, v0 + B over ``span`` = [w0, w1)
        along ``axis`` (default: the whole axis); for ``EMGrid3D.add_conductor``."""
        return tube_mask(size, self.extent_cells(resolution), origin, axis, span)


def tube_mask(size: tuple[int, int, int], extent: tuple[int, int], origin: tuple[int, int],
              axis: Literal["x", "y", "z"] = "z", span: tuple[int, int] | None = None) -> np.ndarray:
    """Boolean mask of a rectangular conductor tube: walls at u0, u0 + A and
    v0, v0 + B (cells) on the axes after ``axis``, over ``span`` along it."""
    if axis not in _AXIS:
        raise ConfigurationError(f"axis must be x, y or z, got {axis!r}")
    w = _AXIS[axis]
    u, v = (w + 1) % 3, (w + 2) % 3
    A, B = (int(e) for e in extent)
    u0, v0 = (int(o) for o in origin)
    w0, w1 = (0, size[w]) if span is None else (int(span[0]), int(span[1]))
    if not (0 <= u0 and u0 + A < size[u] and 0 <= v0 and v0 + B < size[v]
            and 0 <= w0 < w1 <= size[w]):
        raise ConfigurationError(
            f"Waveguide tube origin {origin}, extent {extent}, span {(w0, w1)} out of grid "
            f"bounds {tuple(size)}")
    plane = np.zeros((size[u], size[v]), dtype=bool)
    plane[u0, v0:v0 + B + 1] = True
    plane[u0 + A, v0:v0 + B + 1] = True
    plane[u0:u0 + A + 1, v0] = True
    plane[u0:u0 + A + 1, v0 + B] = True
    mask = np.zeros(size, dtype=bool)
    idx = [slice(None)] * 3
    idx[w] = slice(w0, w1)
    # place the (u, v) plane into the (x, y, z) layout
    order = np.argsort([w, u, v])          # axes of the (w, u, v) stack in x, y, z order
    stacked = np.broadcast_to(plane[None], (w1 - w0, size[u], size[v]))
    mask[tuple(idx)] = np.transpose(stacked, order)
    return mask
