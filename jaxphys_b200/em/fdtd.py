"""2D TM FDTD solver on B200: the drop-in for jaxphys ``EMGrid``.

Mirrors ``src/neurosim/em/fdtd.py`` of the reference: ``PlaneWave``
(``:45-56``), ``Wall`` (``:60-71``), ``EMGrid(size, resolution, boundary,
pml_layers)`` (``:93-113``) with ``EMConfig`` validation, ``size``
(``:115-118``), ``add_source`` (``:120-130``), ``add_conductor`` (``:132-142``)
and ``simulate(t_span, dt, save_every)`` (``:193-386``) returning
``EMFieldHistory``.  The time loop runs in the CUDA kernels of
``jaxphys_b200/csrc`` (float32 on the GPU).
"""

from __future__ import annotations

import ctypes as C
import logging
import math
from dataclasses import dataclass
from typing import Literal

import numpy as np

from .. import _native as nat
from ..config import EMConfig
from ..exceptions import ConfigurationError
from ..state import EMFieldHistory, resolve_output, to_jax
from . import sources as wf

logger = logging.getLogger(__name__)

C0 = 299792458.0
MU0 = 4.0e-7 * math.pi
EPS0 = 1.0 / (MU0 * C0**2)

_BOUNDARY = {
    "absorbing": nat.BND_ABSORBING,
    "periodic": nat.BND_PERIODIC,
    "reflecting": nat.BND_REFLECTING,
}


@dataclass(frozen=True)
class PlaneWave:
    """Plane wave (line) source: Ez[:, y] += amplitude * sin(2 pi f t).

    Attributes:
        frequency: Wave frequency in Hz.
        y: Source y-position (grid index).
        amplitude: Peak electric field amplitude (V/m).
    """

    frequency: float
    y: int
    amplitude: float = 1.0


@dataclass(frozen=True)
class Wall:
    """Conducting wall with optional gap (slit).

    Attributes:
        y: Wall y-position (grid index).
        gap_start: Start of gap (grid index). None for solid wall.
        gap_end: End of gap (grid index). None for solid wall.
    """

    y: int
    gap_start: int | None = None
    gap_end: int | None = None


class EMGrid:
    """2D electromagnetic FDTD simulation grid (TM: Ez, Hx, Hy).

    Example:
        >>> grid = EMGrid(size=(200, 200), resolution=0.01)
        >>> grid.add_source(PlaneWave(frequency=3e9, y=20))
        >>> grid.add_conductor(Wall(y=100, gap_start=90, gap_end=110))
        >>> fields = grid.simulate(t_span=(0, 1e-8), dt=1e-11)
    """

    def __init__(
        self,
        size: tuple[int, int] = (200, 200),
        resolution: float = 0.01,
        boundary: Literal["absorbing", "periodic", "reflecting"] = "absorbing",
        pml_layers: int = 10,
        *,
        device: int | None = None,
    ) -> None:
        self._nx, self._ny = (int(v) for v in size)
        self._dx = resolution
        self._config = EMConfig(
            resolution=resolution,
            courant_number=0.5,
            boundary=boundary,
            pml_layers=pml_layers,
        )
        self._sources: list[PlaneWave] = []
        self._conductors: list[Wall] = []
        self._device = device
        self._h = None
        self._h_key = None

        if self._nx < 10 or self._ny < 10:
            raise ConfigurationError(f"Grid must be at least 10x10, got {size}")

    @property
    def size(self) -> tuple[int, int]:
        """Grid dimensions (nx, ny)."""
        return (self._nx, self._ny)

    def add_source(self, source: PlaneWave) -> None:
        """Add a plane wave source to the grid (fdtd.py:120-130)."""
        if source.y < 0 or source.y >= self._ny:
            raise ConfigurationError(
                f"Source y={source.y} out of grid bounds [0, {self._ny})"
            )
        self._sources.append(source)

    def add_conductor(self, wall: Wall) -> None:
        """Add a conducting wall, optionally with a slit (fdtd.py:132-142)."""
        if wall.y < 0 or wall.y >= self._ny:
            raise ConfigurationError(
                f"Wall y={wall.y} out of grid bounds [0, {self._ny})"
            )
        self._conductors.append(wall)

    def default_dt(self) -> float:
        """CFL step 0.99*dx/(c*sqrt(2)) (fdtd.py:214)."""
        return float(0.99 * self._dx / (C0 * float(np.sqrt(2.0))))

    def _release(self) -> None:
        if self._h is not None:
            try:
                nat.load().jxf_grid2d_destroy(self._h)
            finally:
                self._h = None
                self._h_key = None

    def __del__(self):  # pragma: no cover
        try:
            self._release()
        except Exception:
            pass

    def _prepare(self, dt: float, t_start: float, n_steps: int) -> None:
        import torch

        dev = self._device if self._device is not None else torch.cuda.current_device()
        key = (dt, dev)
        lib = nat.load()
        if self._h is None or self._h_key != key:
            self._release()
            d = nat.Grid2DDesc(nx=self._nx, ny=self._ny, dx=float(self._dx), dt=float(dt),
                               boundary=_BOUNDARY[self._config.boundary],
                               pml_layers=int(self._config.pml_layers), device=int(dev))
            h = C.c_void_p()
            nat.check(lib.jxf_grid2d_create(C.byref(d), C.byref(h)), "jxf_grid2d_create")
            self._h = h
            self._h_key = key
        keys: list = []
        rows = []
        for s in self._sources:
            k = ("sine", float(s.frequency))
            if k not in keys:
                keys.append(k)
            rows.append(keys.index(k))
        ys = np.array([s.y for s in self._sources], dtype=np.int32)
        amp = np.array([s.amplitude for s in self._sources], dtype=np.float32)
        row = np.array(rows, dtype=np.int32)
        nat.check(lib.jxf_grid2d_set_sources(self._h, len(ys), ys.ctypes.data, amp.ctypes.data,
                                             row.ctypes.data), "set_sources")
        table = wf.build_table(keys, max(n_steps, 1), dt, t_start)
        nat.check(lib.jxf_grid2d_set_waveforms(self._h, len(keys), table.shape[1],
                                               table.ctypes.data), "set_waveforms")
        wy, g0, g1 = [], [], []
        for w in self._conductors:
            wy.append(w.y)
            if w.gap_start is not None and w.gap_end is not None:
                # row = (x < gap_start) | (x >= gap_end)  (fdtd.py:153-155)
                g0.append(max(int(w.gap_start), 0))
                g1.append(int(w.gap_end))
            else:
                g0.append(-1)
                g1.append(-1)
        wy_a = np.array(wy, dtype=np.int32)
        g0_a = np.array(g0, dtype=np.int32)
        g1_a = np.array(g1, dtype=np.int32)
        nat.check(lib.jxf_grid2d_set_walls(self._h, len(wy_a), wy_a.ctypes.data, g0_a.ctypes.data,
                                           g1_a.ctypes.data), "set_walls")
        nat.check(lib.jxf_grid2d_reset(self._h, nat.stream_handle()), "reset")

    def simulate(
        self,
        t_span: tuple[float, float] = (0.0, 1e-8),
        dt: float | None = None,
        save_every: int = 10,
        output: Literal["torch", "numpy", "jax", "auto"] = "torch",
    ) -> EMFieldHistory:
        """Run the FDTD simulation (fdtd.py:193-386).

        output: "torch" (tensors), "numpy", "jax" (JAX arrays through DLPack,
        the reference's result type) or "auto" (JAX when importable, else
        torch)."""
        import torch

        output = resolve_output(output)
        dx = self._dx
        nx, ny = self._nx, self._ny
        dt = self.default_dt() if dt is None else float(dt)
        t_start, t_end = t_span
        n_steps = int((t_end - t_start) / dt)
        if not self._sources:
            raise ConfigurationError("At least one source must be added before simulation")
        logger.info("Starting FDTD simulation: grid=%dx%d, dt=%.2e, n_steps=%d", nx, ny, dt, n_steps)
        self._prepare(dt, t_start, n_steps)
        stride = save_every if save_every > 1 else 1
        saved = list(range(0, max(n_steps, 0), stride))
        devname = f"cuda:{self._h_key[1]}"
        hist = [torch.empty((len(saved), nx, ny), dtype=torch.float32, device=devname)
                for _ in range(3)]
        lib = nat.load()
        st = nat.stream_handle()
        done = 0
        for s, k in enumerate(saved):
            if k + 1 > done:
                nat.check(lib.jxf_grid2d_step(self._h, k + 1 - done, st), "jxf_grid2d_step")
                done = k + 1
            for c in range(3):
                nat.check(lib.jxf_grid2d_get_field(self._h, c, hist[c][s].data_ptr(), 0, st),
                          "get_field")
        if n_steps > done:
            nat.check(lib.jxf_grid2d_step(self._h, n_steps - done, st), "jxf_grid2d_step")
        nat.check(lib.jxf_grid2d_check_error(self._h, st), "device error")
        t = np.array([t_start + k * dt + dt for k in saved], dtype=np.float64)
        gx = np.arange(nx) * dx
        gy = np.arange(ny) * dx
        if output == "numpy":
            return EMFieldHistory(t, hist[0].cpu().numpy(), hist[1].cpu().numpy(),
                                  hist[2].cpu().numpy(), gx, gy)
        if output == "jax":
            import jax.numpy as jnp

            return EMFieldHistory(jnp.asarray(t), *[to_jax(h) for h in hist], jnp.asarray(gx),
                                  jnp.asarray(gy))
        return EMFieldHistory(torch.from_numpy(t), hist[0], hist[1], hist[2],
                              torch.from_numpy(gx), torch.from_numpy(gy))


FDTD2D = EMGrid
