"""3D FDTD Maxwell solver on B200: the drop-in for jaxphys ``EMGrid3D``.

Mirrors ``src/neurosim/em/fdtd3d.py`` of the reference:

* ``PointSource3D`` (``:41-55``), ``DielectricRegion`` (``:58-68``) -- same fields
  and defaults; ``PointSource3D`` gains optional waveform fields.
* ``EMGrid3D(size, resolution, boundary, pml_layers)`` (``:90-105``) with the
  same validation and messages, ``size`` (``:107-110``), ``add_source``
  (``:112-120``), ``add_material`` (``:122-130``) and ``simulate(t_span, dt,
  save_every)`` (``:169-417``) returning ``EMFieldHistory3D``.

The time loop runs in the CUDA kernels of ``jaxphys_b200/csrc`` through the C
ABI of ``include/jaxphys_fdtd.h``; only saved frames are copied out (the
reference stores all six fields at every step and subsamples afterwards).
Fields are float32 on the GPU.

Extensions: ``boundary="cpml"`` (convolutional PML with psi recurrences) and
``"pec"``; per-cell permittivity via ``set_permittivity``; probes
(``add_probe`` / ``run``); ``step``/``run``/``reset``/``fields`` for
incremental stepping; ``FDTD3D`` alias.
"""

from __future__ import annotations

import ctypes as C
import logging
import math
from dataclasses import dataclass
from typing import Any, Literal

import numpy as np

from .. import _native as nat
from ..exceptions import ConfigurationError, SimulationError
from ..state import EMFieldHistory3D, resolve_output, to_jax
from . import sources as wf

logger = logging.getLogger(__name__)

# Physical constants (SI), fdtd3d.py:36-38
C0 = 299792458.0
MU0 = 4.0e-7 * math.pi
EPS0 = 1.0 / (MU0 * C0**2)

COMPONENTS = ("ex", "ey", "ez", "hx", "hy", "hz")
_POL = {"x": 0, "y": 1, "z": 2}
_BOUNDARY = {
    "absorbing": nat.BND_ABSORBING,
    "periodic": nat.BND_PERIODIC,
    "pec": nat.BND_PEC,
    "cpml": nat.BND_CPML,
    # learned absorbing band: PEC walls plus the band correction after each step
    "learned": nat.BND_PEC,
}
_PATH = {"auto": nat.PATH_AUTO, "generic": nat.PATH_GENERIC, "tma": nat.PATH_TMA}


@dataclass(frozen=True)
class PointSource3D:
    """Point source specification for 3D FDTD.

    Attributes:
        frequency: Source frequency in Hz (centre frequency for "gauss_sine").
        position: Source location as (ix, iy, iz) grid indices.
        amplitude: Peak electric field amplitude (V/m).
        polarization: Which E-field component to drive.
        waveform: "sine" (reference), "gauss_sine" (Gaussian-modulated
            sinusoid, extension) or "table" (explicit per-step values,
            extension).
        width_steps: Gaussian 1/e half-width in time steps ("gauss_sine").
        delay_steps: Pulse centre in time steps; default four widths.
        samples: ``sources.SampleTable`` of per-step values ("table").
    """

    frequency: float
    position: tuple[int, int, int]
    amplitude: float = 1.0
    polarization: Literal["x", "y", "z"] = "z"
    waveform: Literal["sine", "gauss_sine", "table"] = "sine"
    width_steps: float = 30.0
    delay_steps: float | None = None
    samples: Any = None


@dataclass(frozen=True)
class DielectricRegion:
    """Region with custom permittivity.

    Attributes:
        mask: Boolean array, shape (nx, ny, nz). True where material is.
        epsilon_r: Relative permittivity of the region.
    """

    mask: Any
    epsilon_r: float = 1.0


@dataclass(frozen=True)
class CPMLSpec:
    """Convolutional PML grading (extension; Roden & Gedney 2000).

    sigma(rho) = sigma_max rho^order with
    sigma_max = -(order+1) ln(r0) / (2 eta0 pml_layers dx),
    kappa = 1 + (kappa_max-1) rho^order, alpha = alpha_max (1-rho).
    """

    order: float = 3.0
    r0: float = 1e-6
    kappa_max: float = 1.0
    alpha_max: float = 0.0


def _to_numpy(a) -> np.ndarray:
    if hasattr(a, "detach"):
        a = a.detach().cpu().numpy()
    return np.asarray(a)


def _default_device() -> int:
    import torch

    if not torch.cuda.is_available():
        raise SimulationError("the FDTD engine needs a CUDA device (none is visible)")
    return torch.cuda.current_device()


class EMGrid3D:
    """3D electromagnetic FDTD simulation grid (B200 kernels).

    Example:
        >>> grid = EMGrid3D(size=(60, 60, 60), resolution=0.01)
        >>> grid.add_source(PointSource3D(frequency=3e9, position=(30, 30, 10)))
        >>> fields = grid.simulate(t_span=(0, 5e-9), save_every=20)

    Args:
        size: Grid dimensions (nx, ny, nz) in cells.
        resolution: Cell size in meters (uniform in all directions).
        boundary: "absorbing" (reference damping layers), "periodic",
            "pec" (no boundary treatment), "cpml" (extension) or "learned"
            (extension: the outer 3 cell layers are a learned absorbing band,
            ``jaxphys_b200.em.learned``, applied after every step on either
            kernel path).
        pml_layers: Number of damping / CPML layers.
        cpml: CPML grading (boundary="cpml").
        device: CUDA device ordinal (default: torch's current device).
        path: "auto", "tma" or "generic" kernel path.
        band: boundary="learned": the ``LearnedBand`` to use (default: the
            shipped weights).
    """

    def __init__(
        self,
        size: tuple[int, int, int] = (60, 60, 60),
        resolution: float = 0.01,
        boundary: Literal["absorbing", "periodic", "pec", "cpml", "learned"] = "absorbing",
        pml_layers: int = 8,
        *,
        cpml: CPMLSpec | None = None,
        device: int | None = None,
        path: str = "auto",
        band=None,
    ) -> None:
        self._nx, self._ny, self._nz = (int(v) for v in size)
        self._dx = resolution
        self._boundary = boundary
        self._pml_layers = pml_layers
        self._sources: list[PointSource3D] = []
        self._materials: list[DielectricRegion] = []
        self._eps_override: np.ndarray | None = None
        self._eps_device = None
        self._conductor: np.ndarray | None = None
        self._probes: list[tuple[int, int, int, int]] = []
        self._cpml = cpml or CPMLSpec()
        self._device = device
        self._path = path
        self._band = band
        self._h = None
        self._h_key = None
        self._dt = None
        self._t_start = 0.0
        self._wave_cap = 0
        self._dirty = True

        if min(size) < 8:
            raise ConfigurationError(f"Grid must be at least 8x8x8, got {size}")
        if path not in _PATH:
            raise ConfigurationError(f"path must be one of {sorted(_PATH)}, got {path!r}")

    # ------------------------------------------------------------------ API
    @property
    def size(self) -> tuple[int, int, int]:
        """Grid dimensions (nx, ny, nz)."""
        return (self._nx, self._ny, self._nz)

    def add_source(self, source: PointSource3D) -> None:
        """Add a point source to the grid (fdtd3d.py:112-120).

        Extension: a ``waveguides.ModeSource3D`` (waveguide mode port) adds
        its plane of point sources; a ``charges.MovingCharge3D`` adds the
        current deposit of its trajectory (tabulated with this grid's cell
        size, default time step and current permittivity)."""
        if hasattr(source, "point_sources"):
            for s in source.point_sources(self.size):
                self.add_source(s)
            return
        if hasattr(source, "deposit_sources"):
            dt = self._dt if self._dt is not None else self.default_dt()
            for s in source.deposit_sources(self.size, self._dx, dt, self._t_start,
                                            self.epsilon_r()):
                self.add_source(s)
            return
        ix, iy, iz = source.position
        if not (0 <= ix < self._nx and 0 <= iy < self._ny and 0 <= iz < self._nz):
            raise ConfigurationError(
                f"Source position {source.position} out of grid bounds "
                f"({self._nx}, {self._ny}, {self._nz})"
            )
        if source.polarization not in _POL:
            raise ConfigurationError(f"polarization must be x, y or z, got {source.polarization!r}")
        self._sources.append(source)
        self._dirty = True

    def add_material(self, material: DielectricRegion) -> None:
        """Add a dielectric region to the grid (fdtd3d.py:122-130)."""
        expected = (self._nx, self._ny, self._nz)
        if tuple(material.mask.shape) != expected:
            raise ConfigurationError(
                f"Material mask shape {material.mask.shape} doesn't match "
                f"grid size {expected}"
            )
        self._materials.append(material)
        self._dirty = True

    def add_conductor(self, mask) -> None:
        """Extension: perfect electric conductor cells (metal walls, waveguides).

        ``mask`` is a boolean array of the grid shape; masked cells get an
        infinite permittivity, so the E update factor there is zero and
        Ex, Ey, Ez of those cells stay at zero (staircased metal).  Several
        calls accumulate; the conductors apply over any permittivity set
        by materials, ``set_permittivity`` or ``set_permittivity_device``.
        """
        m = np.asarray(_to_numpy(mask)).astype(bool)
        if m.shape != self.size:
            raise ConfigurationError(
                f"Conductor mask shape {m.shape} doesn't match grid size {self.size}")
        self._conductor = m.copy() if self._conductor is None else (self._conductor | m)
        self._dirty = True

    def set_permittivity(self, eps_r) -> None:
        """Extension: per-cell relative permittivity (replaces the masks).

        A NumPy array (or CPU tensor) is turned into dt/(eps0 dx eps_r) in
        FP64 on the host; a float32 CUDA tensor stays on the device (zero
        copy: its data pointer goes to the C ABI) and the division runs there
        in FP32."""
        if hasattr(eps_r, "is_cuda") and eps_r.is_cuda:
            self.set_permittivity_device(eps_r)
            return
        arr = np.asarray(_to_numpy(eps_r), dtype=np.float64)
        if arr.shape != self.size:
            raise ConfigurationError(
                f"permittivity shape {arr.shape} doesn't match grid size {self.size}")
        if not np.all(np.isfinite(arr)) or np.any(arr <= 0):
            raise ConfigurationError("permittivity must be finite and positive")
        self._eps_override = arr
        self._eps_device = None
        self._dirty = True

    def set_permittivity_device(self, eps_r) -> None:
        """Per-cell permittivity from a float32 CUDA tensor of the grid shape."""
        import torch

        if tuple(eps_r.shape) != self.size:
            raise ConfigurationError(
                f"permittivity shape {tuple(eps_r.shape)} doesn't match grid size {self.size}")
        t = eps_r.to(torch.float32).contiguous()
        self._eps_override = None
        self._eps_device = t
        if self._h is not None and not self._dirty and self._conductor is None:
            nat.check(nat.load().jxf_grid3d_set_eps_device(self._h, t.data_ptr(),
                                                           nat.stream_handle()), "set_eps")
        else:
            self._dirty = True

    def add_probe(self, position: tuple[int, int, int], component: str = "ez") -> int:
        """Extension: record ``component`` at ``position`` after every step."""
        ix, iy, iz = position
        if not (0 <= ix < self._nx and 0 <= iy < self._ny and 0 <= iz < self._nz):
            raise ConfigurationError(
                f"Probe position {position} out of grid bounds ({self._nx}, {self._ny}, {self._nz})")
        if component not in COMPONENTS:
            raise ConfigurationError(f"component must be one of {COMPONENTS}")
        self._probes.append((int(ix), int(iy), int(iz), COMPONENTS.index(component)))
        self._dirty = True
        return len(self._probes) - 1

    def epsilon_r(self) -> np.ndarray:
        """Relative permittivity grid (fdtd3d.py:132-137, or the override)."""
        if self._eps_device is not None:
            eps = self._eps_device.detach().cpu().numpy().astype(np.float64)
        elif self._eps_override is not None:
            eps = self._eps_override
        else:
            eps = np.ones(self.size)
            for mat in self._materials:
                eps = np.where(_to_numpy(mat.mask).astype(bool), mat.epsilon_r, eps)
        if self._conductor is not None:
            eps = np.where(self._conductor, np.inf, eps)
        return eps

    def default_dt(self) -> float:
        """CFL step 0.99*dx/(c*sqrt(3)) (fdtd3d.py:189-192)."""
        return float(0.99 * self._dx / (C0 * float(np.sqrt(3.0))))

    # ---------------------------------------------------------- device side
    def _ensure_handle(self, dt: float) -> None:
        dev = self._device if self._device is not None else _default_device()
        key = (dt, dev)
        if self._h is not None and self._h_key == key:
            return
        self._release()
        lib = nat.load()
        if self._boundary not in _BOUNDARY:
            # the reference runs the non-periodic stencil without damping for
            # any other string (fdtd3d.py:247,302,362)
            bnd = nat.BND_PEC
        else:
            bnd = _BOUNDARY[self._boundary]
        d = nat.Grid3DDesc(
            nx=self._nx, ny=self._ny, nz=self._nz, dx=float(self._dx), dt=float(dt),
            boundary=bnd, pml_layers=int(self._pml_layers),
            cpml_order=float(self._cpml.order), cpml_r0=float(self._cpml.r0),
            cpml_kappa_max=float(self._cpml.kappa_max), cpml_alpha_max=float(self._cpml.alpha_max),
            path=_PATH[self._path], device=int(dev))
        h = C.c_void_p()
        nat.check(lib.jxf_grid3d_create(C.byref(d), C.byref(h)), "jxf_grid3d_create")
        self._h = h
        self._h_key = key
        if self._boundary == "learned":
            from .learned import default_band

            if self._band is None:
                self._band = default_band(int(dev))
            nat.check(lib.jxf_grid3d_set_band(h, self._band._h), "jxf_grid3d_set_band")
        self._dt = dt
        self._wave_cap = 0
        self._dirty = True

    def _release(self) -> None:
        if self._h is not None:
            try:
                nat.load().jxf_grid3d_destroy(self._h)
            finally:
                self._h = None
                self._h_key = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order varies
        try:
            self._release()
        except Exception:
            pass

    def _upload_config(self) -> None:
        lib = nat.load()
        if self._eps_device is not None:
            t = self._eps_device
            if self._conductor is not None:
                import torch

                t = t.masked_fill(torch.from_numpy(self._conductor).to(t.device), float("inf"))
                self._eps_upload = t  # keep alive until the stream has read it
            nat.check(lib.jxf_grid3d_set_eps_device(self._h, t.data_ptr(),
                                                    nat.stream_handle()), "set_eps")
        elif self._eps_override is None and not self._materials and self._conductor is None:
            nat.check(lib.jxf_grid3d_set_eps_host(self._h, None), "set_eps")
        else:
            eps = np.ascontiguousarray(self.epsilon_r(), dtype=np.float64)
            nat.check(lib.jxf_grid3d_set_eps_host(self._h, eps.ctypes.data), "set_eps")
        keys: list = []
        rows = []
        for s in self._sources:
            k = wf.waveform_key(s)
            if k not in keys:
                keys.append(k)
            rows.append(keys.index(k))
        self._wave_keys = keys
        nx, ny, nz = self.size
        cell = np.array([(s.position[0] * ny + s.position[1]) * nz + s.position[2]
                         for s in self._sources], dtype=np.int64)
        comp = np.array([_POL[s.polarization] for s in self._sources], dtype=np.int32)
        amp = np.array([s.amplitude for s in self._sources], dtype=np.float32)
        row = np.array(rows, dtype=np.int32)
        nat.check(lib.jxf_grid3d_set_sources(self._h, len(cell), cell.ctypes.data, comp.ctypes.data,
                                             amp.ctypes.data, row.ctypes.data), "set_sources")
        pc = np.array([(p[0] * ny + p[1]) * nz + p[2] for p in self._probes], dtype=np.int64)
        pk = np.array([p[3] for p in self._probes], dtype=np.int32)
        nat.check(lib.jxf_grid3d_set_probes(self._h, len(pc), pc.ctypes.data, pk.ctypes.data),
                  "set_probes")
        self._wave_cap = 0
        self._dirty = False

    def _ensure_waves(self, upto: int) -> None:
        if upto <= self._wave_cap:
            return
        cap = max(upto, 2 * self._wave_cap, 64)
        table = wf.build_table(self._wave_keys, cap, self._dt, self._t_start)
        nat.check(nat.load().jxf_grid3d_set_waveforms(self._h, len(self._wave_keys), cap,
                                                      table.ctypes.data), "set_waveforms")
        self._wave_table = table  # keep the host copy alive for the call
        self._wave_cap = cap

    def prepare(self, dt: float | None = None, t_start: float = 0.0) -> None:
        """Create the device grid for time step ``dt`` and zero its state."""
        dt = self.default_dt() if dt is None else float(dt)
        self._ensure_handle(dt)
        self._t_start = float(t_start)
        self._upload_config()
        self.reset()

    def reset(self) -> None:
        """Zero all fields (and CPML state); the step counter restarts at 0."""
        if self._h is None:
            self.prepare()
            return
        nat.check(nat.load().jxf_grid3d_reset(self._h, nat.stream_handle()), "reset")

    @property
    def step_count(self) -> int:
        return self.info()["step"] if self._h is not None else 0

    def info(self) -> dict:
        inf = nat.Grid3DInfo()
        nat.check(nat.load().jxf_grid3d_get_info(self._h, C.byref(inf)), "get_info")
        return {f: getattr(inf, f) for f, _ in nat.Grid3DInfo._fields_}

    def kernels_per_step(self) -> int:
        """Step kernels launched per leapfrog step (after the first step)."""
        return int(self.info()["kernels_per_step"])

    def run(self, n_steps: int, record_probes: bool = True):
        """Extension: advance ``n_steps``; returns probe traces
        (n_steps, n_probes) as a device tensor (None without probes)."""
        import torch

        if self._h is None:
            self.prepare(self._dt, self._t_start)
        elif self._dirty:
            self._upload_config()  # keeps the fields and the step counter
        n_steps = int(n_steps)
        if n_steps < 0:
            raise ConfigurationError("n_steps must be >= 0")
        step0 = self.step_count
        if self._sources:
            self._ensure_waves(step0 + n_steps)
        out = None
        if record_probes and self._probes:
            out = torch.empty((n_steps, len(self._probes)), dtype=torch.float32,
                              device=f"cuda:{self._h_key[1]}")
        nat.check(nat.load().jxf_grid3d_step(self._h, n_steps,
                                             None if out is None else out.data_ptr(),
                                             nat.stream_handle()), "jxf_grid3d_step")
        return out

    # ------------------------------------------------------------- adjoint
    def adjoint_forward(self, n_steps: int, checkpoint_every: int | None = None):
        """Extension: reset, run ``n_steps`` keeping sqrt(T) checkpoints for
        :meth:`adjoint_backward`; returns the probe traces (n_steps, P)."""
        import torch

        if self._h is None:
            self.prepare(self._dt, self._t_start)
        elif self._dirty:
            self._upload_config()
        if self._sources:
            self._ensure_waves(int(n_steps))
        out = torch.empty((int(n_steps), len(self._probes)), dtype=torch.float32,
                          device=f"cuda:{self._h_key[1]}")
        nat.check(nat.load().jxf_grid3d_adjoint_forward(
            self._h, int(n_steps), int(checkpoint_every or 0),
            out.data_ptr() if self._probes else None, nat.stream_handle()),
            "jxf_grid3d_adjoint_forward")
        return out

    def adjoint_backward(self, probe_grad):
        """Extension: dJ/d(eps_r) (device tensor of the grid shape) for
        ``probe_grad`` = dJ/d(probe traces) of the last adjoint_forward."""
        import torch

        g = probe_grad.detach().to(torch.float32).contiguous()
        out = torch.empty(self.size, dtype=torch.float32, device=f"cuda:{self._h_key[1]}")
        nat.check(nat.load().jxf_grid3d_adjoint_backward(self._h, g.data_ptr(), out.data_ptr(),
                                                         nat.stream_handle()),
                  "jxf_grid3d_adjoint_backward")
        return out

    def step(self, n: int = 1) -> None:
        """Extension: advance ``n`` steps without probe recording."""
        self.run(n, record_probes=False)

    def field(self, name: str):
        """Copy of one current field component (device tensor, float32)."""
        import torch

        c = COMPONENTS.index(name)
        out = torch.empty(self.size, dtype=torch.float32, device=f"cuda:{self._h_key[1]}")
        nat.check(nat.load().jxf_grid3d_get_field(self._h, c, out.data_ptr(), 0,
                                                  nat.stream_handle()), "get_field")
        return out

    def set_field(self, name: str, value) -> None:
        """Overwrite one current field component from a tensor / array."""
        import torch

        c = COMPONENTS.index(name)
        t = torch.as_tensor(value, dtype=torch.float32)
        if tuple(t.shape) != self.size:
            raise ConfigurationError(f"field shape {tuple(t.shape)} != grid size {self.size}")
        t = t.to(f"cuda:{self._h_key[1]}").contiguous()
        nat.check(nat.load().jxf_grid3d_set_field(self._h, c, t.data_ptr(), 0,
                                                  nat.stream_handle()), "set_field")

    @property
    def fields(self) -> dict:
        """Copies of the six current field components."""
        return {k: self.field(k) for k in COMPONENTS}

    def check(self, finite: bool = True) -> None:
        """Synchronise; raise on a device error flag or on NaN/Inf fields."""
        lib = nat.load()
        nat.check(lib.jxf_grid3d_check_error(self._h, nat.stream_handle()), "device error")
        if finite:
            nat.check(lib.jxf_grid3d_check_finite(self._h, nat.stream_handle()), "fields")

    # ---------------------------------------------------------- simulate
    def simulate(
        self,
        t_span: tuple[float, float] = (0.0, 5e-9),
        dt: float | None = None,
        save_every: int = 20,
        output: Literal["torch", "numpy", "jax", "auto"] = "torch",
        history: Literal["device", "host"] = "device",
    ) -> EMFieldHistory3D:
        """Run the 3D FDTD simulation (fdtd3d.py:169-417).

        Returns the frames the reference keeps: states after steps
        1, 1+s, 1+2s, ... (s = save_every; every step when s <= 1) with their
        times t_start + k*dt + dt.

        history="device" keeps the frames in device memory (torch tensors on
        the GPU).  history="host" streams them into pinned host memory as they
        are produced: each frame is copied into one of two device staging
        slots and from there to the host on a side stream while the next
        steps run, so device memory holds two frames whatever the number of
        frames (the reference materialises every step, fdtd3d.py:371-404).

        output: "torch" (tensors), "numpy", "jax" (JAX arrays through DLPack,
        the reference's result type) or "auto" (JAX when importable, else
        torch).
        """
        import torch

        output = resolve_output(output)
        dx = self._dx
        nx, ny, nz = self.size
        if dt is None:
            dt = self.default_dt()
        dt = float(dt)
        t_start, t_end = t_span
        n_steps = int((t_end - t_start) / dt)
        if not self._sources:
            raise ConfigurationError("At least one source must be added before simulation")
        logger.info("Starting 3D FDTD: grid=%dx%dx%d, dt=%.2e, n_steps=%d", nx, ny, nz, dt, n_steps)

        self._dirty = True
        self.prepare(dt, t_start)
        stride = save_every if save_every > 1 else 1
        saved = list(range(0, max(n_steps, 0), stride))
        dev = f"cuda:{self._h_key[1]}"
        if history not in ("device", "host"):
            raise ConfigurationError(f"history must be 'device' or 'host', got {history!r}")
        to_host = history == "host"
        if to_host:
            hist = [torch.empty((len(saved),) + self.size, dtype=torch.float32, pin_memory=True)
                    for _ in COMPONENTS]
            stage = [torch.empty((6,) + self.size, dtype=torch.float32, device=dev)
                     for _ in range(2)]
            copy_stream = torch.cuda.Stream(device=dev)
            slot_free = [None, None]
        else:
            hist = [torch.empty((len(saved),) + self.size, dtype=torch.float32, device=dev)
                    for _ in COMPONENTS]
        lib = nat.load()
        main = torch.cuda.current_stream(dev)
        st = nat.stream_handle()
        self._ensure_waves(max(n_steps, 1))
        done = 0
        for s, k in enumerate(saved):
            if k + 1 > done:
                nat.check(lib.jxf_grid3d_step(self._h, k + 1 - done, None, st), "jxf_grid3d_step")
                done = k + 1
            if not to_host:
                for c in range(6):
                    nat.check(lib.jxf_grid3d_get_field(self._h, c, hist[c][s].data_ptr(), 0, st),
                              "get_field")
                continue
            slot = s % 2
            if slot_free[slot] is not None:
                main.wait_event(slot_free[slot])  # its previous frame has reached the host
            for c in range(6):
                nat.check(lib.jxf_grid3d_get_field(self._h, c, stage[slot][c].data_ptr(), 0, st),
                          "get_field")
            ready = torch.cuda.Event()
            ready.record(main)
            copy_stream.wait_event(ready)
            with torch.cuda.stream(copy_stream):
                for c in range(6):
                    hist[c][s].copy_(stage[slot][c], non_blocking=True)
                slot_free[slot] = torch.cuda.Event()
                slot_free[slot].record(copy_stream)
        if n_steps > done:
            nat.check(lib.jxf_grid3d_step(self._h, n_steps - done, None, st), "jxf_grid3d_step")
        if to_host:
            copy_stream.synchronize()
        self.check(finite=True)
        t = np.array([t_start + k * dt + dt for k in saved], dtype=np.float64)
        gx = np.arange(nx) * dx
        gy = np.arange(ny) * dx
        gz = np.arange(nz) * dx
        if output == "numpy":
            arrs = [h.cpu().numpy() for h in hist]
            return EMFieldHistory3D(t, *arrs, gx, gy, gz)
        if output == "jax":
            import jax.numpy as jnp

            return EMFieldHistory3D(jnp.asarray(t), *[to_jax(h) for h in hist], jnp.asarray(gx),
                                    jnp.asarray(gy), jnp.asarray(gz))
        return EMFieldHistory3D(torch.from_numpy(t), *hist, torch.from_numpy(gx),
                                torch.from_numpy(gy), torch.from_numpy(gz))


FDTD3D = EMGrid3D
