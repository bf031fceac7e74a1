"""CPU oracle for the FDTD hot path: a line-for-line NumPy restatement.

TEST INFRASTRUCTURE ONLY.  Nothing in the product package imports this
module; only ``tests/``, ``__graft_entry__.smoke()`` and the CPU legs of
``bench.py`` use it, and only as the checker / CPU baseline.

What it restates (paths relative to the jaxphys project root):

* 3D Yee solver, ``src/neurosim/em/fdtd3d.py``
    - constants                 ``:36-38``
    - ``_build_epsilon_r``      ``:132-137``
    - ``_build_pml_sigma_3d``   ``:139-167``
    - dt / n_steps              ``:189-195``
    - coefficients              ``:219-224``
    - ``add_sources``           ``:233-245``
    - periodic curls            ``:249-278,290-301``
    - absorbing step body       ``:303-366``
    - subsample + time axis     ``:371-404``
* 2D TM solver, ``src/neurosim/em/fdtd.py``
    - conductor mask            ``:144-157``
    - ``_build_pml_sigma``      ``:159-191``
    - dt                        ``:214``
    - edge rules                ``:264-302``
    - step body                 ``:304-357``
    - subsample                 ``:371-377``

The reference keeps the full per-step history (``jax.lax.scan`` emits all
fields every step) and subsamples afterwards; this restatement keeps only the
frames that survive the subsample, which gives identical values without the
O(n_steps * N^3) memory.

Extensions with no reference implementation (their semantics are defined by
this file and by the CUDA path together):

* ``boundary="cpml"``: convolutional PML (Roden & Gedney 2000; Taflove &
  Hagness 3rd ed. ch. 7) with polynomial grading ``m`` and reflection ``R0``,
  optional kappa / CFS alpha, applied with the reference's own stencil index
  ranges (no damping multiply).
* Gaussian-modulated sinusoid source waveform.
* Field probes: value of one component at one cell after every step.
* Per-cell relative permittivity array (instead of boolean masks).

Parity of this restatement with the reference source is pinned by
``tests/golden`` (fixtures produced by executing the reference's own
``fdtd3d.py`` / ``fdtd.py`` on a NumPy-backed stand-in for ``jax.numpy``).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# fdtd3d.py:36-38 / fdtd.py:39-41
C0 = 299792458.0
MU0 = 4.0e-7 * np.pi
EPS0 = 1.0 / (MU0 * C0**2)
ETA0 = math.sqrt(MU0 / EPS0)

COMP = {"x": 0, "y": 1, "z": 2}


# --------------------------------------------------------------------------
# Waveforms
# --------------------------------------------------------------------------


def waveform_values(src: dict, n_steps: int, dt: float, t_start: float,
                    step0: int = 0) -> np.ndarray:
    """Source value at steps step0..step0+n_steps-1, FP64.

    ``kind="sine"`` is the reference soft source, fdtd3d.py:227,238:
    ``amplitude * sin(2*pi*f * t_c)`` with ``t_c = t_start + idx*dt``
    (fdtd3d.py:288) -- the time at the *start* of the step, added after the
    E update.

    ``kind="gauss_sine"`` (extension): ``amplitude * exp(-((t_c-t0)/tau)^2)
    * sin(2*pi*f0*(t_c-t0))`` with ``tau = width_steps*dt`` and
    ``t0 = delay_steps*dt``.
    """
    idx = np.arange(step0, step0 + n_steps, dtype=np.float64)
    t_c = t_start + idx * dt
    amp = float(src.get("amplitude", 1.0))
    kind = src.get("kind", "sine")
    if kind == "sine":
        omega = 2.0 * np.pi * float(src["frequency"])
        return amp * np.sin(omega * t_c)
    if kind == "gauss_sine":
        f0 = float(src["frequency"])
        tau = float(src["width_steps"]) * dt
        t0 = float(src["delay_steps"]) * dt
        u = t_c - t0
        return amp * (np.exp(-((u / tau) ** 2)) * np.sin(2.0 * np.pi * f0 * u))
    if kind == "table":
        # extension: explicit per-step values (sample n is added at step n;
        # zero past the end of the table)
        samples = np.asarray(src["samples"], dtype=np.float64)
        out = np.zeros(n_steps, dtype=np.float64)
        lo, hi = step0, min(step0 + n_steps, len(samples))
        if hi > lo:
            out[:hi - lo] = samples[lo:hi]
        return amp * out
    raise ValueError(f"unknown waveform kind {kind!r}")


# --------------------------------------------------------------------------
# Coefficients
# --------------------------------------------------------------------------


def default_dt_3d(dx: float) -> float:
    """fdtd3d.py:190-192."""
    return float(0.99 * dx / (C0 * float(np.sqrt(3.0))))


def default_dt_2d(dx: float) -> float:
    """fdtd.py:214."""
    return float(0.99 * dx / (C0 * float(np.sqrt(2.0))))


def n_steps_from_span(t_span, dt) -> int:
    """fdtd3d.py:194-195 (floor of the span over dt)."""
    t_start, t_end = t_span
    return int((t_end - t_start) / dt)


def pml_sigma_1d(n: int, n_pml: int, dx: float) -> np.ndarray:
    """fdtd3d.py:149-157 (``build_1d``); fdtd.py:173-189 is the same profile.

    Cubic grading from ``sigma_max = 0.8*4/dx`` at the outer cell; the later
    write wins where the two faces overlap, as in the reference loop.
    """
    s = np.zeros(n)
    if n_pml == 0:
        return s
    sigma_max = 0.8 * 4.0 / (dx * 1.0)
    for i in range(n_pml):
        val = sigma_max * ((n_pml - i) / n_pml) ** 3
        s[i] = val
        s[n - 1 - i] = val
    return s


def build_eps_r(shape, materials) -> np.ndarray:
    """fdtd3d.py:132-137: ones, then ``where(mask, eps, prev)`` in order."""
    eps = np.ones(shape)
    for mask, eps_val in materials:
        eps = np.where(np.asarray(mask, dtype=bool), eps_val, eps)
    return eps


def damping_3d(nx, ny, nz, n_pml, dx, dt) -> np.ndarray:
    """fdtd3d.py:220-221,363: ``exp(-sigma_avg*dt/EPS0)`` on the full grid."""
    sx = pml_sigma_1d(nx, n_pml, dx)[:, None, None]
    sy = pml_sigma_1d(ny, n_pml, dx)[None, :, None]
    sz = pml_sigma_1d(nz, n_pml, dx)[None, None, :]
    sigma_avg = (np.broadcast_to(sx, (nx, ny, nz)) + np.broadcast_to(sy, (nx, ny, nz))
                 + np.broadcast_to(sz, (nx, ny, nz))) / 3.0
    return np.exp(-sigma_avg * dt / float(EPS0))


def damping_2d(nx, ny, n_pml, dx, dt) -> np.ndarray:
    """fdtd.py:173-191,242,344 (note ``sigma_max`` divides by sqrt(1.0))."""
    if n_pml == 0:
        sig = np.zeros((nx, ny))
        return np.exp(-sig * dt / float(EPS0))
    sigma_max = 0.8 * (3 + 1) / (dx * np.sqrt(1.0))
    sx = np.zeros(nx)
    sy = np.zeros(ny)
    for i in range(n_pml):
        val = sigma_max * ((n_pml - i) / n_pml) ** 3
        sx[i] = val
        sx[nx - 1 - i] = val
        sy[i] = val
        sy[ny - 1 - i] = val
    sigma_avg = 0.5 * (sx[:, None] + sy[None, :])
    return np.exp(-sigma_avg * dt / float(EPS0))


@dataclass
class CpmlParams:
    """Extension: CPML grading (Taflove & Hagness eq. 7.60, 7.79, 7.102)."""

    order: float = 3.0          # m
    r0: float = 1e-6            # target normal-incidence reflection
    kappa_max: float = 1.0
    alpha_max: float = 0.0      # CFS alpha (S/m); 0 = plain CPML


def cpml_tables_1d(n: int, n_pml: int, dx: float, dt: float, p: CpmlParams):
    """1D CPML coefficient tables for one axis of length ``n``.

    Returns dict with b/c/inverse-kappa for E positions (integer index ``i``)
    and H positions (``i + 1/2``).  Depth into the layer, in [0, 1]:
    ``(n_pml - x)/n_pml`` on the low face, ``(x - (n-1-n_pml))/n_pml`` on the
    high face, 0 in the interior; the two faces are mirror images about
    ``(n-1)/2``.  ``sigma = sigma_max * rho^m`` with
    ``sigma_max = -(m+1) ln(R0) / (2 eta0 n_pml dx)``;
    ``kappa = 1 + (kappa_max-1) rho^m``; ``alpha = alpha_max (1 - rho)``;
    ``b = exp(-(sigma/kappa + alpha) dt/eps0)``;
    ``c = sigma (b-1) / (sigma kappa + kappa^2 alpha)`` (0 where sigma is 0).
    """
    out = {}
    for name, off in (("e", 0.0), ("h", 0.5)):
        x = np.arange(n, dtype=np.float64) + off
        if n_pml > 0:
            lo = (n_pml - x) / n_pml
            hi = (x - (n - 1 - n_pml)) / n_pml
            rho = np.clip(np.maximum(lo, hi), 0.0, 1.0)
            sigma_max = -(p.order + 1.0) * math.log(p.r0) / (2.0 * ETA0 * n_pml * dx)
        else:
            rho = np.zeros(n)
            sigma_max = 0.0
        sigma = sigma_max * rho**p.order
        kappa = 1.0 + (p.kappa_max - 1.0) * rho**p.order
        alpha = p.alpha_max * (1.0 - rho)
        alpha = np.where(rho > 0.0, alpha, 0.0)
        b = np.exp(-(sigma / kappa + alpha) * dt / EPS0)
        denom = sigma * kappa + kappa**2 * alpha
        c = np.where(sigma > 0.0, sigma * (b - 1.0) / np.where(denom > 0, denom, 1.0), 0.0)
        out["b" + name] = b
        out["c" + name] = c
        out["ik" + name] = 1.0 / kappa
    return out


# --------------------------------------------------------------------------
# 3D
# --------------------------------------------------------------------------


@dataclass
class Spec3D:
    """One 3D run.  ``sources`` entries: dict(position=(ix,iy,iz),
    polarization='x'|'y'|'z', amplitude, kind='sine'|'gauss_sine',
    frequency, width_steps, delay_steps).  ``probes``: list of
    (ix, iy, iz, comp) with comp 0..5 = ex,ey,ez,hx,hy,hz."""

    size: tuple
    dx: float = 0.01
    boundary: str = "absorbing"         # absorbing | periodic | pec | cpml
    pml_layers: int = 8
    eps_r: np.ndarray | None = None     # per-cell relative permittivity
    sources: list = field(default_factory=list)
    probes: list = field(default_factory=list)
    cpml: CpmlParams = field(default_factory=CpmlParams)


def _curl_e_periodic(ex, ey, ez):
    """fdtd3d.py:249-264."""
    cx = (np.roll(ez, -1, axis=1) - ez) - (np.roll(ey, -1, axis=2) - ey)
    cy = (np.roll(ex, -1, axis=2) - ex) - (np.roll(ez, -1, axis=0) - ez)
    cz = (np.roll(ey, -1, axis=0) - ey) - (np.roll(ex, -1, axis=1) - ex)
    return cx, cy, cz


def _curl_h_periodic(hx, hy, hz):
    """fdtd3d.py:266-278."""
    cx = (hz - np.roll(hz, 1, axis=1)) - (hy - np.roll(hy, 1, axis=2))
    cy = (hx - np.roll(hx, 1, axis=2)) - (hz - np.roll(hz, 1, axis=0))
    cz = (hy - np.roll(hy, 1, axis=0)) - (hx - np.roll(hx, 1, axis=1))
    return cx, cy, cz


class Oracle3D:
    """Stateful FP64 (or FP32) stepping of one 3D grid."""

    def __init__(self, spec: Spec3D, dt: float | None = None, t_start: float = 0.0,
                 dtype=np.float64):
        self.spec = spec
        nx, ny, nz = spec.size
        self.shape = (nx, ny, nz)
        self.dtype = dtype
        self.dt = default_dt_3d(spec.dx) if dt is None else float(dt)
        self.t_start = float(t_start)
        dx = spec.dx
        eps_r = np.ones(self.shape) if spec.eps_r is None else np.asarray(spec.eps_r, np.float64)
        # fdtd3d.py:223-224
        self.a = self.dt / (float(MU0) * dx)
        self.b = self.dt / (float(EPS0) * dx)
        self.cb = (self.b / eps_r).astype(dtype)
        self.f = [np.zeros(self.shape, dtype) for _ in range(6)]
        self.step_idx = 0
        if spec.boundary == "absorbing":
            self.damp = damping_3d(nx, ny, nz, spec.pml_layers, dx, self.dt).astype(dtype)
        else:
            self.damp = None
        if spec.boundary == "cpml":
            self.tab = [cpml_tables_1d(n, spec.pml_layers, dx, self.dt, spec.cpml)
                        for n in self.shape]
            self.psi = {k: np.zeros(self.shape, dtype) for k in
                        ("hxy", "hxz", "hyz", "hyx", "hzx", "hzy",
                         "exy", "exz", "eyz", "eyx", "ezx", "ezy")}
        self.src = [(tuple(s["position"]), COMP[s.get("polarization", "z")], s)
                    for s in spec.sources]

    # fdtd3d.py:233-245
    def _add_sources(self, n: int):
        ex, ey, ez = self.f[0], self.f[1], self.f[2]
        comps = (ex, ey, ez)
        for (ix, iy, iz), c, s in self.src:
            val = waveform_values(s, 1, self.dt, self.t_start, step0=n)[0]
            comps[c][ix, iy, iz] += self.dtype(val)

    def step(self):
        ex, ey, ez, hx, hy, hz = self.f
        a, cb = self.dtype(self.a), self.cb
        bnd = self.spec.boundary
        n = self.step_idx
        if bnd == "periodic":
            # fdtd3d.py:290-301
            cx, cy, cz = _curl_e_periodic(ex, ey, ez)
            hx = hx - a * cx
            hy = hy - a * cy
            hz = hz - a * cz
            cx, cy, cz = _curl_h_periodic(hx, hy, hz)
            ex = ex + cb * cx
            ey = ey + cb * cy
            ez = ez + cb * cz
        elif bnd != "cpml":
            # fdtd3d.py:305-359 (in-place slices reproduce .at[].set); any
            # boundary string other than periodic runs this stencil, and
            # only "absorbing" damps (fdtd3d.py:362).
            hx = hx.copy(); hy = hy.copy(); hz = hz.copy()
            hx[:, :-1, :-1] = hx[:, :-1, :-1] - a * (
                (ez[:, 1:, :-1] - ez[:, :-1, :-1]) - (ey[:, :-1, 1:] - ey[:, :-1, :-1]))
            hy[:-1, :, :-1] = hy[:-1, :, :-1] - a * (
                (ex[:-1, :, 1:] - ex[:-1, :, :-1]) - (ez[1:, :, :-1] - ez[:-1, :, :-1]))
            hz[:-1, :-1, :] = hz[:-1, :-1, :] - a * (
                (ey[1:, :-1, :] - ey[:-1, :-1, :]) - (ex[:-1, 1:, :] - ex[:-1, :-1, :]))
            ex = ex.copy(); ey = ey.copy(); ez = ez.copy()
            ex[:, 1:, 1:] = ex[:, 1:, 1:] + cb[:, 1:, 1:] * (
                (hz[:, 1:, 1:] - hz[:, :-1, 1:]) - (hy[:, 1:, 1:] - hy[:, 1:, :-1]))
            ey[1:, :, 1:] = ey[1:, :, 1:] + cb[1:, :, 1:] * (
                (hx[1:, :, 1:] - hx[1:, :, :-1]) - (hz[1:, :, 1:] - hz[:-1, :, 1:]))
            ez[1:, 1:, :] = ez[1:, 1:, :] + cb[1:, 1:, :] * (
                (hy[1:, 1:, :] - hy[:-1, 1:, :]) - (hx[1:, 1:, :] - hx[1:, :-1, :]))
            if bnd == "absorbing":
                # fdtd3d.py:361-366
                ex = ex * self.damp
                ey = ey * self.damp
                ez = ez * self.damp
        else:
            ex, ey, ez, hx, hy, hz = self._step_cpml(ex, ey, ez, hx, hy, hz)
        self.f = [ex, ey, ez, hx, hy, hz]
        self._add_sources(n)                       # fdtd3d.py:369
        self.step_idx += 1

    def _step_cpml(self, ex, ey, ez, hx, hy, hz):
        """Extension: reference stencil + CPML psi recurrences.

        H (psi_Hxy etc. use H-position tables of the differencing axis):
          Hx -= a*(ik_y*dEz/dy - ik_z*dEy/dz + psi_hxy - psi_hxz)
          Hy -= a*(ik_z*dEx/dz - ik_x*dEz/dx + psi_hyz - psi_hyx)
          Hz -= a*(ik_x*dEy/dx - ik_y*dEx/dy + psi_hzx - psi_hzy)
        with psi <- b*psi + c*d (d = the raw neighbour difference).
        E (E-position tables):
          Ex += cb*(ik_y*dHz/dy - ik_z*dHy/dz + psi_exy - psi_exz)
          Ey += cb*(ik_z*dHx/dz - ik_x*dHz/dx + psi_eyz - psi_eyx)
          Ez += cb*(ik_x*dHy/dx - ik_y*dHx/dy + psi_ezx - psi_ezy)
        """
        dt_ = self.dtype
        a, cb = dt_(self.a), self.cb
        tx, ty, tz = self.tab
        P = self.psi

        def t(tab, key, axis):
            v = tab[key].astype(dt_)
            shp = [1, 1, 1]
            shp[axis] = -1
            return v.reshape(shp)

        hx = hx.copy(); hy = hy.copy(); hz = hz.copy()
        # Hx on [:, :-1, :-1]
        dy = ez[:, 1:, :-1] - ez[:, :-1, :-1]
        dz = ey[:, :-1, 1:] - ey[:, :-1, :-1]
        s = (slice(None), slice(0, -1), slice(0, -1))
        P["hxy"][s] = t(ty, "bh", 1)[:, :-1] * P["hxy"][s] + t(ty, "ch", 1)[:, :-1] * dy
        P["hxz"][s] = t(tz, "bh", 2)[:, :, :-1] * P["hxz"][s] + t(tz, "ch", 2)[:, :, :-1] * dz
        hx[s] = hx[s] - a * ((t(ty, "ikh", 1)[:, :-1] * dy - t(tz, "ikh", 2)[:, :, :-1] * dz)
                             + (P["hxy"][s] - P["hxz"][s]))
        # Hy on [:-1, :, :-1]
        dz = ex[:-1, :, 1:] - ex[:-1, :, :-1]
        dx = ez[1:, :, :-1] - ez[:-1, :, :-1]
        s = (slice(0, -1), slice(None), slice(0, -1))
        P["hyz"][s] = t(tz, "bh", 2)[:, :, :-1] * P["hyz"][s] + t(tz, "ch", 2)[:, :, :-1] * dz
        P["hyx"][s] = t(tx, "bh", 0)[:-1] * P["hyx"][s] + t(tx, "ch", 0)[:-1] * dx
        hy[s] = hy[s] - a * ((t(tz, "ikh", 2)[:, :, :-1] * dz - t(tx, "ikh", 0)[:-1] * dx)
                             + (P["hyz"][s] - P["hyx"][s]))
        # Hz on [:-1, :-1, :]
        dx = ey[1:, :-1, :] - ey[:-1, :-1, :]
        dy = ex[:-1, 1:, :] - ex[:-1, :-1, :]
        s = (slice(0, -1), slice(0, -1), slice(None))
        P["hzx"][s] = t(tx, "bh", 0)[:-1] * P["hzx"][s] + t(tx, "ch", 0)[:-1] * dx
        P["hzy"][s] = t(ty, "bh", 1)[:, :-1] * P["hzy"][s] + t(ty, "ch", 1)[:, :-1] * dy
        hz[s] = hz[s] - a * ((t(tx, "ikh", 0)[:-1] * dx - t(ty, "ikh", 1)[:, :-1] * dy)
                             + (P["hzx"][s] - P["hzy"][s]))

        ex = ex.copy(); ey = ey.copy(); ez = ez.copy()
        # Ex on [:, 1:, 1:]
        dy = hz[:, 1:, 1:] - hz[:, :-1, 1:]
        dz = hy[:, 1:, 1:] - hy[:, 1:, :-1]
        s = (slice(None), slice(1, None), slice(1, None))
        P["exy"][s] = t(ty, "be", 1)[:, 1:] * P["exy"][s] + t(ty, "ce", 1)[:, 1:] * dy
        P["exz"][s] = t(tz, "be", 2)[:, :, 1:] * P["exz"][s] + t(tz, "ce", 2)[:, :, 1:] * dz
        ex[s] = ex[s] + cb[s] * ((t(ty, "ike", 1)[:, 1:] * dy - t(tz, "ike", 2)[:, :, 1:] * dz)
                                 + (P["exy"][s] - P["exz"][s]))
        # Ey on [1:, :, 1:]
        dz = hx[1:, :, 1:] - hx[1:, :, :-1]
        dx = hz[1:, :, 1:] - hz[:-1, :, 1:]
        s = (slice(1, None), slice(None), slice(1, None))
        P["eyz"][s] = t(tz, "be", 2)[:, :, 1:] * P["eyz"][s] + t(tz, "ce", 2)[:, :, 1:] * dz
        P["eyx"][s] = t(tx, "be", 0)[1:] * P["eyx"][s] + t(tx, "ce", 0)[1:] * dx
        ey[s] = ey[s] + cb[s] * ((t(tz, "ike", 2)[:, :, 1:] * dz - t(tx, "ike", 0)[1:] * dx)
                                 + (P["eyz"][s] - P["eyx"][s]))
        # Ez on [1:, 1:, :]
        dx = hy[1:, 1:, :] - hy[:-1, 1:, :]
        dy = hx[1:, 1:, :] - hx[1:, :-1, :]
        s = (slice(1, None), slice(1, None), slice(None))
        P["ezx"][s] = t(tx, "be", 0)[1:] * P["ezx"][s] + t(tx, "ce", 0)[1:] * dx
        P["ezy"][s] = t(ty, "be", 1)[:, 1:] * P["ezy"][s] + t(ty, "ce", 1)[:, 1:] * dy
        ez[s] = ez[s] + cb[s] * ((t(tx, "ike", 0)[1:] * dx - t(ty, "ike", 1)[:, 1:] * dy)
                                 + (P["ezx"][s] - P["ezy"][s]))
        return ex, ey, ez, hx, hy, hz

    def probe_values(self):
        return np.array([self.f[c][ix, iy, iz] for (ix, iy, iz, c) in self.spec.probes],
                        dtype=np.float64)

    def run(self, n_steps: int, save_every: int | None = None):
        """Step ``n_steps`` times.  Returns dict with ``probes`` (n_steps, P)
        and, if ``save_every`` is given, the reference subsample
        (fdtd3d.py:396-404): frames after steps 1, 1+s, 1+2s, ... and their
        times ``t_c + dt`` (fdtd3d.py:378)."""
        probes = np.zeros((n_steps, len(self.spec.probes)))
        frames = {k: [] for k in ("ex", "ey", "ez", "hx", "hy", "hz")}
        times = []
        s = 1 if (save_every is None or save_every <= 1) else save_every
        for k in range(n_steps):
            t_c = self.t_start + self.step_idx * self.dt
            self.step()
            if self.spec.probes:
                probes[k] = self.probe_values()
            if save_every is not None and k % s == 0:
                for name, arr in zip(frames, self.f):
                    frames[name].append(arr.copy())
                times.append(t_c + self.dt)
        out = {"probes": probes}
        if save_every is not None:
            for name in frames:
                out[name] = (np.stack(frames[name]) if frames[name]
                             else np.zeros((0,) + self.shape, self.dtype))
            out["t"] = np.asarray(times, dtype=np.float64)
        return out


# --------------------------------------------------------------------------
# 2D (TM: Ez, Hx, Hy)
# --------------------------------------------------------------------------


@dataclass
class Spec2D:
    """One 2D run.  ``sources``: list of dict(frequency, y, amplitude)
    (reference ``PlaneWave``, fdtd.py:45-56).  ``walls``: list of
    (y, gap_start, gap_end) (reference ``Wall``, fdtd.py:60-71)."""

    size: tuple
    dx: float = 0.01
    boundary: str = "absorbing"     # absorbing | periodic | reflecting
    pml_layers: int = 10
    sources: list = field(default_factory=list)
    walls: list = field(default_factory=list)


def conductor_mask_2d(nx, ny, walls) -> np.ndarray:
    """fdtd.py:144-157."""
    mask = np.zeros((nx, ny), dtype=bool)
    for (y, g0, g1) in walls:
        row = np.ones(nx, dtype=bool)
        if g0 is not None and g1 is not None:
            gap = np.arange(nx)
            row = (gap < g0) | (gap >= g1)
        mask[:, y] = row
    return mask


def _edges_reflecting(f):
    """fdtd.py:268-271 (sequential: later rows/cols see earlier writes)."""
    f = f.copy()
    f[0, :] = f[1, :]
    f[-1, :] = f[-2, :]
    f[:, 0] = f[:, 1]
    f[:, -1] = f[:, -2]
    return f


def _edges_periodic(f):
    """fdtd.py:288-291."""
    f = f.copy()
    f[0, :] = f[-2, :]
    f[-1, :] = f[1, :]
    f[:, 0] = f[:, -2]
    f[:, -1] = f[:, 1]
    return f


class Oracle2D:
    def __init__(self, spec: Spec2D, dt: float | None = None, t_start: float = 0.0,
                 dtype=np.float64):
        self.spec = spec
        nx, ny = spec.size
        self.shape = (nx, ny)
        self.dtype = dtype
        self.dt = default_dt_2d(spec.dx) if dt is None else float(dt)
        self.t_start = float(t_start)
        dx = spec.dx
        self.a = self.dt / (float(MU0) * dx)       # fdtd.py:254
        self.b = self.dt / (float(EPS0) * dx)      # fdtd.py:255
        self.ez = np.zeros(self.shape, dtype)
        self.hx = np.zeros(self.shape, dtype)
        self.hy = np.zeros(self.shape, dtype)
        self.mask = conductor_mask_2d(nx, ny, spec.walls)
        self.damp = damping_2d(nx, ny, spec.pml_layers, dx, self.dt).astype(dtype)
        self.step_idx = 0

    def step(self):
        """fdtd.py:304-357."""
        ez, hx, hy = self.ez, self.hx, self.hy
        a, b = self.dtype(self.a), self.dtype(self.b)
        bnd = self.spec.boundary
        n = self.step_idx
        if bnd == "periodic":
            hx = hx - a * (np.roll(ez, -1, axis=1) - ez)
            hy = hy + a * (np.roll(ez, -1, axis=0) - ez)
            dhy = hy - np.roll(hy, 1, axis=0)
            dhx = hx - np.roll(hx, 1, axis=1)
            ez = ez + b * (dhy - dhx)
        else:
            hx = hx.copy(); hy = hy.copy(); ez = ez.copy()
            hx[:, :-1] = hx[:, :-1] - a * (ez[:, 1:] - ez[:, :-1])
            hy[:-1, :] = hy[:-1, :] + a * (ez[1:, :] - ez[:-1, :])
            dhy = hy[1:, :] - hy[:-1, :]
            dhx = hx[:, 1:] - hx[:, :-1]
            ez[1:, 1:] = ez[1:, 1:] + b * (dhy[:, 1:] - dhx[1:, :])
        if bnd == "absorbing":
            ez = ez * self.damp
        elif bnd == "reflecting":
            ez, hx, hy = _edges_reflecting(ez), _edges_reflecting(hx), _edges_reflecting(hy)
        elif bnd == "periodic":
            ez, hx, hy = _edges_periodic(ez), _edges_periodic(hx), _edges_periodic(hy)
        # fdtd.py:257-262,354
        for s in self.spec.sources:
            val = waveform_values(s, 1, self.dt, self.t_start, step0=n)[0]
            ez[:, int(s["y"])] += self.dtype(val)
        ez = np.where(self.mask, self.dtype(0.0), ez)   # fdtd.py:357
        self.ez, self.hx, self.hy = ez, hx, hy
        self.step_idx += 1

    def run(self, n_steps: int, save_every: int | None = None):
        frames = {"ez": [], "hx": [], "hy": []}
        times = []
        s = 1 if (save_every is None or save_every <= 1) else save_every
        for k in range(n_steps):
            t_c = self.t_start + self.step_idx * self.dt
            self.step()
            if save_every is not None and k % s == 0:
                frames["ez"].append(self.ez.copy())
                frames["hx"].append(self.hx.copy())
                frames["hy"].append(self.hy.copy())
                times.append(t_c + self.dt)
        out = {}
        if save_every is not None:
            for k in frames:
                out[k] = (np.stack(frames[k]) if frames[k]
                          else np.zeros((0,) + self.shape, self.dtype))
            out["t"] = np.asarray(times)
        return out


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = float(np.sqrt(np.sum(b * b)))
    num = float(np.sqrt(np.sum((a - b) ** 2)))
    return num / den if den > 0 else num
