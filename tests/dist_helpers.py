"""CPU stand-in for the CUDA slab stepper of jaxphys_b200/em/distributed.py
(test infrastructure): the reference update of src/neurosim/em/fdtd3d.py
(305-369, as restated in oracle/ref_numpy.py) on one rank's planes plus ghost
planes, in FP64 NumPy, with the update ranges taken in GLOBAL x."""

from __future__ import annotations

import numpy as np
import torch

from cases import rn


class NumpySlabStepper:
    def __init__(self, size, x0, x1, dx, dt, boundary, pml_layers, cpml):
        nx, ny, nz = size
        if boundary not in (0, 2):  # ABSORBING, PEC
            raise ValueError("the CPU stand-in covers the absorbing and pec boundaries")
        self.gnx, self.x0, self.nloc = nx, x0, x1 - x0
        shape = (self.nloc + 2, ny, nz)
        self.shape = shape
        self.f = [np.zeros(shape) for _ in range(6)]
        self.a = dt / (float(rn.MU0) * dx)
        self.b = dt / (float(rn.EPS0) * dx)
        self.cb = np.full(shape, self.b)
        self.damp = None
        if boundary == 0:
            full = rn.damping_3d(nx, ny, nz, pml_layers, dx, dt)
            self.damp = np.ones(shape)
            self.damp[1:self.nloc + 1] = full[x0:x1]
        self.device = torch.device("cpu")
        self.dtype = torch.float64
        self.src, self.probes = [], []
        self.n_step = 0

    def close(self):
        pass

    def set_eps(self, eps_local):
        self.cb = self.b / np.asarray(eps_local, np.float64)

    def set_sources(self, cell, comp, amp, row):
        self.src = list(zip(cell.tolist(), comp.tolist(), amp.tolist(), row.tolist()))

    def set_waveforms(self, table):
        self.wave = np.asarray(table, np.float64)

    def set_probes(self, cell, comp):
        self.probes = list(zip(cell.tolist(), comp.tolist()))

    def reset(self):
        for a in self.f:
            a[...] = 0.0
        self.n_step = 0

    def get_plane(self, comp, plane):
        return torch.from_numpy(self.f[comp][plane].copy())

    def set_plane(self, comp, plane, t):
        self.f[comp][plane] = t.double().cpu().numpy()

    def new_probe_buffer(self, n_steps, n_local):
        return torch.zeros((n_steps, n_local), dtype=torch.float64)

    def field(self, comp, local_shape):
        return torch.from_numpy(self.f[comp].copy())

    def half_step_part(self, half, part, probe_row=None):
        """Part 1: the plane handed to a neighbour (H: last owned plane, E:
        first owned plane); part 2: the other owned planes (E: then probes and
        the step counter)."""
        if part == 0:
            return self.half_step(half, probe_row)
        b = self.nloc if half == 0 else 1
        if part == 1:
            lo, hi = b, b + 1
        else:
            lo, hi = (1, self.nloc) if half == 0 else (2, self.nloc + 1)
        return self.half_step(half, probe_row, lo, hi, final=(part == 2))

    def half_step(self, half, probe_row=None, lo=None, hi=None, final=True):
        ex, ey, ez, hx, hy, hz = self.f
        a, cb = self.a, self.cb
        full = lo is None
        if full:
            lo, hi = 1, self.nloc + 1                   # owned local planes
        glob = lambda p: p + self.x0 - 1                 # noqa: E731
        if half == 0:
            L = slice(lo, hi)
            hx[L, :-1, :-1] = hx[L, :-1, :-1] - a * (
                (ez[L, 1:, :-1] - ez[L, :-1, :-1]) - (ey[L, :-1, 1:] - ey[L, :-1, :-1]))
            for p in range(lo, hi):
                if glob(p) < self.gnx - 1:
                    hy[p, :, :-1] = hy[p, :, :-1] - a * (
                        (ex[p, :, 1:] - ex[p, :, :-1]) - (ez[p + 1, :, :-1] - ez[p, :, :-1]))
                    hz[p, :-1, :] = hz[p, :-1, :] - a * (
                        (ey[p + 1, :-1, :] - ey[p, :-1, :]) - (ex[p, 1:, :] - ex[p, :-1, :]))
            return
        L = slice(lo, hi)
        ex[L, 1:, 1:] = ex[L, 1:, 1:] + cb[L, 1:, 1:] * (
            (hz[L, 1:, 1:] - hz[L, :-1, 1:]) - (hy[L, 1:, 1:] - hy[L, 1:, :-1]))
        for p in range(lo, hi):
            if glob(p) >= 1:
                ey[p, :, 1:] = ey[p, :, 1:] + cb[p, :, 1:] * (
                    (hx[p, :, 1:] - hx[p, :, :-1]) - (hz[p, :, 1:] - hz[p - 1, :, 1:]))
                ez[p, 1:, :] = ez[p, 1:, :] + cb[p, 1:, :] * (
                    (hy[p, 1:, :] - hy[p - 1, 1:, :]) - (hx[p, 1:, :] - hx[p, :-1, :]))
        if self.damp is not None:
            for c in (ex, ey, ez):
                c[L] = c[L] * self.damp[L]
        flat = [c.reshape(-1) for c in (ex, ey, ez, hx, hy, hz)]
        plane = self.shape[1] * self.shape[2]
        for cell, comp, amp, row in self.src:
            if lo <= cell // plane < hi:
                flat[comp][cell] += amp * self.wave[row, self.n_step]
        if not final:
            return
        if probe_row is not None:
            for k, (cell, comp) in enumerate(self.probes):
                probe_row[k] = float(flat[comp][cell])
        self.n_step += 1


class NumpyWholeStepSlabStepper(NumpySlabStepper):
    """Whole steps as a TMA slab takes them: H on the owned planes and on the
    low ghost plane (a replica of the previous rank's last plane, from the
    ghost E plane received before the step; skipped when that plane lies
    outside the grid), then E on the owned planes only."""

    whole_steps = True

    def step(self, probe_row=None):
        beg = 0 if self.x0 >= 1 else 1
        self.half_step(0, None, beg, self.nloc + 1)
        self.half_step(1, probe_row)


def free_port() -> int:
    import socket

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port
