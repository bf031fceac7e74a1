"""Driver of the FP64 C oracle (oracle/cpu_fdtd.c) -- TEST INFRASTRUCTURE ONLY.

``Oracle3DC`` has the interface of ``ref_numpy.Oracle3D`` (``f``, ``run``,
``step_idx``) and takes its coefficients from ``ref_numpy`` (so the reference
restatement stays single-sourced); only the stencil loops run in C.
Used by the parity tests for grids where NumPy would take minutes, and by
``bench.py`` as the timed CPU baseline.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import ref_numpy as rn

_LIB = None
MODES = {"absorbing": 0, "periodic": 1, "pec": 2, "cpml": 3}


def lib():
    global _LIB
    if _LIB is None:
        from .build import build

        path = build()
        L = C.CDLL(str(path))
        L.oracle3d_run.restype = C.c_int
        L.oracle3d_run.argtypes = [C.c_int] * 4 + [C.c_double, C.c_void_p, C.c_double, C.c_void_p,
                                                   C.c_void_p, C.c_void_p, C.c_void_p,
                                                   C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                                   C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                                   C.c_int]
        L.oracle_num_threads.restype = C.c_int
        _LIB = L
    return _LIB


def _ptr_array(arrs):
    a = (C.c_void_p * len(arrs))(*[x.ctypes.data for x in arrs])
    return a


class Oracle3DC:
    def __init__(self, spec: rn.Spec3D, dt: float | None = None, t_start: float = 0.0):
        self.spec = spec
        nx, ny, nz = spec.size
        self.shape = (nx, ny, nz)
        self.dt = rn.default_dt_3d(spec.dx) if dt is None else float(dt)
        self.t_start = float(t_start)
        eps = np.ones(self.shape) if spec.eps_r is None else np.asarray(spec.eps_r, np.float64)
        self.a = self.dt / (float(rn.MU0) * spec.dx)
        self.b = self.dt / (float(rn.EPS0) * spec.dx)
        self.cb = np.ascontiguousarray(self.b / eps)
        self.f = [np.zeros(self.shape) for _ in range(6)]
        self.mode = MODES.get(spec.boundary, MODES["pec"])
        self.damp = (np.ascontiguousarray(rn.damping_3d(nx, ny, nz, spec.pml_layers, spec.dx, self.dt))
                     if spec.boundary == "absorbing" else None)
        self.tabs = None
        self.psi = None
        if spec.boundary == "cpml":
            t = [rn.cpml_tables_1d(n, spec.pml_layers, spec.dx, self.dt, spec.cpml)
                 for n in self.shape]
            self.tabs = [np.ascontiguousarray(t[ax][k]) for ax in range(3)
                         for k in ("be", "ce", "ike", "bh", "ch", "ikh")]
            self.psi = [np.zeros(self.shape) for _ in range(12)]
        self.step_idx = 0
        self.src = spec.sources
        self.src_cell = np.array([(s["position"][0] * ny + s["position"][1]) * nz + s["position"][2]
                                  for s in spec.sources], dtype=np.int64)
        self.src_comp = np.array([rn.COMP[s.get("polarization", "z")] for s in spec.sources],
                                 dtype=np.int32)
        self.probe_cell = np.array([(p[0] * ny + p[1]) * nz + p[2] for p in spec.probes],
                                   dtype=np.int64)
        self.probe_comp = np.array([p[3] for p in spec.probes], dtype=np.int32)

    def run(self, n_steps: int) -> dict:
        nx, ny, nz = self.shape
        n_src = len(self.src)
        vals = np.zeros((max(n_steps, 1), max(n_src, 1)))
        cache = {}
        for k, s in enumerate(self.src):
            key = (s.get("kind", "sine"), s.get("frequency"), s.get("width_steps"),
                   s.get("delay_steps"))
            if key not in cache:  # unit-amplitude samples of each distinct waveform
                unit = dict(s, amplitude=1.0)
                cache[key] = rn.waveform_values(unit, n_steps, self.dt, self.t_start,
                                                step0=self.step_idx)
            vals[:n_steps, k] = float(s.get("amplitude", 1.0)) * cache[key]
        vals = np.ascontiguousarray(vals)
        probes = np.zeros((max(n_steps, 1), max(len(self.probe_cell), 1)))
        tab_p = _ptr_array(self.tabs) if self.tabs is not None else None
        psi_p = _ptr_array(self.psi) if self.psi is not None else None
        f_p = _ptr_array(self.f)
        rc = lib().oracle3d_run(nx, ny, nz, self.mode, self.a, self.cb.ctypes.data, 0.0,
                                None if self.damp is None else self.damp.ctypes.data,
                                tab_p, psi_p, f_p, n_src, self.src_cell.ctypes.data,
                                self.src_comp.ctypes.data, vals.ctypes.data,
                                len(self.probe_cell), self.probe_cell.ctypes.data,
                                self.probe_comp.ctypes.data, probes.ctypes.data, n_steps)
        if rc != 0:
            raise RuntimeError(f"oracle3d_run failed ({rc})")
        self.step_idx += n_steps
        return {"probes": probes[:n_steps, :len(self.probe_cell)]}


def num_threads() -> int:
    return lib().oracle_num_threads()
