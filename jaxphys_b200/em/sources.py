"""Source waveforms, tabulated on the host in FP64 for the device kernels.

The kernels add ``amplitude * wave[row][n]`` to one field cell after the E
update of step ``n``; this module builds the ``wave`` rows.

* ``"sine"`` -- the reference soft source ``sin(2*pi*f*t_c)`` with
  ``t_c = t_start + n*dt``, the time at the start of the step
  (``src/neurosim/em/fdtd3d.py:227,238,288``; 2D ``src/neurosim/em/fdtd.py:245,260,312``).
* ``"gauss_sine"`` -- extension: Gaussian-modulated sinusoid
  ``exp(-((t_c-t0)/tau)^2) * sin(2*pi*f*(t_c-t0))`` with ``tau = width_steps*dt``
  and ``t0 = delay_steps*dt`` (default delay: four widths).
* ``"table"`` -- extension: explicit per-step values (a ``SampleTable``;
  sample n is the value of step n, zero past the end), e.g. the current
  deposit of a moving charge (``charges.py``).
"""

from __future__ import annotations

import numpy as np


class SampleTable:
    """Per-step source values (float64), compared by identity so that a
    table is one waveform row however many sources share it."""

    __slots__ = ("values",)

    def __init__(self, values):
        self.values = np.ascontiguousarray(values, dtype=np.float64)


def waveform_key(src) -> tuple:
    kind = getattr(src, "waveform", "sine")
    if kind == "table":
        table = getattr(src, "samples", None)
        if not isinstance(table, SampleTable):
            raise ValueError("a 'table' waveform needs samples=SampleTable(values)")
        return ("table", table)
    if kind == "sine":
        return ("sine", float(src.frequency))
    if kind == "gauss_sine":
        width = float(getattr(src, "width_steps", 30.0))
        delay = getattr(src, "delay_steps", None)
        delay = 4.0 * width if delay is None else float(delay)
        return ("gauss_sine", float(src.frequency), width, delay)
    raise ValueError(f"unknown waveform {kind!r}")


def tabulate(key: tuple, n_samples: int, dt: float, t_start: float) -> np.ndarray:
    """Samples of one waveform at absolute steps 0..n_samples-1 (FP64)."""
    if key[0] == "table":
        out = np.zeros(n_samples, dtype=np.float64)
        v = key[1].values[:n_samples]
        out[:len(v)] = v
        return out
    n = np.arange(n_samples, dtype=np.float64)
    t_c = t_start + n * dt
    if key[0] == "sine":
        return np.sin(2.0 * np.pi * key[1] * t_c)
    _, f0, width, delay = key
    tau = width * dt
    u = t_c - delay * dt
    return np.exp(-((u / tau) ** 2)) * np.sin(2.0 * np.pi * f0 * u)


def build_table(keys: list, n_samples: int, dt: float, t_start: float) -> np.ndarray:
    """Row-major float32 [len(keys)][n_samples] table."""
    out = np.zeros((len(keys), n_samples), dtype=np.float32)
    for r, k in enumerate(keys):
        out[r] = tabulate(k, n_samples, dt, t_start).astype(np.float32)
    return out
