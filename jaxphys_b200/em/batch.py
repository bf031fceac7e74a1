"""Batches of independent 3D grids advanced together (extension).

``FDTDBatch(grids)`` takes ``EMGrid3D`` objects of any mix of sizes and one
boundary mode, all on one kernel path, and advances all of them together (C
ABI ``jxf_batch3d_*``):

* TMA path (nz % 4 == 0; ``path="auto"`` or ``"tma"``): one persistent launch
  per step (and per CPML part) over a work list of every grid's
  (tile, x-chunk) blocks, heaviest first; blocks take work through an atomic
  counter.  The launch shape (tile, chunk, single-axis CPML split) is tuned
  per batch on the first run.  Every grid must hold its state in the same
  buffer set (same step parity), and all or none carry a permittivity map.
* generic path: one kernel per phase per step over the whole batch (any
  shape, odd nz included).

``run(n)`` captures the n-step sequence once into a CUDA graph and replays it
with a single launch.  Each grid keeps its own permittivity, sources, probes
and field accessors.  Typical use: many design candidates, or many source
positions, of one device.
"""

from __future__ import annotations

import ctypes as C

from .. import _native as nat
from ..exceptions import ConfigurationError


class FDTDBatch:
    def __init__(self, grids):
        if not grids:
            raise ConfigurationError("empty batch")
        paths = set()
        for g in grids:
            if g._h is None:
                g.prepare(g._dt, g._t_start)
            elif g._dirty:
                g._upload_config()
            paths.add(g.info()["path"])
        if len(paths) != 1:
            raise ConfigurationError("batched grids must all use one kernel path (build them "
                                     "with the same path=)")
        self.path = "tma" if paths == {nat.PATH_TMA} else "generic"
        self.grids = list(grids)
        lib = nat.load()
        arr = (C.c_void_p * len(grids))(*[g._h for g in grids])
        h = C.c_void_p()
        nat.check(lib.jxf_batch3d_create(len(grids), arr, C.byref(h)), "jxf_batch3d_create")
        self._h = h
        self._last_n = 0
        self.band = None
        learned = [g for g in grids if g._boundary == "learned"]
        if learned:
            if len(learned) != len(grids) or any(g._band is not learned[0]._band for g in learned):
                raise ConfigurationError("a batch with learned boundaries needs every grid "
                                         "learned, with one shared band")
            self.set_band(learned[0]._band)

    def set_band(self, model) -> None:
        """Attach a learned absorbing band (``LearnedBand``; PEC grids only)
        applied after every step; ``None`` detaches it."""
        nat.check(nat.load().jxf_batch3d_set_band(self._h, None if model is None else model._h),
                  "jxf_batch3d_set_band")
        self.band = model

    def kernels_per_step(self) -> int:
        """Kernel launches per leapfrog step of the last run's shape."""
        return int(nat.load().jxf_batch3d_kernels_per_step(self._h))

    def launch(self) -> dict:
        """Launch shape of a TMA batch: registry entry, x chunk, single-axis
        split (all -1 on the generic path)."""
        v = (C.c_int32 * 3)()
        nat.check(nat.load().jxf_batch3d_launch(self._h, v), "jxf_batch3d_launch")
        return {"tma_config": v[0], "x_chunk": v[1], "axis_split": v[2]}

    def close(self):
        if self._h is not None:
            nat.load().jxf_batch3d_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def reset(self):
        nat.check(nat.load().jxf_batch3d_reset(self._h, nat.stream_handle()), "batch reset")

    @property
    def cells(self) -> int:
        return sum(g.size[0] * g.size[1] * g.size[2] for g in self.grids)

    def run(self, n_steps: int, use_graph: bool = True):
        """Advance every grid by n_steps; returns the probe traces of each grid
        (device tensors (n_steps, P_g), None for grids without probes)."""
        import torch

        for g in self.grids:
            if g._dirty:
                g._upload_config()
            if g._sources:
                g._ensure_waves(g.step_count + int(n_steps))
        nat.check(nat.load().jxf_batch3d_step(self._h, int(n_steps), 1 if use_graph else 0,
                                              nat.stream_handle()), "jxf_batch3d_step")
        out = []
        for i, g in enumerate(self.grids):
            if not g._probes:
                out.append(None)
                continue
            t = torch.empty((int(n_steps), len(g._probes)), dtype=torch.float32,
                            device=f"cuda:{g._h_key[1]}")
            nat.check(nat.load().jxf_batch3d_probes(self._h, i, int(n_steps), t.data_ptr(),
                                                    nat.stream_handle()), "batch probes")
            out.append(t)
        return out
