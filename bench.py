"""Throughput benchmark of the 3D FDTD hot path (Gcell-updates/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c2|c1|c3|c5]

A bench step is one complete simulation of the workload: zero the fields,
run all its leapfrog steps with probe recording.  Default workload (c2):
128^3 cells, FP32, 1000 leapfrog steps, 10-cell CPML (m=3, R0=1e-6),
eps_r=4 sphere of radius 20 cells at a seeded offset, Gaussian-modulated Ez
dipole at the centre (f0 = 0.05/dt, width 30 steps), 16 seeded Ez probes.
Inputs are synthetic (seeded); no dataset is involved.

`value` times the device work with the inputs resident in HBM; `e2e` times
the same simulation through the public Python API with host buffers (the
permittivity map goes in from pinned host memory, the probe traces come
back to the host) every step.  L2 is flushed (a 256 MiB write) between timed
steps; each step is bracketed by CUDA events on the launching stream.

--impl reference times the CPU restatement of the reference algorithm
(oracle/cpu_fdtd.c, FP64, every host thread) on a bounded sample of the
same workload; under torchrun only rank 0 runs it.

With --gpus N > 1 (torchrun, one process per GPU) every rank runs its own
independent grid of the same workload (grids do not exchange data), so the
scaling is weak and `value` sums the cell updates of all ranks over the
slowest rank's time.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOADS = {
    # name: (n, leapfrog steps, pml layers, description)
    "c2": (128, 1000, 10, "fdtd3d-128^3-cpml10-sphere-eps4-pulse-16probes"),
    "c1": (64, 500, 8, "fdtd3d-64^3-cpml8-vacuum-pulse-8probes"),
    "c3": (512, 200, 12, "fdtd3d-512^3-cpml12-smoothnoise-eps1to12"),
    # config 3 at 256^3: the size the kernel profiles are captured at (fields
    # and psi ~1 GB, above L2, small enough for multi-pass ncu captures)
    "c3s": (256, 200, 12, "fdtd3d-256^3-cpml12-smoothnoise-eps1to12"),
    # differentiable inverse design: forward with sqrt(T) checkpoints and the
    # adjoint (time-reversed Yee) backward, dJ/d theta of 32^3 design cells
    "c4": (96, 2000, 10, "adjoint-96^3-cpml10-2000steps-design32-planeEx-z15-probe-z80"),
    # batched learned boundary: 64 grids, interior sides uniform in [48, 160]
    "c5": (64, 1000, 3, "batch64-sides48to160-eps1to6-dipoles-learnedband3-vs-cpml10"),
}
BAND_WEIGHTS = ROOT / "jaxphys_b200" / "em" / "band_weights.npz"



# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum, ncu) per leapfrog
# step of a workload, keyed by the launch shape they were captured at: a
# figure applies only when the run's autotuned launch is that shape.
NCU_TRAFFIC: dict = {
    # config 2 at registry entry 8 (64x4 tile, 3 stages), 16-plane chunks,
    # single-axis split, one step per pass: general + z-only shell launches
    ("c2", 8, 16, 1, -1, 0): 80.7e6,
    # config 3 at 256^3, blocked passes of registry entry 2, 32-plane chunks,
    # one-step entry 8: the eight launches of a pass / 2
    ("c3s", 8, 32, 1, 2, 32): 610.7e6,
}


def ncu_traffic(workload: str, launch: dict):
    key = (workload, launch["tma_config"], launch["x_chunk"], launch["axis_split"],
           launch["blocked_config"], launch["blocked_x_chunk"])
    return NCU_TRAFFIC.get(key)


def make_inputs(name: str, seed: int = 0):
    """Permittivity map, source and probes of a workload (seeded)."""
    n, steps, pml, _ = WORKLOADS[name]
    rng = np.random.default_rng(seed + 2)
    if name == "c2":
        c = np.array([n // 2] * 3) + rng.integers(-16, 17, size=3)
        ix, iy, iz = np.ogrid[:n, :n, :n]
        mask = (ix - c[0]) ** 2 + (iy - c[1]) ** 2 + (iz - c[2]) ** 2 <= 20 ** 2
        eps = np.where(mask, 4.0, 1.0)
        n_probes = 16
    elif name == "c1":
        eps = None
        n_probes = 8
    else:
        from scipy.ndimage import gaussian_filter

        u = gaussian_filter(rng.random((n, n, n), dtype=np.float32), sigma=6, mode="wrap")
        u = (u - u.min()) / (u.max() - u.min())
        eps = 1.0 + 11.0 * u
        n_probes = 16
    prng = np.random.default_rng(seed + 1)
    probes = [tuple(int(v) for v in prng.integers(n // 8, n - n // 8, size=3))
              for _ in range(n_probes)]
    return eps, probes


def psi_bytes_per_cell(n: int, pml: int) -> float:
    """CPML psi traffic per cell update: 12 psi arrays, each read and written
    (8 B) over its slab storage (2*(pml+1) planes of n^2 cells)."""
    P = pml + 1
    frac = min(2 * P, n) / n
    return 12 * frac * 8.0


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def run_ours(args, world, rank, local, pg, workload=None, steps=None, warmup=None,
             with_cpu=True, emit=True):
    """One independent grid of a single-grid workload per rank; returns the
    JSON line (printed by rank 0 when ``emit``)."""
    import torch

    from jaxphys_b200 import CPMLSpec, EMGrid3D, PointSource3D

    workload = workload or args.workload
    n_timed = args.steps if steps is None else steps
    n_warm = args.warmup if warmup is None else warmup
    torch.cuda.set_device(local)
    dev = torch.device(f"cuda:{local}")
    n, nsteps, pml, wname = WORKLOADS[workload]
    eps, probes = make_inputs(workload, seed=rank)
    g = EMGrid3D(size=(n, n, n), resolution=1.0, boundary="cpml", pml_layers=pml,
                 cpml=CPMLSpec(order=3.0, r0=1e-6), device=local)
    dt = g.default_dt()
    g.add_source(PointSource3D(frequency=0.05 / dt, position=(n // 2, n // 2, n // 2),
                               waveform="gauss_sine", width_steps=30.0))
    for p in probes:
        g.add_probe(p, "ez")
    if eps is not None:
        g.set_permittivity(eps)
    g.prepare(dt=dt)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()

    def one_step():
        g.reset()
        return g.run(nsteps)

    def barrier():
        torch.cuda.synchronize()
        if pg is not None:
            pg.barrier()

    for _ in range(n_warm):
        one_step()
    g.check()
    barrier()

    # ---- device-resident timing: K steps, L2 flushed between them
    sampler = ClockSampler(local)
    sampler.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(n_timed)]
    kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(n_timed)]
    barrier()
    for k in range(n_timed):
        flush.fill_(k & 0xFF)
        ev[k][0].record(stream)
        g.reset()
        kev[k][0].record(stream)
        g.run(nsteps)
        kev[k][1].record(stream)
        ev[k][1].record(stream)
    barrier()
    clocks = sampler.stop()
    g.check()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    kern_ms = [a.elapsed_time(b) for a, b in kev]
    total_ms = float(sum(step_ms))
    if pg is not None:
        t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        total_ms = float(t.item())

    # ---- end to end through the public API with host buffers
    eps_host = None
    if eps is not None:
        eps_host = torch.from_numpy(np.ascontiguousarray(eps, dtype=np.float32)).pin_memory()
    eps_dev = torch.empty((n, n, n), dtype=torch.float32, device=dev)
    probe_host = torch.empty((nsteps, len(probes)), dtype=torch.float32).pin_memory()

    def e2e_step():
        if eps_host is not None:
            eps_dev.copy_(eps_host, non_blocking=True)
            g.set_permittivity_device(eps_dev)
        g.reset()
        tr = g.run(nsteps)
        probe_host.copy_(tr, non_blocking=True)
        return tr

    e2e_step()
    barrier()
    e_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
            for _ in range(n_timed)]
    for k in range(n_timed):
        flush.fill_(k & 0xFF)
        e_ev[k][0].record(stream)
        e2e_step()
        e_ev[k][1].record(stream)
    barrier()
    e2e_ms = float(sum(a.elapsed_time(b) for a, b in e_ev))
    if pg is not None:
        t = torch.tensor([e2e_ms], dtype=torch.float64, device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_ms = float(t.item())
    h2d = 0 if eps_host is None else eps_host.numel() * 4
    d2h = probe_host.numel() * 4

    cells = n ** 3
    updates = cells * nsteps * n_timed * world
    value = updates / (total_ms * 1e-3) / 1e9
    e2e_value = updates / (e2e_ms * 1e-3) / 1e9

    # ---- roofline of the dominant kernel (the fused TMA step)
    info = g.info()
    # one leapfrog step = the step launch(es) of one time step (the probe
    # gather that ends each run is < 0.1 % of it)
    per_launch_ms = statistics.mean(kern_ms) / nsteps
    b_cell = 52.0 + psi_bytes_per_cell(n, pml) if eps is not None else 48.0 + psi_bytes_per_cell(n, pml)
    bytes_per_launch = cells * b_cell
    achieved = bytes_per_launch / (per_launch_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peaks()
    launch = {"tma_config": info["tma_config"], "x_chunk": info["x_chunk"],
              "axis_split": info["axis_split"], "blocked_config": info["blocked_config"],
              "blocked_x_chunk": info["blocked_x_chunk"]}
    traffic = ncu_traffic(workload, launch)
    blocked = info["blocked_config"] >= 0
    if blocked:
        # pairs of steps per blocked pass (+ one ordinary step for an odd count)
        launches = (nsteps // 2) * info["blocked_kernels_per_pass"] + \
            (nsteps % 2) * g.kernels_per_step() + 1
    else:
        launches = nsteps * g.kernels_per_step() + 1

    line = {
        "metric": "FDTD3D Gcell-updates/s",
        "value": round(value, 3),
        "unit": "Gcell/s",
        "n_gpus": world,
        "steps": n_timed,
        "warmup": n_warm,
        "ms_per_step": round(total_ms / n_timed, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded eps_r sphere, pulsed dipole, seeded probes)",
        "config": {"workload": wname, "cells": cells, "leapfrog_steps_per_step": nsteps,
                   "boundary": "cpml", "pml_layers": pml, "l2": "flushed (256 MiB write) between steps",
                   "path": "tma" if info["path"] == 2 else "generic",
                   "tile": [info["tile_z"], info["tile_y"], info["rows_per_thread"],
                            info["stages"], info["x_chunk"]],
                   "launch": launch,
                   "parallelism": f"independent grid per GPU x{world}"},
        "e2e": {"value": round(e2e_value, 3), "unit": "Gcell/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic,
                     "peak_source": peak_kind, "bytes_per_cell_update": round(b_cell, 2),
                     "kernel": ("k3d_tb2 two-level blocked pass (every launch of a pass), "
                                "per leapfrog step" if blocked else
                                "k3d_tma step (every launch of one leapfrog step)"),
                     "ms_per_leapfrog_step": round(per_launch_ms, 5)},
        "gpu_launches": launches * n_timed,
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and with_cpu and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(workload, budget_s=args.cpu_seconds)
    g._release()
    del flush
    if rank == 0 and emit:
        print(json.dumps(line), flush=True)
    return line


def pack_by_cells(cells: list, parts: int) -> list:
    """Indices of each part: largest item first onto the least-loaded part."""
    order = sorted(range(len(cells)), key=lambda i: -cells[i])
    load = [0] * parts
    out = [[] for _ in range(parts)]
    for i in order:
        r = min(range(parts), key=lambda k: load[k])
        out[r].append(i)
        load[r] += cells[i]
    return [sorted(o) for o in out]


def c5_cases(seed: int = 5, n_grids: int = 64):
    """The batched learned-boundary workload: seeded interior sides uniform in
    [48, 160] (half cubes, half boxes), smoothed eps_r in [1, 6], one dipole of
    random position and orientation per grid (Gaussian-modulated sinusoid,
    f0 = 0.05/dt, width 30 steps)."""
    from jaxphys_b200.em.learned import random_case

    rng = np.random.default_rng(seed)
    cases = []
    for _ in range(n_grids):
        if rng.random() < 0.5:
            s = int(rng.integers(48, 161))
            size = (s, s, s)
        else:
            size = tuple(int(v) for v in rng.integers(48, 161, 3))
        cases.append(random_case(rng, size, eps_range=(1.0, 6.0), n_sources=1, margin=4))
    return cases


def run_batch(args, world, rank, local, pg, steps=None, warmup=None, reflection=None,
              emit=True):
    """c5: the same 64-grid batch with the learned 3-cell band, with 10-cell
    CPML, with the CPML of equal measured error (4 cells) and with bare PEC
    walls.  value = interior cell updates per second of the learned run."""
    import torch

    n_timed = args.steps if steps is None else steps
    n_warm = args.warmup if warmup is None else warmup
    n_refl = args.reflection if reflection is None else reflection

    from jaxphys_b200.em.batch import FDTDBatch
    from jaxphys_b200.em.learned import BAND_LAYERS, LearnedBand, reflection_db, train_band

    torch.cuda.set_device(local)
    n_grids, nsteps, _, wname = WORKLOADS["c5"]
    n_grids = getattr(args, "batch_grids", None) or n_grids
    nsteps = getattr(args, "leapfrog_steps", None) or nsteps
    kinds = [k for k in getattr(args, "batch_kinds", "learned,cpml10,cpml4,pec").split(",") if k]
    if kinds[0] != "learned":
        raise SystemExit("--batch-kinds must start with learned")
    if n_grids != WORKLOADS["c5"][0]:
        wname = f"{wname}-first{n_grids}"
    if nsteps != WORKLOADS["c5"][1]:
        wname = f"{wname}-{nsteps}steps"
    # the 64 grids are bin-packed by cell count over the ranks (largest first
    # onto the least-loaded rank): a fixed total batch, so strong scaling
    all_cases = c5_cases(seed=5, n_grids=n_grids)
    cases = [all_cases[i] for i in pack_by_cells([int(np.prod(c.size)) for c in all_cases],
                                                 world)[rank]]
    interior = sum(int(np.prod(c.size)) for c in cases)
    interior_total = sum(int(np.prod(c.size)) for c in all_cases)
    model = LearnedBand.load(BAND_WEIGHTS) if BAND_WEIGHTS.exists() else train_band(seed=0)
    stream = torch.cuda.current_stream()

    def barrier():
        torch.cuda.synchronize()
        if pg is not None:
            pg.barrier()

    def build(kind):
        grids = []
        for c in cases:
            # every c5 grid is padded to nz % 4 == 0: the batch runs on the
            # persistent TMA kernel
            if kind in ("learned", "pec"):
                g = c.grid(BAND_LAYERS, "pec", 0, path="tma")
            else:
                k = int(kind[4:])
                g = c.grid(k, "cpml", k, path="tma")
            g.prepare()
            grids.append(g)
        b = FDTDBatch(grids)
        if kind == "learned":
            b.set_band(model)
        return grids, b

    results = {}
    launches = 0
    sampler = None
    for kind in kinds:
        grids, b = build(kind)
        cells = sum(int(np.prod(g.size)) for g in grids)
        cells_total = cells
        if pg is not None:
            t = torch.tensor([float(cells)], dtype=torch.float64, device=f"cuda:{local}")
            pg.all_reduce(t)
            cells_total = int(t.item())
        for _ in range(max(n_warm, 1)):
            b.reset()
            b.run(nsteps)
        barrier()
        if kind == "learned":
            sampler = ClockSampler(local)
            sampler.start()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(n_timed)]
        for k in range(n_timed):
            b.reset()
            ev[k][0].record(stream)
            b.run(nsteps)
            ev[k][1].record(stream)
        barrier()
        clocks = sampler.stop() if kind == "learned" else None
        ms = float(sum(a.elapsed_time(bb) for a, bb in ev))
        if pg is not None:
            t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{local}")
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            ms = float(t.item())
        for g in grids[:2]:
            g.check()
        results[kind] = {"ms_per_step": round(ms / n_timed, 3), "grid_cells": cells_total,
                         "interior_gcell_s": round(interior_total * nsteps * n_timed / ms / 1e6, 3),
                         "grid_gcell_s": round(cells_total * nsteps * n_timed / ms / 1e6, 3)}
        if kind == "learned":
            results[kind]["clocks"] = clocks
            launches = b.kernels_per_step() * nsteps * n_timed
            results[kind]["launch"] = b.launch()
        b.close()
        for g in grids:
            g._release()
    model.check()
    refl = {}
    if rank == 0 and n_refl > 0:
        small = sorted(range(len(cases)), key=lambda i: np.prod(cases[i].size))[:n_refl]
        for i in small:
            r = reflection_db(cases[i], nsteps, model=model, cpml_layers=(4, 10), every=10)
            refl[str(cases[i].size)] = {k: round(v, 2) for k, v in r.items()}
    lr = results["learned"]
    peak, peak_kind = measured_peaks()
    # algorithmic bytes of one leapfrog step of the learned batch: the Yee
    # update (6 components read + written, eps read: 52 B per cell) and the
    # band (outer cells: 24 B stencil centre read, 24 B correction written
    # and read back, 24 B field read-modify-write: 120 B per outer cell)
    outer = sum(int(np.prod(np.array(c.size) + 6)) - int(np.prod(np.array(c.size) + 4))
                for c in all_cases)
    step_bytes = lr["grid_cells"] * 52.0 + outer * 120.0
    # per GPU (the batch is split over the ranks)
    achieved = step_bytes / world / (lr["ms_per_step"] / nsteps * 1e-3) / 1e9
    line = {
        "metric": "learned-band batch interior Gcell-updates/s",
        "value": lr["interior_gcell_s"],
        "unit": "Gcell/s",
        "n_gpus": world,
        "steps": n_timed,
        "warmup": n_warm,
        "ms_per_step": lr["ms_per_step"],
        "higher_is_better": True,
        "scaling": "strong",
        "vs_baseline": None,
        "dtype": "f32 fields, bf16 MLP with f32 accumulation",
        "data": "synthetic (seeded sizes, eps_r maps, dipoles)",
        "config": {"workload": wname, "grids": n_grids, "interior_cells": interior_total,
                   "leapfrog_steps_per_step": nsteps, "band_layers": BAND_LAYERS,
                   "l2": "inputs larger than L2 (>= 360 MB of fields)",
                   "path": "tma (persistent batch launch)", "launch": lr.pop("launch", None),
                   "parallelism": f"the {n_grids} grids bin-packed by cell count over {world} GPU(s)"},
        "compare": {k: results[k] for k in ("cpml10", "cpml4", "pec") if k in results},
        "reflection_db": refl,
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": None, "peak_source": peak_kind,
                     "kernel": "whole learned-batch leapfrog step (Yee + band)"},
        "gpu_launches": launches,
        "clocks": lr.pop("clocks"),
    }
    for k, key in (("cpml10", "speedup_vs_cpml10"), ("cpml4", "speedup_vs_cpml4_equal_error")):
        if k in results:
            line[key] = round(results[k]["ms_per_step"] / lr["ms_per_step"], 3)
    if rank == 0 and emit:
        print(json.dumps(line), flush=True)
    return line


def run_adjoint(args, world, rank, local, pg, steps=None, warmup=None, emit=True):
    """c4: one gradient evaluation of config 4 = a forward run of 2000 steps
    keeping sqrt(T) checkpoints + the adjoint backward (recomputing each
    segment from its checkpoint, then the transposed steps); value = forward
    cell updates per second of the whole gradient evaluation."""
    import torch

    from jaxphys_b200 import CPMLSpec, EMGrid3D, PointSource3D

    n_timed = args.steps if steps is None else steps
    n_warm = args.warmup if warmup is None else warmup
    torch.cuda.set_device(local)
    dev = torch.device(f"cuda:{local}")
    n, nsteps, pml, wname = WORKLOADS["c4"]
    g = EMGrid3D(size=(n, n, n), resolution=1.0, boundary="cpml", pml_layers=pml,
                 cpml=CPMLSpec(), device=local)
    dt = g.default_dt()
    for i in range(n):  # plane-wave Ex source at z = 15
        for j in range(n):
            g.add_source(PointSource3D(frequency=0.05 / dt, position=(i, j, 15), polarization="x",
                                       waveform="gauss_sine", width_steps=30.0))
    g.add_probe((n // 2, n // 2, 80), "ez")
    g.prepare(dt=dt)
    rng = np.random.default_rng(4 + rank)
    theta = torch.tensor(rng.standard_normal((32, 32, 32)), dtype=torch.float32, device=dev)
    eps = torch.ones((n, n, n), dtype=torch.float32, device=dev)
    eps[32:64, 32:64, 32:64] = 1.0 + 11.0 * torch.sigmoid(theta)
    g.set_permittivity_device(eps)
    stream = torch.cuda.current_stream()

    def one():
        tr = g.adjoint_forward(nsteps)
        grad = g.adjoint_backward(2.0 * tr)  # J = sum of squared probe values
        return grad

    for _ in range(max(n_warm, 1)):
        one()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(n_timed)]
    for k in range(n_timed):
        ev[k][0].record(stream)
        one()
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    g.check()
    ms = float(sum(a.elapsed_time(b) for a, b in ev))
    if pg is not None:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = float(t.item())
    value = n ** 3 * nsteps * n_timed * world / (ms * 1e-3) / 1e9
    line = {
        "metric": "adjoint gradient evaluation, forward Gcell-updates/s",
        "value": round(value, 3), "unit": "Gcell/s", "n_gpus": world, "steps": n_timed,
        "warmup": n_warm, "ms_per_step": round(ms / n_timed, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (dJ/dcb accumulated in f64)",
        "data": "synthetic (seeded theta ~ N(0,1) on the central 32^3 cells)",
        "config": {"workload": wname, "cells": n ** 3, "leapfrog_steps": nsteps,
                   "checkpoints": "every ceil(sqrt(T)) steps",
                   "note": "a gradient = forward + segment recompute + transposed steps"},
        "gpu_launches": None, "clocks": clocks,
    }
    g._release()
    if rank == 0 and emit:
        print(json.dumps(line), flush=True)
    return line


def cpu_baseline(workload: str, budget_s: float = 10.0, steps: int | None = None):
    """The FP64 C restatement of the reference step on every host thread, on a
    bounded sample (a prefix of the workload's leapfrog steps)."""
    from oracle import ref_numpy as rn
    from oracle.cpu_oracle import Oracle3DC, num_threads

    n, nsteps, pml, wname = WORKLOADS[workload]
    eps, probes = make_inputs(workload)
    dt = rn.default_dt_3d(1.0)
    spec = rn.Spec3D(size=(n, n, n), dx=1.0, boundary="cpml", pml_layers=pml, eps_r=eps,
                     sources=[dict(position=(n // 2,) * 3, polarization="z", amplitude=1.0,
                                   kind="gauss_sine", frequency=0.05 / dt, width_steps=30.0,
                                   delay_steps=120.0)],
                     probes=[p + (2,) for p in probes])
    o = Oracle3DC(spec, dt=dt)
    o.run(2)
    if steps is None:
        t0 = time.perf_counter()
        o.run(4)
        per = (time.perf_counter() - t0) / 4
        steps = max(4, min(nsteps, int(budget_s / max(per, 1e-6))))
    t0 = time.perf_counter()
    o.run(steps)
    el = time.perf_counter() - t0
    v = n ** 3 * steps / el / 1e9
    return {"value": round(v, 4), "unit": "Gcell/s", "cores": num_threads(), "kind": "port",
            "sample": f"{wname}: {steps} leapfrog steps of the same grid, source and "
                      f"permittivity (FP64, oracle/cpu_fdtd.c, {num_threads()} threads)",
            "seconds": round(el, 4)}


def run_reference(args, world, rank):
    """The reference arm: the CPU restatement of the reference step (FP64 C,
    every host thread) on the same workload.  A bench step is the whole
    workload (all its leapfrog steps) when that takes at most
    ``JXF_REF_STEP_SECONDS`` (default 12 s) on this host, else the longest
    prefix that fits; ``value`` is the cell updates of all timed steps over
    their total time."""
    if rank != 0:
        return
    if args.workload in ("c4", "c5"):
        print(json.dumps({"impl": "reference", "unavailable": "the reference has neither an "
                          "FDTD gradient nor a learned boundary or batched grids; its CPU Yee "
                          "path is timed under the c1/c2/c3 workloads"}), flush=True)
        return
    n, nsteps, pml, wname = WORKLOADS[args.workload]
    budget = float(os.environ.get("JXF_REF_STEP_SECONDS", "12"))
    probe = cpu_baseline(args.workload, steps=4)
    per_step = probe["seconds"] / 4
    sample = max(4, min(nsteps, int(budget / max(per_step, 1e-9))))
    for _ in range(args.warmup):
        cpu_baseline(args.workload, steps=2)
    times, updates = [], 0
    res = None
    for _ in range(args.steps):
        res = cpu_baseline(args.workload, steps=sample)
        times.append(res["seconds"])
        updates += n ** 3 * sample
    value = round(updates / sum(times) / 1e9, 4)
    line = {
        "metric": "FDTD3D Gcell-updates/s",
        "value": value,
        "unit": "Gcell/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(1e3 * statistics.mean(times), 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded eps_r map, pulsed dipole, seeded probes)",
        "config": {"workload": wname, "cells": n ** 3, "leapfrog_steps_per_step": sample,
                   "boundary": "cpml", "pml_layers": pml,
                   "same_config": sample == nsteps},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "Gcell/s", "cores": res["cores"], "kind": "port",
                         "sample": res["sample"]},
        "e2e": {"value": value, "unit": "Gcell/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def secondary(args, world, rank, local, pg):
    """Config 3 (512^3, 12-cell CPML, eps_r in [1, 12]), config 5 (64
    batched grids, learned band against CPML) and config 4 (adjoint gradient
    of the 96^3 inverse-design problem) measured in the same run as the
    headline line, with their own short step counts (3, 2 and 2 timed
    steps)."""
    out = {}
    c3 = run_ours(args, world, rank, local, pg, workload="c3", steps=3, warmup=1,
                  with_cpu=False, emit=False)
    out["c3"] = {k: c3[k] for k in ("value", "unit", "ms_per_step", "steps", "warmup",
                                    "roofline", "gpu_launches", "clocks", "e2e")}
    out["c3"]["config"] = c3["config"]
    c5 = run_batch(args, world, rank, local, pg, steps=2, warmup=1, reflection=2, emit=False)
    out["c5"] = {k: c5[k] for k in ("metric", "value", "unit", "ms_per_step", "steps", "warmup",
                                    "compare", "speedup_vs_cpml10",
                                    "speedup_vs_cpml4_equal_error", "reflection_db",
                                    "roofline", "gpu_launches", "clocks", "dtype")}
    out["c5"]["config"] = c5["config"]
    c4 = run_adjoint(args, world, rank, local, pg, steps=2, warmup=1, emit=False)
    out["c4"] = {k: c4[k] for k in ("metric", "value", "unit", "ms_per_step", "steps", "warmup",
                                    "clocks", "config")}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", choices=tuple(WORKLOADS), default="c2")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--reflection", type=int, default=2,
                    help="c5: grids whose reflection is measured against a padded reference")
    ap.add_argument("--batch-grids", type=int, default=None,
                    help="c5: run only the first N grids of the seeded 64 (profiling)")
    ap.add_argument("--leapfrog-steps", type=int, default=None,
                    help="c5: leapfrog steps per timed run instead of 1000 (profiling)")
    ap.add_argument("--batch-kinds", default="learned,cpml10,cpml4,pec",
                    help="c5: boundary variants to time, learned first (profiling)")
    ap.add_argument("--no-secondary", action="store_true",
                    help="default workload: skip the config-3 and config-5 measurements")
    args = ap.parse_args()
    world, rank, local, pg = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        elif args.workload == "c5":
            run_batch(args, world, rank, local, pg)
        elif args.workload == "c4":
            run_adjoint(args, world, rank, local, pg)
        elif args.workload == "c2" and world == 1 and not args.no_secondary:
            line = run_ours(args, world, rank, local, pg, emit=False)
            line["secondary"] = secondary(args, world, rank, local, pg)
            print(json.dumps(line), flush=True)
        else:
            run_ours(args, world, rank, local, pg)
    finally:
        if pg is not None:
            pg.barrier()
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
