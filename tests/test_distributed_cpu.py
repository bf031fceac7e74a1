"""x-slab decomposition of one grid over ranks (jaxphys_b200/em/distributed.py)
on CPU: world_size 2 and 3 over gloo, with the NumPy stand-in stepper,
against the undecomposed FP64 oracle (same update; source values pass through
the FP32 waveform table, hence the 1e-6 tolerance)."""

import os
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

from cases import rn

SIZE = (13, 10, 12)
STEPS = 30


def _sources(dt):
    from jaxphys_b200 import PointSource3D

    return [PointSource3D(frequency=0.05 / dt, position=(6, 5, 6), waveform="gauss_sine",
                          width_steps=5.0),
            PointSource3D(frequency=0.03 / dt, position=(4, 2, 9), polarization="x",
                          amplitude=0.5),
            PointSource3D(frequency=0.04 / dt, position=(9, 7, 3), polarization="y")]


PROBES = [(6, 5, 9, "ez"), (2, 8, 2, "hy"), (11, 3, 7, "ex"), (4, 4, 4, "hz")]


def _worker(rank, world, port, boundary, out_path, overlap=True, whole=False):
    import torch.distributed as dist

    from dist_helpers import NumpySlabStepper, NumpyWholeStepSlabStepper
    from jaxphys_b200.em.distributed import DistributedGrid3D

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        g = DistributedGrid3D(SIZE, resolution=1.0, boundary=boundary, pml_layers=3,
                              stepper_factory=lambda **kw: (NumpyWholeStepSlabStepper(**kw) if whole
                                                            else NumpySlabStepper(**kw)),
                              overlap=overlap)
        assert g.overlap == overlap
        for s in _sources(g.dt):
            g.add_source(s)
        for p in PROBES:
            g.add_probe(p[:3], p[3])
        rng = np.random.default_rng(0)
        g.set_permittivity(1.0 + 2.0 * rng.random(SIZE))
        tr = g.run(STEPS // 2).numpy()
        tr2 = g.run(STEPS - STEPS // 2).numpy()
        fields = [g.gather_field(k).numpy() for k in ("ex", "ey", "ez", "hx", "hy", "hz")]
        if rank == 0:
            np.savez(out_path, probes=np.vstack([tr, tr2]), *fields)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("boundary", ["absorbing", "pec"])
@pytest.mark.parametrize("schedule", ["overlap", "plain", "whole"])
def test_slab_decomposition_matches_oracle(world, boundary, schedule):
    """The three schedules: half steps plain (exchange, then the whole
    half-step) and overlapped (the neighbour's plane first, the exchange
    during the rest), and the whole steps of TMA slabs (E ghost planes of
    both neighbours exchanged, then H including the low ghost plane's
    replica, then E on the owned planes)."""
    from dist_helpers import free_port

    overlap, whole = schedule != "plain", schedule == "whole"
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "r.npz")
        mp.start_processes(_worker, args=(world, free_port(), boundary, out, overlap, whole),
                           nprocs=world,
                           join=True, start_method="spawn")
        res = np.load(out)
        dt = rn.default_dt_3d(1.0)
        rng = np.random.default_rng(0)
        eps = 1.0 + 2.0 * rng.random(SIZE)
        srcs = [dict(position=s.position, polarization=s.polarization, amplitude=s.amplitude,
                     kind=s.waveform, frequency=s.frequency, width_steps=s.width_steps,
                     delay_steps=4 * s.width_steps) for s in _sources(dt)]
        comp = {"ex": 0, "ey": 1, "ez": 2, "hx": 3, "hy": 4, "hz": 5}
        spec = rn.Spec3D(size=SIZE, dx=1.0, boundary=boundary, pml_layers=3, eps_r=eps,
                         sources=srcs, probes=[p[:3] + (comp[p[3]],) for p in PROBES])
        o = rn.Oracle3D(spec, dt=dt)
        out_o = o.run(STEPS)
        for k in range(6):
            assert rn.rel_l2(res[f"arr_{k}"], o.f[k]) <= 1e-6, k
        assert rn.rel_l2(res["probes"], out_o["probes"]) <= 1e-6


def test_slab_ranges():
    from jaxphys_b200.em.distributed import slab_ranges

    for nx in (8, 13, 128):
        for w in (1, 2, 3, 8):
            if w > nx:
                continue
            r = slab_ranges(nx, w)
            assert r[0][0] == 0 and r[-1][1] == nx
            assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
            sizes = [b - a for a, b in r]
            assert max(sizes) - min(sizes) <= 1
