"""x-slab decomposition with the CUDA slab kernels: two (or three) processes
on one GPU exchange ghost planes through gloo (host memory; no kernel waits on
another process) and must reproduce the undecomposed generic-path run of the
same grid bit for bit (same kernels, same operations)."""

import os
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

from cases import rn
from gpu_helpers import smooth_eps

pytestmark = pytest.mark.gpu

SIZE = (25, 20, 24)
STEPS = 40
PROBES = [(12, 10, 18, "ez"), (3, 4, 5, "hy"), (20, 15, 7, "ex"), (12, 11, 12, "hz")]


def _sources(dt):
    from jaxphys_b200 import PointSource3D

    return [PointSource3D(frequency=0.05 / dt, position=(12, 10, 12), waveform="gauss_sine",
                          width_steps=6.0),
            PointSource3D(frequency=0.04 / dt, position=(5, 14, 6), polarization="x",
                          waveform="gauss_sine", width_steps=5.0, amplitude=0.6),
            PointSource3D(frequency=0.04 / dt, position=(13, 3, 20), polarization="y",
                          waveform="gauss_sine", width_steps=5.0)]


def _worker(rank, world, port, boundary, out_path, overlap=True, path="generic"):
    import torch
    import torch.distributed as dist

    from jaxphys_b200.em.distributed import DistributedGrid3D

    torch.cuda.set_device(0)
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        g = DistributedGrid3D(SIZE, resolution=1.0, boundary=boundary, pml_layers=4, device=0,
                              overlap=overlap, path=path)
        for s in _sources(g.dt):
            g.add_source(s)
        for p in PROBES:
            g.add_probe(p[:3], p[3])
        g.set_permittivity(smooth_eps(SIZE, 1.0, 4.0, seed=9))
        tr = g.run(STEPS).cpu().numpy()
        fields = [g.gather_field(k).cpu().numpy() for k in ("ex", "ey", "ez", "hx", "hy", "hz")]
        g.st.check()
        if rank == 0:
            np.savez(out_path, tr, *fields)
        g.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,boundary", [(2, "cpml"), (3, "absorbing"), (2, "pec")])
@pytest.mark.parametrize("overlap", [True, False])
def test_decomposed_run_equals_single_grid(cuda, world, boundary, overlap):
    """Plain and overlapped (boundary plane first, exchange during the other
    planes) schedules, bit for bit against the undecomposed grid."""
    from dist_helpers import free_port
    from jaxphys_b200 import EMGrid3D

    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "r.npz")
        mp.start_processes(_worker, args=(world, free_port(), boundary, out, overlap),
                           nprocs=world, join=True, start_method="spawn")
        res = np.load(out)
        g = EMGrid3D(SIZE, resolution=1.0, boundary=boundary, pml_layers=4, path="generic")
        dt = g.default_dt()
        for s in _sources(dt):
            g.add_source(s)
        for p in PROBES:
            g.add_probe(p[:3], p[3])
        g.set_permittivity(smooth_eps(SIZE, 1.0, 4.0, seed=9))
        g.prepare(dt=dt)
        tr = g.run(STEPS).cpu().numpy()
        assert np.array_equal(res["arr_0"], tr)
        for k, name in enumerate(("ex", "ey", "ez", "hx", "hy", "hz")):
            assert np.array_equal(res[f"arr_{k + 1}"], g.field(name).cpu().numpy()), name
        assert rn.rel_l2(tr, tr) == 0.0


@pytest.mark.parametrize("world,boundary", [(2, "cpml"), (3, "cpml"), (3, "absorbing"), (2, "pec")])
def test_tma_slabs_equal_single_tma_grid(cuda, world, boundary):
    """x-slabs on the one-step TMA kernel: each rank marches its owned planes
    and recomputes H on its low ghost plane (a replica of the neighbour's last
    plane); ghost E planes are exchanged before every step.  Bit for bit
    against the undecomposed grid on the TMA path."""
    from dist_helpers import free_port
    from jaxphys_b200 import EMGrid3D

    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "r.npz")
        mp.start_processes(_worker, args=(world, free_port(), boundary, out, True, "tma"),
                           nprocs=world, join=True, start_method="spawn")
        res = np.load(out)
        g = EMGrid3D(SIZE, resolution=1.0, boundary=boundary, pml_layers=4, path="tma")
        dt = g.default_dt()
        for s in _sources(dt):
            g.add_source(s)
        for p in PROBES:
            g.add_probe(p[:3], p[3])
        g.set_permittivity(smooth_eps(SIZE, 1.0, 4.0, seed=9))
        g.prepare(dt=dt)
        tr = g.run(STEPS).cpu().numpy()
        assert np.abs(tr).max() > 0
        assert np.array_equal(res["arr_0"], tr)
        for k, name in enumerate(("ex", "ey", "ez", "hx", "hy", "hz")):
            assert np.array_equal(res[f"arr_{k + 1}"], g.field(name).cpu().numpy()), name


def test_tma_slab_rejects_half_steps_and_multi_step_calls(cuda):
    import ctypes as C

    from jaxphys_b200 import _native as nat

    lib = nat.load()
    d = nat.Grid3DDesc(nx=24, ny=16, nz=16, dx=1.0, dt=0.0, boundary=nat.BND_CPML, pml_layers=4,
                       cpml_order=3.0, cpml_r0=1e-6, cpml_kappa_max=1.0, cpml_alpha_max=0.0,
                       path=nat.PATH_TMA, device=0)
    h = C.c_void_p()
    nat.check(lib.jxf_grid3d_create_slab(C.byref(d), 8, 16, C.byref(h)), "create_slab")
    try:
        assert lib.jxf_grid3d_half_step(h, 0, None, None) == nat.ERR_INVALID
        assert "whole steps" in nat.last_error()
        assert lib.jxf_grid3d_step(h, 2, None, None) == nat.ERR_INVALID
        assert "one step per call" in nat.last_error()
        assert lib.jxf_grid3d_set_blocked(h, 0, 8) == nat.ERR_INVALID
        assert lib.jxf_grid3d_step(h, 1, None, None) == nat.OK
    finally:
        lib.jxf_grid3d_destroy(h)
