"""Batched grids (jxf_batch3d_*): uneven sizes, odd extents, sources and
probes; the batch (graph-captured and plain launches) equals each grid
stepped alone on the same kernels, bit for bit."""

import numpy as np
import pytest

from cases import rn
from gpu_helpers import smooth_eps, to_np

pytestmark = pytest.mark.gpu

SIZES = [(24, 20, 28), (17, 23, 19), (30, 16, 22), (12, 12, 12), (21, 27, 25)]
COMPS = ("ex", "ey", "ez", "hx", "hy", "hz")


def _grid(i, size, bnd):
    from jaxphys_b200 import EMGrid3D, PointSource3D

    dt = rn.default_dt_3d(1.0)
    g = EMGrid3D(size=size, resolution=1.0, boundary=bnd, pml_layers=4, path="generic")
    c = tuple(s // 2 for s in size)
    g.add_source(PointSource3D(frequency=0.05 / dt, position=c, polarization="xyz"[i % 3],
                               waveform="gauss_sine", width_steps=6.0 + i))
    g.add_probe((c[0], c[1], min(c[2] + 3, size[2] - 1)), "ez")
    g.add_probe((1, 2, 3), "hx")
    g.set_permittivity(smooth_eps(size, 1.0, 3.0 + i, seed=i))
    g.prepare(dt=dt)
    return g


@pytest.mark.parametrize("bnd", ["cpml", "absorbing"])
@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_equals_individual_runs(cuda, bnd, use_graph):
    from jaxphys_b200.em.batch import FDTDBatch

    grids = [_grid(i, s, bnd) for i, s in enumerate(SIZES)]
    b = FDTDBatch(grids)
    tr1 = b.run(25, use_graph=use_graph)
    tr2 = b.run(15, use_graph=use_graph)
    for i, s in enumerate(SIZES):
        ref = _grid(i, s, bnd)
        r = to_np(ref.run(40))
        got = np.vstack([to_np(tr1[i]), to_np(tr2[i])])
        assert np.array_equal(got, r), i
        for k in COMPS:
            assert np.array_equal(to_np(grids[i].field(k)), to_np(ref.field(k))), (i, k)
    # replay from rest reuses the captured graph and reproduces the run
    b.reset()
    tr3 = b.run(25, use_graph=use_graph)
    for i in range(len(SIZES)):
        assert np.array_equal(to_np(tr3[i]), to_np(tr1[i]))
    b.close()


# ---- TMA batches: one persistent launch per step over all grids' blocks

TMA_SIZES = [(24, 20, 28), (17, 23, 20), (30, 16, 24), (12, 12, 12), (21, 27, 36),
             (40, 33, 44)]


def _grid_path(i, size, bnd, path, eps=True):
    from jaxphys_b200 import EMGrid3D, PointSource3D

    dt = rn.default_dt_3d(1.0)
    g = EMGrid3D(size=size, resolution=1.0, boundary=bnd, pml_layers=4, path=path)
    c = tuple(s // 2 for s in size)
    g.add_source(PointSource3D(frequency=0.05 / dt, position=c, polarization="xyz"[i % 3],
                               waveform="gauss_sine", width_steps=6.0 + i))
    g.add_source(PointSource3D(frequency=0.04 / dt, position=(0, size[1] - 1, 3),
                               polarization="y", waveform="gauss_sine", width_steps=9.0))
    g.add_probe((c[0], c[1], min(c[2] + 3, size[2] - 1)), "ez")
    g.add_probe((1, 2, 3), "hx")
    if eps:
        g.set_permittivity(smooth_eps(size, 1.0, 3.0 + i, seed=i))
    g.prepare(dt=dt)
    return g


@pytest.mark.parametrize("bnd", ["cpml", "absorbing", "pec"])
@pytest.mark.parametrize("use_graph", [True, False])
@pytest.mark.parametrize("eps", [True, False])
def test_tma_batch_equals_generic_runs(cuda, bnd, use_graph, eps):
    """The persistent TMA batch (odd then even step counts, so both buffer
    parities start a run) equals every grid stepped alone on the generic
    kernels, bit for bit: fields and probe traces."""
    from jaxphys_b200.em.batch import FDTDBatch

    grids = [_grid_path(i, s, bnd, "tma", eps) for i, s in enumerate(TMA_SIZES)]
    b = FDTDBatch(grids)
    assert b.path == "tma"
    tr1 = b.run(25, use_graph=use_graph)
    tr2 = b.run(16, use_graph=use_graph)
    for i, s in enumerate(TMA_SIZES):
        ref = _grid_path(i, s, bnd, "generic", eps)
        r = to_np(ref.run(41))
        got = np.vstack([to_np(tr1[i]), to_np(tr2[i])])
        assert np.array_equal(got, r), i
        for k in COMPS:
            assert np.array_equal(to_np(grids[i].field(k)), to_np(ref.field(k))), (i, k)
    b.reset()
    tr3 = b.run(25, use_graph=use_graph)
    for i in range(len(TMA_SIZES)):
        assert np.array_equal(to_np(tr3[i]), to_np(tr1[i]))
    b.close()


@pytest.mark.parametrize("launch", ["0,4,0", "2,8,1", "7,16,1", "8,4,0", "11,8,1"])
def test_tma_batch_every_shape(cuda, launch, monkeypatch):
    """Every batch launch shape (tile, chunk, single-axis split) on a CPML
    batch against the generic kernels."""
    from jaxphys_b200.em.batch import FDTDBatch

    monkeypatch.setenv("JXF_BATCH_LAUNCH", launch)
    grids = [_grid_path(i, s, "cpml", "tma") for i, s in enumerate(TMA_SIZES)]
    b = FDTDBatch(grids)
    b.run(21, use_graph=False)
    for i, s in enumerate(TMA_SIZES):
        ref = _grid_path(i, s, "cpml", "generic")
        ref.run(21)
        for k in COMPS:
            assert np.array_equal(to_np(grids[i].field(k)), to_np(ref.field(k))), (i, k)
    b.close()


def test_tma_batch_learned_band_equals_generic(cuda):
    """A learned band on a TMA batch (applied to the buffer set each step
    wrote) equals the same band on the generic batch."""
    from jaxphys_b200.em.batch import FDTDBatch
    from jaxphys_b200.em.learned import default_band

    sizes = [(24, 20, 28), (30, 26, 32), (20, 22, 24)]
    out = {}
    for path in ("tma", "generic"):
        grids = [_grid_path(i, s, "pec", path) for i, s in enumerate(sizes)]
        b = FDTDBatch(grids)
        b.set_band(default_band())
        b.run(13, use_graph=True)
        out[path] = [{k: to_np(g.field(k)) for k in COMPS} for g in grids]
        b.close()
    for i in range(len(sizes)):
        for k in COMPS:
            np.testing.assert_allclose(out["tma"][i][k], out["generic"][i][k], rtol=0,
                                       atol=0, err_msg=f"{i} {k}")


def test_tma_batch_rejects_mixed_parity(cuda):
    from jaxphys_b200 import ConfigurationError
    from jaxphys_b200.em.batch import FDTDBatch

    grids = [_grid_path(i, s, "cpml", "tma") for i, s in enumerate(TMA_SIZES[:2])]
    grids[0].step(1)
    b = FDTDBatch(grids)
    with pytest.raises(ConfigurationError):
        b.run(2)
    b.reset()
    b.run(2)
    b.close()
