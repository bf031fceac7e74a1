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
