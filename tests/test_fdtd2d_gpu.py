"""2D CUDA path against the reference's golden vectors and its own tests
(tests/test_em.py:18-79)."""

import numpy as np
import pytest

from cases import golden, load_cases
from gpu_helpers import grid2d_from_case, rel_l2, to_np

pytestmark = pytest.mark.gpu

CASES = load_cases()["2d"]


@pytest.mark.parametrize("case", CASES, ids=lambda c: c["name"])
def test_golden_parity(cuda, case):
    g = grid2d_from_case(case)
    h = g.simulate(t_span=tuple(case["t_span"]), save_every=case["save_every"])
    ref = golden("2d", case["name"])
    assert h.t.shape[0] == int(ref["n_saved"])
    np.testing.assert_array_equal(to_np(h.t), ref["t"])
    fr = ref["frames"]
    for k in ("ez", "hx", "hy"):
        r = np.asarray(ref[k], np.float64)
        got = to_np(getattr(h, k))[fr]
        if np.sqrt(np.sum(r * r)) < 1e-12:
            assert np.abs(got).max() < 1e-9
        else:
            assert rel_l2(got, r) <= 1e-5, k


def test_basic_simulation(cuda):
    from jaxphys_b200 import EMGrid, PlaneWave

    grid = EMGrid(size=(50, 50), resolution=0.01)
    grid.add_source(PlaneWave(frequency=3e9, y=10))
    f = grid.simulate(t_span=(0, 1e-9), save_every=10)
    assert f.ez.shape[1:] == (50, 50)
    assert f.t.shape[0] > 0


def test_with_conductor_zeroes_wall(cuda):
    from jaxphys_b200 import EMGrid, PlaneWave, Wall

    grid = EMGrid(size=(50, 50), resolution=0.01)
    grid.add_source(PlaneWave(frequency=3e9, y=10))
    grid.add_conductor(Wall(y=25, gap_start=20, gap_end=30))
    f = grid.simulate(t_span=(0, 5e-10), save_every=5)
    ez = to_np(f.ez[-1])
    assert np.all(ez[:20, 25] == 0) and np.all(ez[30:, 25] == 0)


def test_multiple_sources_are_applied(cuda):
    from jaxphys_b200 import EMGrid, PlaneWave

    grid = EMGrid(size=(50, 50), resolution=0.01)
    grid.add_source(PlaneWave(frequency=3e9, y=10, amplitude=1.0))
    grid.add_source(PlaneWave(frequency=5e9, y=35, amplitude=0.5))
    f = grid.simulate(t_span=(0, 2e-10), save_every=1)
    assert float(f.ez[-1, :, 10].abs().max()) > 0
    assert float(f.ez[-1, :, 35].abs().max()) > 0


def test_boundary_modes_affect_solution(cuda):
    import torch

    from jaxphys_b200 import EMGrid, PlaneWave

    per = EMGrid(size=(40, 40), resolution=0.01, boundary="periodic", pml_layers=0)
    ref = EMGrid(size=(40, 40), resolution=0.01, boundary="reflecting", pml_layers=0)
    s = PlaneWave(frequency=3e9, y=2, amplitude=1.0)
    per.add_source(s)
    ref.add_source(s)
    a = per.simulate(t_span=(0, 2e-10), save_every=1)
    b = ref.simulate(t_span=(0, 2e-10), save_every=1)
    assert not torch.allclose(a.ez[-1], b.ez[-1])
