"""Moving-charge current deposit on the CUDA path: fields against the FP64
oracle (relative L2 of E and of H <= 1e-5), TMA kernel bit-identical to the
generic kernel, and Gauss's law kept by the FP32 step (<= 1e-4 of the
density of the whole charge on one node)."""

import numpy as np
import pytest

from gpu_helpers import family_errors, grid_fields
from test_charges import DX, _gauss_error, _run_oracle

pytestmark = pytest.mark.gpu

SIZE = (20, 18, 24)
N = 80


def _charge():
    from jaxphys_b200.em.charges import MovingCharge3D
    from oracle import ref_numpy as rn

    dt = rn.default_dt_3d(DX)
    p0 = np.array([7.3, 8.6, 9.1]) * DX
    v = np.array([0.2, -0.15, 0.1]) * 3e8
    return MovingCharge3D(charge=1e-12, times=[0.0, N * dt], positions=[p0, p0 + v * N * dt])


def _grid(path):
    from jaxphys_b200 import EMGrid3D

    g = EMGrid3D(SIZE, resolution=DX, boundary="pec", path=path)
    g.add_source(_charge())
    g.prepare()
    g.step(N)
    return g


def test_moving_charge_matches_oracle_and_gauss_law(cuda):
    q = _charge()
    o, _, dt = _run_oracle(SIZE, q, N)
    out = []
    for path in ("tma", "generic"):
        got = grid_fields(_grid(path))
        eE, eH = family_errors(got, o.f)
        assert eE <= 1e-5 and eH <= 1e-5, (path, eE, eH)
        out.append(got)
    for a, b in zip(*out):
        assert np.array_equal(a, b)

    class _F:  # the GPU fields in the oracle's shape for the Gauss check
        shape = SIZE
        f = [x.astype(np.float64) for x in out[0]]

    assert _gauss_error(_F, q, dt, N) < 1e-4
