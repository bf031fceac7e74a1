"""Moving charges as grid sources, on the CPU: the Esirkepov deposit's
discrete continuity, and Gauss's law eps0 div(eps_r E) = rho(t) - rho(0) kept
by the oracle's Yee update with the deposit as sources."""

import numpy as np
import pytest

from jaxphys_b200 import ConfigurationError
from jaxphys_b200.em.charges import (MovingCharge3D, charges_from_trajectory, deposit_step,
                                     node_density)
from oracle import ref_numpy as rn

DX = 1e-3


def _div(ex, ey, ez, eps=None):
    """Node divergence of (eps_r E) on the Yee grid (E_x at i + 1/2, ...)."""
    if eps is not None:
        ex, ey, ez = ex * eps, ey * eps, ez * eps
    d = np.zeros(ex.shape)
    d[1:, 1:, 1:] = ((ex[1:, 1:, 1:] - ex[:-1, 1:, 1:]) + (ey[1:, 1:, 1:] - ey[1:, :-1, 1:])
                     + (ez[1:, 1:, 1:] - ez[1:, 1:, :-1])) / DX
    return d


def _run_oracle(size, charge, steps, eps=None, dtype=np.float64):
    dt = rn.default_dt_3d(DX)
    srcs = charge.deposit_sources(size, DX, dt, 0.0, eps)
    spec = rn.Spec3D(size=size, dx=DX, boundary="pec", eps_r=eps,
                     sources=[dict(position=s.position, polarization=s.polarization,
                                   amplitude=1.0, kind="table", samples=s.samples.values)
                              for s in srcs])
    o = rn.Oracle3D(spec, dt=dt, dtype=dtype)
    for _ in range(steps):
        o.step()
    return o, srcs, dt


def test_deposit_is_charge_conserving():
    rng = np.random.default_rng(1)
    for _ in range(50):
        xi0 = rng.uniform(3, 6, 3)
        xi1 = xi0 + rng.uniform(-0.9, 0.9, 3)
        base, fx, fy, fz = deposit_step(xi0, xi1)
        # -div F per node equals the change of the node weights
        div = np.zeros((4, 4, 4))
        div += fx - np.concatenate([np.zeros((1, 4, 4)), fx[:-1]], axis=0)
        div += fy - np.concatenate([np.zeros((4, 1, 4)), fy[:, :-1]], axis=1)
        div += fz - np.concatenate([np.zeros((4, 4, 1)), fz[:, :, :-1]], axis=2)
        size = tuple(int(v) for v in base + 8)
        s0 = node_density(xi0, size)[base[0]:base[0] + 4, base[1]:base[1] + 4,
                                     base[2]:base[2] + 4]
        s1 = node_density(xi1, size)[base[0]:base[0] + 4, base[1]:base[1] + 4,
                                     base[2]:base[2] + 4]
        np.testing.assert_allclose(div, s1 - s0, atol=1e-14)
        # the flux leaves the window at zero
        assert np.allclose(fx[-1], 0) and np.allclose(fy[:, -1], 0) and np.allclose(fz[:, :, -1], 0)


def _gauss_error(o, charge, dt, steps, eps=None):
    size = o.shape
    xi = charge.grid_path(DX, dt, 0.0)
    rho = charge.charge * (node_density(xi[min(steps, len(xi) - 1)], size)
                           - node_density(xi[0], size)) / DX ** 3
    err = rn.EPS0 * _div(o.f[0], o.f[1], o.f[2], eps) - rho
    # relative to the density of the whole charge on one node
    return np.abs(err).max() / (abs(charge.charge) / DX ** 3)


def test_gauss_law_straight_path_vacuum():
    size = (20, 18, 22)
    dt = rn.default_dt_3d(DX)
    n = 80
    p0 = np.array([7.3, 8.6, 9.1]) * DX
    v = np.array([0.2, -0.15, 0.1]) * 3e8
    q = MovingCharge3D(charge=1e-12, times=[0.0, n * dt], positions=[p0, p0 + v * n * dt])
    o, srcs, dt = _run_oracle(size, q, n)
    assert len(srcs) > 50
    assert _gauss_error(o, q, dt, n) < 1e-12
    assert max(np.abs(a).max() for a in o.f[:3]) > 1.0   # the fields are not trivial


def test_gauss_law_circular_path_in_dielectric():
    size = (22, 22, 20)
    dt = rn.default_dt_3d(DX)
    n = 120
    t = np.linspace(0.0, n * dt, 61)
    w = 2 * np.pi / (n * dt)
    c = np.array([11.0, 11.0, 9.5]) * DX
    r = 4.0 * DX
    pos = np.stack([c[0] + r * np.cos(w * t), c[1] + r * np.sin(w * t),
                    c[2] + 0.5 * DX * np.sin(2 * w * t)], axis=1)
    q = MovingCharge3D(charge=-2e-12, times=t, positions=pos)
    rng = np.random.default_rng(3)
    eps = 1.0 + 3.0 * rng.random(size)
    for steps in (n // 2 + 7, n + 10):   # half way round, and back at the start
        o, _, dt = _run_oracle(size, q, steps, eps=eps)
        assert _gauss_error(o, q, dt, steps, eps=eps) < 1e-12, steps


def test_errors_and_trajectory_helper():
    dt = rn.default_dt_3d(DX)
    with pytest.raises(ConfigurationError, match="out of grid"):
        MovingCharge3D(1e-12, [0, 10 * dt], [[0.5 * DX, 5 * DX, 5 * DX]] * 2).deposit_sources(
            (12, 12, 12), DX, dt)
    with pytest.raises(ConfigurationError, match="a cell or more"):
        MovingCharge3D(1e-12, [0, dt], [[4 * DX] * 3, [5.5 * DX] * 3]).deposit_sources(
            (12, 12, 12), DX, dt)
    with pytest.raises(ConfigurationError, match="increasing"):
        MovingCharge3D(1e-12, [0, 0], [[4 * DX] * 3] * 2).grid_path(DX, dt, 0.0)
    traj = np.zeros((5, 2, 3)) + 5 * DX
    traj[:, 1, 0] += np.linspace(0, 2 * DX, 5)
    qs = charges_from_trajectory(np.linspace(0, 40 * dt, 5), traj, [1e-12, -1e-12])
    assert len(qs) == 2 and qs[1].charge == -1e-12
    np.testing.assert_array_equal(qs[1].positions, traj[:, 1, :])
    with pytest.raises(ConfigurationError):
        charges_from_trajectory(np.zeros(5), traj, [1e-12])


def test_grid_accepts_moving_charge():
    from jaxphys_b200 import EMGrid3D

    g = EMGrid3D((16, 16, 16), resolution=DX, boundary="pec")
    dt = g.default_dt()
    q = MovingCharge3D(1e-12, [0, 30 * dt], [[6.3 * DX, 6.4 * DX, 6.2 * DX],
                                             [7.1 * DX, 6.9 * DX, 6.6 * DX]])
    g.add_source(q)
    assert len(g._sources) > 10
    assert all(s.waveform == "table" for s in g._sources)
