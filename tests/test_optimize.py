"""optimize(): the reference's gradient-descent / Adam loop
(src/neurosim/optimize.py:49-207) over torch autograd; inverse design through
the CUDA adjoint on the GPU."""

import numpy as np
import pytest
import torch

from jaxphys_b200.optimize import optimize


def _ref_loop(grad, x0, lr, iters, tol, method):
    """The reference's update rules, restated in NumPy (optimize.py:105-207)."""
    x = np.array(x0, dtype=np.float64)
    traj = [x.copy()]
    if method == "adam":
        m = np.zeros_like(x)
        v = np.zeros_like(x)
        for i in range(1, iters + 1):
            g = grad(x)
            if np.sqrt(np.sum(g ** 2)) < tol:
                return x, i, True, traj
            m = 0.9 * m + 0.1 * g
            v = 0.999 * v + 0.001 * g ** 2
            x = x - lr * (m / (1 - 0.9 ** i)) / (np.sqrt(v / (1 - 0.999 ** i)) + 1e-8)
            traj.append(x.copy())
        return x, iters, False, traj
    for i in range(iters):
        g = grad(x)
        if np.sqrt(np.sum(g ** 2)) < tol:
            return x, i, True, traj
        x = x - lr * g
        traj.append(x.copy())
    return x, iters, False, traj


A = np.array([[3.0, 0.5, 0.0], [0.5, 2.0, 0.3], [0.0, 0.3, 1.0]])
B = np.array([1.0, -2.0, 0.5])


def _obj(x):
    At = torch.as_tensor(A, dtype=x.dtype)
    Bt = torch.as_tensor(B, dtype=x.dtype)
    return 0.5 * x @ At @ x - Bt @ x


@pytest.mark.parametrize("method,lr,iters", [("gradient_descent", 0.1, 200), ("adam", 0.05, 150)])
def test_matches_reference_update_rules(method, lr, iters):
    x0 = np.array([0.3, 0.1, -0.2])
    res = optimize(_obj, torch.tensor(x0), learning_rate=lr, max_iterations=iters,
                   tolerance=1e-10, method=method, track_trajectory=True)
    xr, nr, cr, traj = _ref_loop(lambda x: A @ x - B, x0, lr, iters, 1e-10, method)
    assert res.n_iterations == nr and res.converged == cr
    np.testing.assert_allclose(res.x.numpy(), xr, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(res.trajectory.numpy(), np.stack(traj), rtol=1e-12, atol=1e-14)
    assert abs(res.fun - float(_obj(torch.tensor(xr)))) < 1e-12


def test_converges_and_reports():
    res = optimize(_obj, torch.zeros(3, dtype=torch.float64), learning_rate=0.2,
                   max_iterations=5000, tolerance=1e-9)
    assert res.converged and res.n_iterations < 5000
    np.testing.assert_allclose(res.x.numpy(), np.linalg.solve(A, B), atol=1e-8)
    with pytest.raises(ValueError):
        optimize(_obj, torch.zeros(3), method="lbfgs")


@pytest.mark.gpu
def test_inverse_design_through_adjoint(cuda):
    from jaxphys_b200 import EMGrid3D, PointSource3D
    from jaxphys_b200.em.adjoint import probe_traces

    n = (24, 24, 24)
    g = EMGrid3D(n, resolution=1.0, boundary="cpml", pml_layers=6, path="generic")
    dt = g.default_dt()
    g.add_source(PointSource3D(frequency=0.05 / dt, position=(12, 12, 7), polarization="x",
                               waveform="gauss_sine", width_steps=15.0))
    g.add_probe((12, 12, 17), "ez")
    g.add_probe((12, 13, 17), "ex")
    g.prepare(dt)
    region = (slice(9, 15), slice(9, 15), slice(10, 14))

    def objective(theta):
        eps = torch.ones(n, device="cuda")
        eps[region] = 1.0 + 11.0 * torch.sigmoid(theta)
        return -(probe_traces(g, eps, 160) ** 2).sum()

    theta0 = torch.zeros((6, 6, 4), device="cuda")
    res = optimize(objective, theta0, learning_rate=0.5, max_iterations=4, method="adam",
                   track_trajectory=True)
    f0 = float(objective(theta0).detach())
    assert res.fun < f0, (res.fun, f0)
    assert res.trajectory.shape == (5, 6, 6, 4)
    assert torch.isfinite(res.x).all()


# The reference's own optimizer tests (tests/test_optimize.py:14-80 and
# tests/test_edge_cases.py:1398-1440), on torch tensors.


def test_reference_quadratic_minimum():
    res = optimize(lambda x: (x - 3.0) ** 2, 0.0, learning_rate=0.1, max_iterations=1000)
    assert res.converged
    assert float(res.x) == pytest.approx(3.0, abs=1e-4)
    assert res.fun < 1e-6


def test_reference_adam():
    res = optimize(lambda x: (x - 5.0) ** 2 + 1.0, 0.0, learning_rate=0.1, max_iterations=1000,
                   method="adam")
    assert float(res.x) == pytest.approx(5.0, abs=0.1)


def test_reference_trajectory_and_multivariate():
    res = optimize(lambda x: x ** 2, 10.0, learning_rate=0.1, max_iterations=100,
                   track_trajectory=True)
    assert res.trajectory is not None and res.trajectory.shape[0] > 1
    target = torch.tensor([1.0, 2.0], dtype=torch.float64)
    res = optimize(lambda x: torch.sum((x - target) ** 2), torch.zeros(2, dtype=torch.float64),
                   learning_rate=0.1, max_iterations=1000)
    assert torch.allclose(res.x, target, atol=0.1)


def test_reference_edge_cases():
    res = optimize(lambda x: x ** 2, 0.0, learning_rate=0.1, tolerance=1e-8)
    assert res.converged and res.n_iterations == 0
    res = optimize(lambda x: (x - 100.0) ** 2, 0.0, learning_rate=0.001, max_iterations=5)
    assert not res.converged and res.n_iterations == 5


def test_reference_sensitivity():
    from jaxphys_b200.optimize import sensitivity

    s = sensitivity(lambda p: p ** 2, [3.0])
    assert s.shape == (1, 1) and float(s[0, 0]) == pytest.approx(6.0, abs=1e-6)
    j = sensitivity(lambda p: torch.stack([p[0] * p[1], p[1] ** 3]), [2.0, 3.0])
    np.testing.assert_allclose(j.numpy(), [[3.0, 2.0], [0.0, 27.0]])
