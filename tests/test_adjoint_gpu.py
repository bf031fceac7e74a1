"""Adjoint (permittivity gradient) of the CUDA path.

* small grids: the hand-written adjoint (FP32, sqrt(T) checkpointing with
  uneven segments) against FP64 reverse-mode autodiff through the torch
  restatement of the step (oracle/torch_ref.py, the stand-in for jax.grad),
  relative L2 of the gradient <= 1e-3;
* config 4: 96^3, 2000 steps, 10-cell CPML, 32^3 design region with
  eps_r = 1 + 11 sigmoid(theta), theta ~ N(0,1) seeded, Ex plane source at
  z=15, J = sum_t Ez(probe at z=80)^2; dJ/dtheta against central finite
  differences (h=1e-3) of the FP64 C oracle on 32 seeded design cells,
  relative L2 <= 1e-3.
"""

import numpy as np
import pytest

from cases import rn
from gpu_helpers import rel_l2, smooth_eps, to_np

pytestmark = pytest.mark.gpu


def _grid(size, bnd, sources, probes, pml):
    from jaxphys_b200 import EMGrid3D, PointSource3D

    g = EMGrid3D(size=size, resolution=1.0, boundary=bnd, pml_layers=pml)
    for s in sources:
        g.add_source(PointSource3D(**s))
    for p in probes:
        g.add_probe(p[:3], ("ex", "ey", "ez", "hx", "hy", "hz")[p[3]])
    return g


@pytest.mark.parametrize("bnd", ["absorbing", "pec", "cpml"])
def test_adjoint_matches_fp64_autodiff(cuda, bnd):
    import torch

    from jaxphys_b200.em.adjoint import probe_traces
    from oracle import torch_ref

    size = (20, 18, 24)
    dt = rn.default_dt_3d(1.0)
    eps = smooth_eps(size, 1.0, 5.0, seed=11)
    sources = [dict(frequency=0.05 / dt, position=(10, 9, 12), polarization="z",
                    waveform="gauss_sine", width_steps=8.0),
               dict(frequency=0.04 / dt, position=(4, 13, 6), polarization="x",
                    waveform="gauss_sine", width_steps=6.0, amplitude=0.7)]
    probes = [(10, 9, 18, 2), (15, 4, 20, 4), (5, 14, 4, 0)]
    n = 120
    rng = np.random.default_rng(3)
    w = rng.random((n, len(probes)))
    g = _grid(size, bnd, sources, probes, pml=4)
    g.prepare(dt=dt)
    e = torch.tensor(eps, dtype=torch.float32, device=cuda, requires_grad=True)
    tr = probe_traces(g, e, n, checkpoint_every=7)
    J = (torch.as_tensor(w, dtype=torch.float32, device=cuda) * tr ** 2).sum()
    J.backward()
    grad = to_np(e.grad)

    src64 = [dict(position=s["position"], polarization=s["polarization"],
                  amplitude=s.get("amplitude", 1.0), kind="gauss_sine", frequency=s["frequency"],
                  width_steps=s["width_steps"], delay_steps=4 * s["width_steps"])
             for s in sources]
    spec = rn.Spec3D(size=size, dx=1.0, boundary=bnd, pml_layers=4, eps_r=eps, sources=src64,
                     probes=probes)
    J64, grad64, tr64 = torch_ref.grad_eps(spec, eps, n, dt, w)
    assert rel_l2(to_np(tr), tr64) <= 1e-5
    assert abs(J.item() - J64) <= 1e-5 * abs(J64)
    e_rel = rel_l2(grad, grad64)
    assert e_rel <= 1e-3, e_rel
    # the forward of the adjoint run is the regular forward
    g2 = _grid(size, bnd, sources, probes, pml=4)
    g2.prepare(dt=dt)
    g2.set_permittivity_device(e.detach())
    assert np.array_equal(to_np(g2.run(n)), to_np(tr))


def test_config4_adjoint_vs_finite_differences(cuda):
    import torch

    from jaxphys_b200.em.adjoint import probe_traces
    from oracle.cpu_oracle import Oracle3DC

    n_side, steps, pml = 96, 2000, 10
    size = (n_side,) * 3
    dt = rn.default_dt_3d(1.0)
    lo, hi = 32, 64  # central 32^3 design region
    rng = np.random.default_rng(4)
    theta = rng.standard_normal((32, 32, 32))
    probe = (48, 48, 80, 2)
    # plane-wave Ex source: one Gaussian-pulse point source per (x, y) at z=15
    srcs = [dict(frequency=0.05 / dt, position=(i, j, 15), polarization="x",
                 waveform="gauss_sine", width_steps=30.0)
            for i in range(n_side) for j in range(n_side)]
    g = _grid(size, "cpml", srcs, [probe], pml)
    g.prepare(dt=dt)
    th = torch.tensor(theta, dtype=torch.float32, device=cuda, requires_grad=True)
    eps = torch.ones(size, dtype=torch.float32, device=cuda)
    eps = eps.index_put((torch.arange(lo, hi, device=cuda)[:, None, None],
                         torch.arange(lo, hi, device=cuda)[None, :, None],
                         torch.arange(lo, hi, device=cuda)[None, None, :]),
                        1.0 + 11.0 * torch.sigmoid(th))
    tr = probe_traces(g, eps, steps)
    J = (tr.double() ** 2).sum()
    J.backward()
    grad = to_np(th.grad).astype(np.float64)

    cells = [tuple(int(v) for v in c) for c in rng.integers(0, 32, size=(32, 3))]
    src64 = [dict(position=s["position"], polarization="x", amplitude=1.0, kind="gauss_sine",
                  frequency=s["frequency"], width_steps=30.0, delay_steps=120.0) for s in srcs]

    def J_of(th_np):
        e = np.ones(size)
        e[lo:hi, lo:hi, lo:hi] = 1.0 + 11.0 / (1.0 + np.exp(-th_np))
        spec = rn.Spec3D(size=size, dx=1.0, boundary="cpml", pml_layers=pml, eps_r=e,
                         sources=src64, probes=[probe])
        return float(np.sum(Oracle3DC(spec, dt=dt).run(steps)["probes"] ** 2))

    h = 1e-3
    fd = []
    for c in cells:
        tp = theta.copy()
        tp[c] += h
        tm = theta.copy()
        tm[c] -= h
        fd.append((J_of(tp) - J_of(tm)) / (2 * h))
    fd = np.array(fd)
    adj = np.array([grad[c] for c in cells])
    err = rel_l2(adj, fd)
    print("config4 adjoint vs FD: rel L2", err, "max rel",
          float(np.max(np.abs(adj - fd) / np.maximum(np.abs(fd), 1e-30))))
    assert err <= 1e-3
