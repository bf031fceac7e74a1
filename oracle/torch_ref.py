"""Autodiff oracle: the 3D step restated in torch (FP64, CPU) -- TEST
INFRASTRUCTURE ONLY.

Stands in for ``jax.grad`` through the reference's ``EMGrid3D`` step (JAX is
not installable here): the same update as ``oracle/ref_numpy.py`` (which is
pinned bit for bit to ``src/neurosim/em/fdtd3d.py:280-379`` by tests/golden),
written with out-of-place torch ops so reverse-mode autograd through every
step gives the exact gradient of a probe objective with respect to the
per-cell permittivity.  Small grids only (it keeps the whole tape).
"""

from __future__ import annotations

import numpy as np
import torch

from . import ref_numpy as rn


def run(spec: rn.Spec3D, eps_r: torch.Tensor, n_steps: int, dt: float):
    """Probe traces (n_steps, P) as a differentiable function of eps_r."""
    nx, ny, nz = spec.size
    dev, dt_ = eps_r.device, torch.float64
    a = dt / (float(rn.MU0) * spec.dx)
    b = dt / (float(rn.EPS0) * spec.dx)
    cb = b / eps_r
    z = lambda: torch.zeros((nx, ny, nz), dtype=dt_, device=dev)  # noqa: E731
    ex, ey, ez, hx, hy, hz = (z() for _ in range(6))
    bnd = spec.boundary
    damp = None
    if bnd == "absorbing":
        damp = torch.from_numpy(rn.damping_3d(nx, ny, nz, spec.pml_layers, spec.dx, dt)).to(dev)
    if bnd == "cpml":
        tabs = [rn.cpml_tables_1d(n, spec.pml_layers, spec.dx, dt, spec.cpml) for n in spec.size]

        def t(ax, key, sl):
            v = torch.from_numpy(tabs[ax][key]).to(dev)
            shp = [1, 1, 1]
            shp[ax] = -1
            return v.reshape(shp)[sl]

        P = {k: z() for k in ("hxy", "hxz", "hyz", "hyx", "hzx", "hzy",
                               "exy", "exz", "eyz", "eyx", "ezx", "ezy")}
    srcs = [(tuple(s["position"]), rn.COMP[s.get("polarization", "z")],
             torch.from_numpy(rn.waveform_values(s, n_steps, dt, 0.0)))
            for s in spec.sources]
    traces = []
    S = slice
    for n in range(n_steps):
        hx, hy, hz = hx.clone(), hy.clone(), hz.clone()
        if bnd == "cpml":
            s_ = (S(None), S(0, -1), S(0, -1))
            dy = ez[:, 1:, :-1] - ez[:, :-1, :-1]
            dz = ey[:, :-1, 1:] - ey[:, :-1, :-1]
            P["hxy"] = P["hxy"].clone(); P["hxz"] = P["hxz"].clone()
            P["hxy"][s_] = t(1, "bh", (S(None), S(0, -1))) * P["hxy"][s_] + t(1, "ch", (S(None), S(0, -1))) * dy
            P["hxz"][s_] = t(2, "bh", (S(None), S(None), S(0, -1))) * P["hxz"][s_] + t(2, "ch", (S(None), S(None), S(0, -1))) * dz
            hx[s_] = hx[s_] - a * ((t(1, "ikh", (S(None), S(0, -1))) * dy - t(2, "ikh", (S(None), S(None), S(0, -1))) * dz) + (P["hxy"][s_] - P["hxz"][s_]))
            s_ = (S(0, -1), S(None), S(0, -1))
            dz = ex[:-1, :, 1:] - ex[:-1, :, :-1]
            dx = ez[1:, :, :-1] - ez[:-1, :, :-1]
            P["hyz"] = P["hyz"].clone(); P["hyx"] = P["hyx"].clone()
            P["hyz"][s_] = t(2, "bh", (S(None), S(None), S(0, -1))) * P["hyz"][s_] + t(2, "ch", (S(None), S(None), S(0, -1))) * dz
            P["hyx"][s_] = t(0, "bh", (S(0, -1),)) * P["hyx"][s_] + t(0, "ch", (S(0, -1),)) * dx
            hy[s_] = hy[s_] - a * ((t(2, "ikh", (S(None), S(None), S(0, -1))) * dz - t(0, "ikh", (S(0, -1),)) * dx) + (P["hyz"][s_] - P["hyx"][s_]))
            s_ = (S(0, -1), S(0, -1), S(None))
            dx = ey[1:, :-1, :] - ey[:-1, :-1, :]
            dy = ex[:-1, 1:, :] - ex[:-1, :-1, :]
            P["hzx"] = P["hzx"].clone(); P["hzy"] = P["hzy"].clone()
            P["hzx"][s_] = t(0, "bh", (S(0, -1),)) * P["hzx"][s_] + t(0, "ch", (S(0, -1),)) * dx
            P["hzy"][s_] = t(1, "bh", (S(None), S(0, -1))) * P["hzy"][s_] + t(1, "ch", (S(None), S(0, -1))) * dy
            hz[s_] = hz[s_] - a * ((t(0, "ikh", (S(0, -1),)) * dx - t(1, "ikh", (S(None), S(0, -1))) * dy) + (P["hzx"][s_] - P["hzy"][s_]))
            ex, ey, ez = ex.clone(), ey.clone(), ez.clone()
            s_ = (S(None), S(1, None), S(1, None))
            dy = hz[:, 1:, 1:] - hz[:, :-1, 1:]
            dz = hy[:, 1:, 1:] - hy[:, 1:, :-1]
            P["exy"] = P["exy"].clone(); P["exz"] = P["exz"].clone()
            P["exy"][s_] = t(1, "be", (S(None), S(1, None))) * P["exy"][s_] + t(1, "ce", (S(None), S(1, None))) * dy
            P["exz"][s_] = t(2, "be", (S(None), S(None), S(1, None))) * P["exz"][s_] + t(2, "ce", (S(None), S(None), S(1, None))) * dz
            ex[s_] = ex[s_] + cb[s_] * ((t(1, "ike", (S(None), S(1, None))) * dy - t(2, "ike", (S(None), S(None), S(1, None))) * dz) + (P["exy"][s_] - P["exz"][s_]))
            s_ = (S(1, None), S(None), S(1, None))
            dz = hx[1:, :, 1:] - hx[1:, :, :-1]
            dx = hz[1:, :, 1:] - hz[:-1, :, 1:]
            P["eyz"] = P["eyz"].clone(); P["eyx"] = P["eyx"].clone()
            P["eyz"][s_] = t(2, "be", (S(None), S(None), S(1, None))) * P["eyz"][s_] + t(2, "ce", (S(None), S(None), S(1, None))) * dz
            P["eyx"][s_] = t(0, "be", (S(1, None),)) * P["eyx"][s_] + t(0, "ce", (S(1, None),)) * dx
            ey[s_] = ey[s_] + cb[s_] * ((t(2, "ike", (S(None), S(None), S(1, None))) * dz - t(0, "ike", (S(1, None),)) * dx) + (P["eyz"][s_] - P["eyx"][s_]))
            s_ = (S(1, None), S(1, None), S(None))
            dx = hy[1:, 1:, :] - hy[:-1, 1:, :]
            dy = hx[1:, 1:, :] - hx[1:, :-1, :]
            P["ezx"] = P["ezx"].clone(); P["ezy"] = P["ezy"].clone()
            P["ezx"][s_] = t(0, "be", (S(1, None),)) * P["ezx"][s_] + t(0, "ce", (S(1, None),)) * dx
            P["ezy"][s_] = t(1, "be", (S(None), S(1, None))) * P["ezy"][s_] + t(1, "ce", (S(None), S(1, None))) * dy
            ez[s_] = ez[s_] + cb[s_] * ((t(0, "ike", (S(1, None),)) * dx - t(1, "ike", (S(None), S(1, None))) * dy) + (P["ezx"][s_] - P["ezy"][s_]))
        else:
            # fdtd3d.py:305-366
            hx[:, :-1, :-1] = hx[:, :-1, :-1] - a * ((ez[:, 1:, :-1] - ez[:, :-1, :-1]) - (ey[:, :-1, 1:] - ey[:, :-1, :-1]))
            hy[:-1, :, :-1] = hy[:-1, :, :-1] - a * ((ex[:-1, :, 1:] - ex[:-1, :, :-1]) - (ez[1:, :, :-1] - ez[:-1, :, :-1]))
            hz[:-1, :-1, :] = hz[:-1, :-1, :] - a * ((ey[1:, :-1, :] - ey[:-1, :-1, :]) - (ex[:-1, 1:, :] - ex[:-1, :-1, :]))
            ex, ey, ez = ex.clone(), ey.clone(), ez.clone()
            ex[:, 1:, 1:] = ex[:, 1:, 1:] + cb[:, 1:, 1:] * ((hz[:, 1:, 1:] - hz[:, :-1, 1:]) - (hy[:, 1:, 1:] - hy[:, 1:, :-1]))
            ey[1:, :, 1:] = ey[1:, :, 1:] + cb[1:, :, 1:] * ((hx[1:, :, 1:] - hx[1:, :, :-1]) - (hz[1:, :, 1:] - hz[:-1, :, 1:]))
            ez[1:, 1:, :] = ez[1:, 1:, :] + cb[1:, 1:, :] * ((hy[1:, 1:, :] - hy[:-1, 1:, :]) - (hx[1:, 1:, :] - hx[1:, :-1, :]))
            if damp is not None:
                ex, ey, ez = ex * damp, ey * damp, ez * damp
        f = [ex, ey, ez]
        for (ix, iy, iz), c, w in srcs:
            f[c] = f[c].clone()
            f[c][ix, iy, iz] = f[c][ix, iy, iz] + w[n]
        ex, ey, ez = f
        allf = (ex, ey, ez, hx, hy, hz)
        traces.append(torch.stack([allf[c][i, j, k] for (i, j, k, c) in spec.probes]))
    return torch.stack(traces)


def grad_eps(spec: rn.Spec3D, eps_r: np.ndarray, n_steps: int, dt: float, weights: np.ndarray):
    """J = sum(weights * traces**2) and dJ/d(eps_r), FP64 autograd."""
    e = torch.tensor(eps_r, dtype=torch.float64, requires_grad=True)
    tr = run(spec, e, n_steps, dt)
    J = (torch.from_numpy(weights) * tr ** 2).sum()
    J.backward()
    return float(J.detach()), e.grad.numpy(), tr.detach().numpy()
