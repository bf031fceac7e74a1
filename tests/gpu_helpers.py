"""Helpers shared by the GPU tests: run golden cases through the package."""

from __future__ import annotations

import numpy as np

from cases import box_mask, rn


def grid3d_from_case(case, path="auto"):
    from jaxphys_b200 import DielectricRegion, EMGrid3D, PointSource3D

    g = EMGrid3D(size=tuple(case["size"]), resolution=case["resolution"],
                 boundary=case["boundary"], pml_layers=case["pml_layers"], path=path)
    for s in case["sources"]:
        g.add_source(PointSource3D(frequency=s["frequency"], position=tuple(s["position"]),
                                   amplitude=s["amplitude"], polarization=s["polarization"]))
    for m in case["materials"]:
        g.add_material(DielectricRegion(mask=box_mask(tuple(case["size"]), m["box"]),
                                        epsilon_r=m["epsilon_r"]))
    return g


def grid2d_from_case(case):
    from jaxphys_b200 import EMGrid, PlaneWave, Wall

    g = EMGrid(size=tuple(case["size"]), resolution=case["resolution"],
               boundary=case["boundary"], pml_layers=case["pml_layers"])
    for s in case["sources"]:
        g.add_source(PlaneWave(frequency=s["frequency"], y=s["y"], amplitude=s["amplitude"]))
    for w in case["walls"]:
        g.add_conductor(Wall(y=w["y"], gap_start=w["gap_start"], gap_end=w["gap_end"]))
    return g


def rel_l2(a, b):
    return rn.rel_l2(np.asarray(a, np.float64), np.asarray(b, np.float64))


def to_np(t):
    return t.detach().cpu().numpy() if hasattr(t, "detach") else np.asarray(t)


def smooth_eps(shape, lo, hi, seed, sigma=2.0):
    from scipy.ndimage import gaussian_filter

    rng = np.random.default_rng(seed)
    u = gaussian_filter(rng.random(shape), sigma=sigma, mode="wrap")
    u = (u - u.min()) / (u.max() - u.min())
    return lo + (hi - lo) * u


def family_errors(got6, ref6):
    """Relative L2 of the E and H vector fields (each three components)."""
    g = [np.asarray(x, np.float64) for x in got6]
    r = [np.asarray(x, np.float64) for x in ref6]
    return (rn.rel_l2(np.stack(g[:3]), np.stack(r[:3])),
            rn.rel_l2(np.stack(g[3:]), np.stack(r[3:])))


def grid_fields(g):
    return [to_np(g.field(k)) for k in ("ex", "ey", "ez", "hx", "hy", "hz")]
