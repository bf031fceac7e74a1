"""The FP64 C oracle (oracle/cpu_fdtd.c) is the checker of the large GPU
parity cases and the timed CPU baseline, so it is pinned here twice, on the
CPU:

* against the golden frames that the reference's own FDTD source produced
  (tests/golden, jaxphys src/neurosim/em/fdtd3d.py:280-404): every saved frame
  of every 3D case, all six components, bit for bit;
* against the NumPy restatement (oracle/ref_numpy.py) in the extension modes
  the reference lacks (CPML with kappa = 1, with kappa > 1 and CFS alpha, over
  a smooth permittivity map; PEC walls; Gaussian-pulse and sine sources;
  probes), bit for bit.
"""

import numpy as np
import pytest

from cases import eps_from_case3d, golden, load_cases, rn
from oracle.cpu_oracle import Oracle3DC

CASES = load_cases()
NAMES = ("ex", "ey", "ez", "hx", "hy", "hz")


@pytest.mark.parametrize("case", CASES["3d"], ids=lambda c: c["name"])
def test_c_oracle_equals_reference_frames(case):
    shape = tuple(case["size"])
    srcs = [dict(position=tuple(s["position"]), polarization=s["polarization"],
                 amplitude=s["amplitude"], kind="sine", frequency=s["frequency"])
            for s in case["sources"]]
    spec = rn.Spec3D(size=shape, dx=case["resolution"], boundary=case["boundary"],
                     pml_layers=case["pml_layers"], eps_r=eps_from_case3d(case), sources=srcs)
    dt = rn.default_dt_3d(case["resolution"])
    n = rn.n_steps_from_span(case["t_span"], dt)
    o = Oracle3DC(spec, dt=dt, t_start=case["t_span"][0])
    s = max(int(case["save_every"]), 1)
    frames = []
    for k in range(n):  # the reference keeps the state after steps 1, 1+s, ...
        o.run(1)
        if k % s == 0:
            frames.append([f.copy() for f in o.f])
    g = golden("3d", case["name"])
    assert len(frames) == int(g["n_saved"])
    for fi, gi in enumerate(g["frames"]):
        for c, name in enumerate(NAMES):
            np.testing.assert_array_equal(frames[gi][c], g[name][fi], err_msg=f"{name} {gi}")


def _cpml_spec(size, boundary, **kw):
    dt = rn.default_dt_3d(1.0)
    src = [dict(position=(size[0] // 2, size[1] // 2, size[2] // 2), polarization="z",
                amplitude=1.0, kind="gauss_sine", frequency=0.05 / dt, width_steps=6.0,
                delay_steps=20.0),
           dict(position=(3, 2, size[2] - 4), polarization="x", amplitude=0.5, kind="sine",
                frequency=0.03 / dt),
           dict(position=(size[0] - 3, 4, 5), polarization="y", amplitude=-0.7,
                kind="gauss_sine", frequency=0.04 / dt, width_steps=9.0, delay_steps=27.0)]
    probes = [(5, 5, 5, 2), (size[0] - 5, 3, size[2] - 5, 4), (2, 2, 2, 0), (7, 1, 9, 5)]
    return rn.Spec3D(size=size, dx=1.0, boundary=boundary, sources=src, probes=probes, **kw), dt


def _smooth_eps(shape, seed, lo, hi):
    from scipy.ndimage import gaussian_filter

    u = gaussian_filter(np.random.default_rng(seed).random(shape), sigma=2.0)
    u = (u - u.min()) / (u.max() - u.min())
    return lo + (hi - lo) * u


EXT_CASES = {
    "cpml_kappa1": dict(boundary="cpml", pml_layers=4, cpml=rn.CpmlParams()),
    "cpml_kappa_cfs": dict(boundary="cpml", pml_layers=5,
                           cpml=rn.CpmlParams(order=4.0, r0=1e-8, kappa_max=5.0,
                                              alpha_max=0.05)),
    "cpml_smooth_eps": dict(boundary="cpml", pml_layers=4, cpml=rn.CpmlParams(),
                            eps_r=_smooth_eps((14, 12, 16), 7, 1.0, 12.0)),
    "pec_smooth_eps": dict(boundary="pec", pml_layers=0,
                           eps_r=_smooth_eps((14, 12, 16), 8, 1.0, 6.0)),
    "absorbing_pulse": dict(boundary="absorbing", pml_layers=3),
}


@pytest.mark.parametrize("name", list(EXT_CASES))
def test_c_oracle_equals_numpy_restatement(name):
    kw = dict(EXT_CASES[name])
    spec, dt = _cpml_spec((14, 12, 16), **kw)
    a = rn.Oracle3D(spec, dt=dt)
    b = Oracle3DC(spec, dt=dt)
    pa = a.run(70)["probes"]
    pb = b.run(70)["probes"]
    assert np.abs(pa).max() > 0
    np.testing.assert_array_equal(pa, pb)
    for c, nm in enumerate(NAMES):
        np.testing.assert_array_equal(a.f[c], b.f[c], err_msg=nm)
    if spec.boundary == "cpml":  # the psi state as well
        for k, arr in zip(("hxy", "hxz", "hyz", "hyx", "hzx", "hzy",
                           "exy", "exz", "eyz", "eyx", "ezx", "ezy"), b.psi):
            np.testing.assert_array_equal(a.psi[k], arr, err_msg=k)
