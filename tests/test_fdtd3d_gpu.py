"""3D CUDA path against the oracle and the reference's golden vectors.

Tolerances (written per test):
  * FP32 fields against the FP64 reference: relative L2 of the E and of the H
    vector field <= 1e-5 while the fields carry the signal (a single
    component, e.g. Hz of a z-dipole, can be pure rounding noise, and a field
    that has decayed by decades into an absorbing layer leaves only the FP32
    rounding floor relative to its peak);
  * probe traces over the whole run against FP64: relative L2 <= 1e-5;
  * against the FP32 oracle (the same roundings): relative L2 <= 1e-6;
  * TMA kernel against generic kernel: bit for bit (same operations, same
    order), compared with np.array_equal (kappa = 1 CPML warps apply the
    CPML form with zero psi outside the slabs, equal in value to the plain
    update; only the sign of an exact zero may differ).
"""

import numpy as np
import pytest

from cases import golden, load_cases, rn
from gpu_helpers import (family_errors, grid3d_from_case, grid_fields, rel_l2, smooth_eps,
                         to_np)

pytestmark = pytest.mark.gpu

CASES = load_cases()["3d"]
COMPS = ("ex", "ey", "ez", "hx", "hy", "hz")
TOL = 1e-5


def _assert_fields(got6, ref6, tol=TOL, what=""):
    eE, eH = family_errors(got6, ref6)
    assert eE <= tol and eH <= tol, f"{what}: rel L2 E {eE:.3e} H {eH:.3e} > {tol}"


@pytest.mark.parametrize("path", ["auto", "generic"])
@pytest.mark.parametrize("case", CASES, ids=lambda c: c["name"])
def test_golden_parity(cuda, case, path):
    g = grid3d_from_case(case, path=path)
    h = g.simulate(t_span=tuple(case["t_span"]), save_every=case["save_every"])
    ref = golden("3d", case["name"])
    assert h.t.shape[0] == int(ref["n_saved"])
    np.testing.assert_allclose(to_np(h.t), ref["t"], rtol=0, atol=0)
    fr = ref["frames"]
    for j in range(len(fr)):
        got = [to_np(getattr(h, k))[fr[j]] for k in COMPS]
        want = [ref[k][j] for k in COMPS]
        if max(np.abs(w).max() for w in want) == 0.0:
            assert max(np.abs(x).max() for x in got) == 0.0
            continue
        _assert_fields(got, want, what=f"{case['name']} frame {fr[j]}")
    np.testing.assert_array_equal(to_np(h.grid_z), ref["grid_z"])


@pytest.mark.parametrize("case", [c for c in CASES if c["size"][2] % 4 == 0
                                  and c["boundary"] != "periodic"], ids=lambda c: c["name"])
def test_tma_bitwise_equals_generic(cuda, case):
    a = grid3d_from_case(case, path="tma").simulate(tuple(case["t_span"]), save_every=1)
    b = grid3d_from_case(case, path="generic").simulate(tuple(case["t_span"]), save_every=1)
    for k in COMPS:
        assert np.array_equal(to_np(getattr(a, k)), to_np(getattr(b, k))), k


# launch shapes in the library's TMA registry (checked against the library below)
N_TMA_CONFIGS = 12


def test_tma_registry_size(cuda):
    from jaxphys_b200 import _native as nat

    assert nat.load().jxf_num_tma_configs() == N_TMA_CONFIGS


def _cpml_grid(path, size, eps, sources, probes, n_pml=6, cpml=None):
    from jaxphys_b200 import CPMLSpec, EMGrid3D, PointSource3D

    g = EMGrid3D(size=size, resolution=1.0, boundary="cpml", pml_layers=n_pml, path=path,
                 cpml=cpml or CPMLSpec())
    for s in sources:
        g.add_source(PointSource3D(**s))
    if eps is not None:
        g.set_permittivity(eps)
    for p in probes:
        g.add_probe(p[:3], ("ex", "ey", "ez", "hx", "hy", "hz")[p[3]])
    return g


def _oracle_cpml(size, eps, sources, probes, n_steps, n_pml=6, cpml=None, dtype=np.float64):
    dt = rn.default_dt_3d(1.0)
    srcs = []
    for s in sources:
        d = dict(position=s["position"], polarization=s.get("polarization", "z"),
                 amplitude=s.get("amplitude", 1.0), kind=s.get("waveform", "sine"),
                 frequency=s["frequency"], width_steps=s.get("width_steps", 30.0))
        d["delay_steps"] = s.get("delay_steps") or 4.0 * d["width_steps"]
        srcs.append(d)
    cp = rn.CpmlParams() if cpml is None else rn.CpmlParams(cpml.order, cpml.r0, cpml.kappa_max,
                                                            cpml.alpha_max)
    spec = rn.Spec3D(size=size, dx=1.0, boundary="cpml", pml_layers=n_pml, eps_r=eps,
                     sources=srcs, probes=probes, cpml=cp)
    o = rn.Oracle3D(spec, dt=dt, dtype=dtype)
    out = o.run(n_steps)
    return o, out


def _gauss(pos, pol="z", amp=1.0, width=10.0, f=None):
    dt = rn.default_dt_3d(1.0)
    return dict(frequency=f if f is not None else 0.05 / dt, position=pos, amplitude=amp,
                polarization=pol, waveform="gauss_sine", width_steps=width)


@pytest.mark.parametrize("path", ["tma", "generic"])
def test_cpml_parity_with_eps_and_probes(cuda, path):
    size = (26, 22, 28)
    eps = smooth_eps(size, 1.0, 6.0, seed=3)
    sources = [_gauss((13, 11, 14)), _gauss((5, 17, 8), "x", 1.0, 8.0),
               _gauss((20, 3, 24), "y", 1.0, 12.0)]
    probes = [(13, 11, 20, 2), (2, 2, 2, 0), (24, 20, 26, 4), (10, 10, 10, 5), (0, 21, 27, 1)]
    n_mid, n = 45, 160
    g = _cpml_grid(path, size, eps, sources, probes)
    g.prepare(dt=rn.default_dt_3d(1.0))
    tr1 = to_np(g.run(n_mid))
    o64, out64 = _oracle_cpml(size, eps, sources, probes, n_mid)
    o32, out32 = _oracle_cpml(size, eps, sources, probes, n_mid, dtype=np.float32)
    # pulse inside the box: FP32 GPU vs FP64
    _assert_fields(grid_fields(g), o64.f, what="t=45 vs FP64")
    tr2 = to_np(g.run(n - n_mid))
    p64 = np.vstack([out64["probes"], o64.run(n - n_mid)["probes"]])
    p32 = np.vstack([out32["probes"], o32.run(n - n_mid)["probes"]])
    tr = np.vstack([tr1, tr2])
    # after the pulse has gone into the CPML: same-precision oracle
    _assert_fields(grid_fields(g), o32.f, tol=1e-6, what="t=160 vs FP32")
    assert rel_l2(tr, p64) <= TOL
    assert rel_l2(tr, p32) <= 1e-6


def test_cpml_tma_bitwise_generic_with_kappa_alpha(cuda):
    from jaxphys_b200 import CPMLSpec

    size = (24, 24, 32)
    eps = smooth_eps(size, 1.0, 4.0, seed=5)
    sources = [_gauss((12, 12, 16)), _gauss((3, 3, 3), "y")]
    cp = CPMLSpec(order=3.0, r0=1e-6, kappa_max=4.0, alpha_max=0.05)
    res = []
    for path in ("tma", "generic"):
        g = _cpml_grid(path, size, eps, sources, [], n_pml=8, cpml=cp)
        g.prepare(dt=rn.default_dt_3d(1.0))
        g.run(100)
        res.append({k: to_np(g.field(k)) for k in COMPS})
    for k in COMPS:
        assert np.array_equal(res[0][k], res[1][k]), k
    o, _ = _oracle_cpml(size, eps, sources, [], 100, n_pml=8, cpml=cp, dtype=np.float32)
    _assert_fields([res[0][k] for k in COMPS], o.f, tol=1e-6, what="vs FP32")


@pytest.mark.parametrize("cfg", range(N_TMA_CONFIGS))
@pytest.mark.parametrize("chunk", [1, 3, 64])
@pytest.mark.parametrize("split", [0, 1])
def test_every_launch_shape_bitwise(cuda, cfg, chunk, split):
    """Every TMA tile shape and x-chunk (including 1-plane chunks, ragged tiles
    and sources on chunk seams) reproduces the generic kernel exactly."""
    from jaxphys_b200 import _native as nat

    size = (19, 37, 44)  # ragged against every tile
    eps = smooth_eps(size, 1.0, 3.0, seed=cfg)
    sources = [_gauss((3, 18, 22)), _gauss((6, 0, 43), "x"), _gauss((18, 36, 0), "y"),
               _gauss((9, 15, 31), "z", 0.5), _gauss((9, 15, 31), "z", 0.25)]
    probes = [(3, 18, 22, 2), (18, 36, 43, 0)]
    out = []
    for path in ("tma", "generic"):
        for bnd in ("cpml",):
            g = _cpml_grid(path, size, eps, sources, probes, n_pml=4)
            g.prepare(dt=rn.default_dt_3d(1.0))
            if path == "tma":
                nat.check(nat.load().jxf_grid3d_set_launch(g._h, cfg, chunk), "set_launch")
                nat.check(nat.load().jxf_grid3d_set_axis_split(g._h, split), "set_axis_split")
            tr = to_np(g.run(60))
            out.append(({k: to_np(g.field(k)) for k in COMPS}, tr))
    for k in COMPS:
        assert np.array_equal(out[0][0][k], out[1][0][k]), k
    assert np.array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("cfg", range(N_TMA_CONFIGS))
def test_absorbing_launch_shapes_bitwise(cuda, cfg):
    from jaxphys_b200 import EMGrid3D, PointSource3D
    from jaxphys_b200 import _native as nat

    res = []
    for path in ("tma", "generic"):
        g = EMGrid3D(size=(21, 33, 40), resolution=0.01, pml_layers=5, path=path)
        g.add_source(PointSource3D(frequency=5e9, position=(10, 16, 20)))
        g.add_source(PointSource3D(frequency=4e9, position=(0, 32, 39), polarization="x"))
        g.prepare()
        if path == "tma":
            nat.check(nat.load().jxf_grid3d_set_launch(g._h, cfg, 4), "set_launch")
        g.run(50)
        res.append({k: to_np(g.field(k)) for k in COMPS})
    for k in COMPS:
        assert np.array_equal(res[0][k], res[1][k]), k


def test_config1_reference_semantics(cuda):
    """64^3, 500 steps, dx=1, 8-cell damping boundary, Ez sine point source at
    the centre (f = 0.05/dt), 8 seeded interior Ez probes: the reference's own
    semantics (fdtd3d.py) against the FP64 oracle."""
    from jaxphys_b200 import EMGrid3D, PointSource3D
    from oracle.cpu_oracle import Oracle3DC

    dt = rn.default_dt_3d(1.0)
    rng = np.random.default_rng(1)
    probes = [tuple(int(v) for v in rng.integers(8, 56, size=3)) + (2,) for _ in range(8)]
    g = EMGrid3D(size=(64, 64, 64), resolution=1.0, boundary="absorbing", pml_layers=8)
    g.add_source(PointSource3D(frequency=0.05 / dt, position=(32, 32, 32)))
    for p in probes:
        g.add_probe(p[:3], "ez")
    g.prepare()
    tr = to_np(g.run(500))
    spec = rn.Spec3D(size=(64, 64, 64), dx=1.0, boundary="absorbing", pml_layers=8,
                     sources=[dict(position=(32, 32, 32), polarization="z", amplitude=1.0,
                                   kind="sine", frequency=0.05 / dt)], probes=probes)
    o = Oracle3DC(spec, dt=dt)
    out = o.run(500)
    _assert_fields(grid_fields(g), o.f, what="fields after 500 steps")
    assert rel_l2(tr, out["probes"]) <= TOL


def _cfg_probes(n, count, seed):
    rng = np.random.default_rng(seed)
    return [tuple(int(v) for v in rng.integers(n // 8, n - n // 8, size=3)) + (2,)
            for _ in range(count)]


@pytest.mark.parametrize("path", ["tma", "generic"])
def test_config1_cpml_pulse(cuda, path):
    """Config 1 in extension semantics: 64^3, 8-cell CPML (m=3, R0=1e-6),
    Gaussian-modulated Ez dipole (f0=0.05/dt, width 30 steps), 500 steps,
    8 seeded interior Ez probes."""
    from oracle.cpu_oracle import Oracle3DC

    n = 64
    probes = _cfg_probes(n, 8, seed=1)
    src = [_gauss((32, 32, 32), width=30.0)]
    g = _cpml_grid(path, (n, n, n), None, src, probes, n_pml=8)
    g.prepare(dt=rn.default_dt_3d(1.0))
    tr1 = to_np(g.run(160))
    spec = rn.Spec3D(size=(n, n, n), dx=1.0, boundary="cpml", pml_layers=8,
                     sources=[dict(position=(32, 32, 32), polarization="z", amplitude=1.0,
                                   kind="gauss_sine", frequency=0.05 / rn.default_dt_3d(1.0),
                                   width_steps=30.0, delay_steps=120.0)], probes=probes)
    o = Oracle3DC(spec, dt=rn.default_dt_3d(1.0))
    p1 = o.run(160)["probes"]
    _assert_fields(grid_fields(g), o.f, what="t=160")
    tr2 = to_np(g.run(340))
    p2 = o.run(340)["probes"]
    assert rel_l2(np.vstack([tr1, tr2]), np.vstack([p1, p2])) <= TOL


def test_config2_sphere_checksum(cuda):
    """Config 2: 128^3, 10-cell CPML, eps_r=4 sphere (radius 20) at a seeded
    offset, pulsed Ez dipole, 16 probes over 1000 steps, plus the full-field
    checksum (sum and L2 of E and H) while the pulse is in the box."""
    from jaxphys_b200 import DielectricRegion, EMGrid3D, PointSource3D
    from oracle.cpu_oracle import Oracle3DC

    n = 128
    dt = rn.default_dt_3d(1.0)
    rng = np.random.default_rng(2)
    c = np.array([64, 64, 64]) + rng.integers(-16, 17, size=3)
    ix, iy, iz = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    mask = (ix - c[0]) ** 2 + (iy - c[1]) ** 2 + (iz - c[2]) ** 2 <= 20 ** 2
    probes = _cfg_probes(n, 16, seed=2)
    g = EMGrid3D(size=(n, n, n), resolution=1.0, boundary="cpml", pml_layers=10)
    g.add_source(PointSource3D(frequency=0.05 / dt, position=(64, 64, 64),
                               waveform="gauss_sine", width_steps=30.0))
    g.add_material(DielectricRegion(mask=mask, epsilon_r=4.0))
    for p in probes:
        g.add_probe(p[:3], "ez")
    g.prepare()
    tr1 = to_np(g.run(250))
    spec = rn.Spec3D(size=(n, n, n), dx=1.0, boundary="cpml", pml_layers=10,
                     eps_r=np.where(mask, 4.0, 1.0),
                     sources=[dict(position=(64, 64, 64), polarization="z", amplitude=1.0,
                                   kind="gauss_sine", frequency=0.05 / dt, width_steps=30.0,
                                   delay_steps=120.0)], probes=probes)
    o = Oracle3DC(spec, dt=dt)
    p1 = o.run(250)["probes"]
    got = grid_fields(g)
    _assert_fields(got, o.f, what="t=250")
    for fam in (slice(0, 3), slice(3, 6)):
        s_got = sum(float(np.sum(np.asarray(x, np.float64))) for x in got[fam])
        s_ref = sum(float(np.sum(x)) for x in o.f[fam])
        l2_got = np.sqrt(sum(float(np.sum(np.asarray(x, np.float64) ** 2)) for x in got[fam]))
        l2_ref = np.sqrt(sum(float(np.sum(x ** 2)) for x in o.f[fam]))
        assert abs(l2_got - l2_ref) <= 1e-5 * l2_ref
        assert abs(s_got - s_ref) <= 1e-5 * l2_ref * np.sqrt(n ** 3)
    tr2 = to_np(g.run(750))
    p2 = o.run(750)["probes"]
    assert rel_l2(np.vstack([tr1, tr2]), np.vstack([p1, p2])) <= TOL


def _rel_l2_by_component(got_fn, ref6, comps):
    """Relative L2 of a vector field over the components ``comps``, summed
    one component at a time (a 512^3 FP64 stack would take 3 GB of host
    memory per family)."""
    num = den = 0.0
    for c in comps:
        g = np.asarray(got_fn(c), np.float64)
        num += float(np.sum((g - ref6[c]) ** 2))
        den += float(np.sum(ref6[c] ** 2))
        del g
    return float(np.sqrt(num / den))


def test_config3_512_cpml12_smooth_eps(cuda):
    """Config 3: 512^3 FP32, 200 steps, 12-cell CPML (m=3, R0=1e-6), eps_r
    from seeded uniform noise smoothed by a Gaussian (sigma = 6 cells) and
    rescaled to [1, 12], Gaussian-modulated Ez dipole at the centre (f0 =
    0.05/dt, width 30 steps), 16 seeded Ez probes.  Checked against the FP64
    C oracle: probe traces over the whole run and the E and H fields after
    step 200 (the pulse is still inside the box), relative L2 <= 1e-5
    (tolerance of the 3D FP32 path).  The probes sit within 20 cells of the
    source: in 200 steps the pulse (peak at step 120, eps_r ~ 6.5 on average)
    travels ~30 cells, and probes further out would see only the Yee
    stencil's precursor (FP64 values of 1e-40 and below), which FP32 cannot
    represent and which says nothing about the kernel."""
    import psutil
    from scipy.ndimage import gaussian_filter

    from oracle.cpu_oracle import Oracle3DC

    # the FP64 oracle holds 6 fields, 12 full-size psi arrays and cb: ~20 GB
    if psutil.virtual_memory().available < 48e9:
        pytest.skip("the 512^3 FP64 oracle needs ~20 GB of free host memory")
    n, steps, pml = 512, 200, 12
    dt = rn.default_dt_3d(1.0)
    rng = np.random.default_rng(3)
    u = gaussian_filter(rng.random((n, n, n), dtype=np.float32), sigma=6, mode="wrap")
    u = (u - u.min()) / (u.max() - u.min())
    eps = (1.0 + 11.0 * u.astype(np.float64))
    del u
    prng = np.random.default_rng(3)
    probes = [tuple(int(n // 2 + v) for v in prng.integers(-20, 21, size=3)) + (2,)
              for _ in range(16)]
    src = [_gauss((n // 2, n // 2, n // 2), width=30.0)]
    g = _cpml_grid("auto", (n, n, n), None, src, probes, n_pml=pml)
    g.set_permittivity(eps)
    g.prepare(dt=dt)
    assert g.info()["path"] == 2, "512^3 CPML must run on the TMA path"
    tr = to_np(g.run(steps))
    g.check()
    spec = rn.Spec3D(size=(n, n, n), dx=1.0, boundary="cpml", pml_layers=pml, eps_r=eps,
                     sources=[dict(position=(n // 2,) * 3, polarization="z", amplitude=1.0,
                                   kind="gauss_sine", frequency=0.05 / dt, width_steps=30.0,
                                   delay_steps=120.0)], probes=probes)
    del eps
    o = Oracle3DC(spec, dt=dt)
    out = o.run(steps)
    assert np.abs(out["probes"]).max() > 1e-4  # the probes see the pulse
    assert rel_l2(tr, out["probes"]) <= TOL
    eE = _rel_l2_by_component(lambda c: to_np(g.field(COMPS[c])), o.f, (0, 1, 2))
    eH = _rel_l2_by_component(lambda c: to_np(g.field(COMPS[c])), o.f, (3, 4, 5))
    assert eE <= TOL and eH <= TOL, (eE, eH)


def test_finite_check_raises(cuda):
    from jaxphys_b200 import EMGrid3D, NumericalInstabilityError, PointSource3D

    g = EMGrid3D(size=(16, 16, 16))
    g.add_source(PointSource3D(frequency=5e9, position=(8, 8, 8)))
    g.prepare()
    bad = np.zeros((16, 16, 16), np.float32)
    bad[3, 4, 5] = np.nan
    g.set_field("hx", bad)
    g.step(2)
    with pytest.raises(NumericalInstabilityError):
        g.check()


# -------- the reference's own behaviour tests (tests/test_fdtd3d.py:16-139) --------

def test_basic_simulation(cuda):
    from jaxphys_b200 import EMGrid3D, PointSource3D

    grid = EMGrid3D(size=(20, 20, 20), resolution=0.01)
    grid.add_source(PointSource3D(frequency=3e9, position=(10, 10, 10)))
    fields = grid.simulate(t_span=(0, 5e-10), save_every=10)
    assert fields.ez.shape[1:] == (20, 20, 20)
    assert fields.t.shape[0] > 0


def test_source_excites_field(cuda):
    from jaxphys_b200 import EMGrid3D, PointSource3D

    grid = EMGrid3D(size=(20, 20, 20), resolution=0.01)
    grid.add_source(PointSource3D(frequency=3e9, position=(10, 10, 10), amplitude=1.0))
    fields = grid.simulate(t_span=(0, 3e-10), save_every=5)
    assert float(fields.ez[-1].abs().max()) > 0.0


def test_all_six_components(cuda):
    from jaxphys_b200 import EMGrid3D, PointSource3D

    grid = EMGrid3D(size=(16, 16, 16), resolution=0.01)
    grid.add_source(PointSource3D(frequency=5e9, position=(8, 8, 8)))
    f = grid.simulate(t_span=(0, 2e-10), save_every=5)
    assert f.ex.shape == f.ey.shape == f.ez.shape == f.hx.shape == f.hy.shape == f.hz.shape
    assert f.ex.shape[1:] == (16, 16, 16)


@pytest.mark.parametrize("pol", ["x", "y"])
def test_polarization(cuda, pol):
    from jaxphys_b200 import EMGrid3D, PointSource3D

    grid = EMGrid3D(size=(16, 16, 16), resolution=0.01)
    grid.add_source(PointSource3D(frequency=3e9, position=(8, 8, 8), polarization=pol))
    f = grid.simulate(t_span=(0, 2e-10), save_every=5)
    assert float(getattr(f, "e" + pol)[-1].abs().max()) > 0.0


def test_dielectric_material(cuda):
    import torch

    from jaxphys_b200 import DielectricRegion, EMGrid3D, PointSource3D

    free = EMGrid3D(size=(16, 16, 16), resolution=0.01)
    free.add_source(PointSource3D(frequency=5e9, position=(8, 8, 8)))
    diel = EMGrid3D(size=(16, 16, 16), resolution=0.01)
    diel.add_source(PointSource3D(frequency=5e9, position=(8, 8, 8)))
    mask = np.zeros((16, 16, 16), dtype=bool)
    mask[10:] = True
    diel.add_material(DielectricRegion(mask=mask, epsilon_r=4.0))
    a = free.simulate(t_span=(0, 1e-9), save_every=20)
    b = diel.simulate(t_span=(0, 1e-9), save_every=20)
    assert not torch.allclose(a.ez[-1], b.ez[-1])


def test_periodic_boundary(cuda):
    import torch

    from jaxphys_b200 import EMGrid3D, PointSource3D

    ga = EMGrid3D(size=(16, 16, 16), resolution=0.01, boundary="absorbing")
    gp = EMGrid3D(size=(16, 16, 16), resolution=0.01, boundary="periodic", pml_layers=0)
    s = PointSource3D(frequency=5e9, position=(8, 8, 8))
    ga.add_source(s)
    gp.add_source(s)
    a = ga.simulate(t_span=(0, 2e-10), save_every=5)
    p = gp.simulate(t_span=(0, 2e-10), save_every=5)
    assert not torch.allclose(a.ez[-1], p.ez[-1])


def test_grid_coordinates(cuda):
    from jaxphys_b200 import EMGrid3D, PointSource3D

    grid = EMGrid3D(size=(16, 16, 16), resolution=0.02)
    grid.add_source(PointSource3D(frequency=1e9, position=(8, 8, 8)))
    f = grid.simulate(t_span=(0, 1e-10), save_every=5)
    assert f.grid_x.shape == (16,)
    assert float(f.grid_x[1] - f.grid_x[0]) == pytest.approx(0.02)


def test_history_streamed_to_host_equals_device(cuda):
    """simulate(history="host") streams frames to pinned host memory through
    two device staging slots; the frames equal the device-resident history."""
    from jaxphys_b200 import EMGrid3D, PointSource3D

    def make():
        g = EMGrid3D(size=(20, 24, 28), resolution=0.01, boundary="absorbing", pml_layers=4)
        g.add_source(PointSource3D(frequency=5e9, position=(10, 12, 14)))
        return g

    t_span = (0.0, 60 * make().default_dt())
    a = make().simulate(t_span, save_every=7)
    b = make().simulate(t_span, save_every=7, history="host")
    assert not b.ez.is_cuda and b.ez.is_pinned()
    np.testing.assert_array_equal(to_np(a.t), to_np(b.t))
    for k in COMPS:
        assert np.array_equal(to_np(getattr(a, k)), to_np(getattr(b, k))), k
    c = make().simulate(t_span, save_every=7, history="host", output="numpy")
    assert isinstance(c.hx, np.ndarray) and np.array_equal(c.hx, to_np(a.hx))
