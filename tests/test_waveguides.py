"""Waveguide analysis and mode ports on the CPU.

The analysis tests follow the reference's own (``tests/test_em.py:82-123``,
``tests/test_edge_cases.py:289-298,1328-1359``).  The port tests check the
transverse profiles on the Yee grid, the conductor tube, and -- through the
NumPy oracle with +inf permittivity on the walls -- that a TE10 port drives a
guided mode above cutoff and an evanescent field below it.
"""

import numpy as np
import pytest

from jaxphys_b200 import ConfigurationError, PhysicsError
from jaxphys_b200.em.waveguides import ModeSource3D, RectangularWaveguide, tube_mask
from oracle import ref_numpy as rn

C0 = 299792458.0


def test_wr90_cutoff():
    wg = RectangularWaveguide(a=0.02286, b=0.01016)
    assert wg.cutoff_frequency(1, 0) == pytest.approx(6.56e9, rel=0.01)


def test_te10_mode():
    mode = RectangularWaveguide(a=0.02286, b=0.01016).compute_mode("TE", 1, 0, n_points=50)
    assert mode.field_pattern.shape == (50, 50)
    assert mode.cutoff_frequency > 0
    np.testing.assert_allclose(mode.field_pattern[:, 7], np.cos(np.pi * mode.x / 0.02286))


def test_tm11_mode():
    mode = RectangularWaveguide(a=0.02, b=0.01).compute_mode("TM", 1, 1, n_points=50)
    assert mode.mode_type == "TM"
    assert np.all(mode.field_pattern[[0, -1], :] < 1e-12)


def test_evanescent_mode():
    with pytest.raises(PhysicsError):
        RectangularWaveguide(a=0.02286, b=0.01016).propagation_constant(1e9, 1, 0)


def test_propagation_constant():
    wg = RectangularWaveguide(a=0.02286, b=0.01016)
    f = 10e9
    k = 2 * np.pi * f / C0
    kc = np.pi / 0.02286
    assert wg.propagation_constant(f, 1, 0) == pytest.approx(np.sqrt(k * k - kc * kc), rel=1e-12)


def test_invalid_te00():
    with pytest.raises(ConfigurationError):
        RectangularWaveguide(a=0.02, b=0.01).compute_mode("TE", 0, 0)


def test_dispersion_relation():
    wg = RectangularWaveguide(a=0.02286, b=0.01016)
    freqs = np.linspace(5e9, 15e9, 100)
    beta = wg.dispersion_relation(1, 0, freqs)
    fc = wg.cutoff_frequency(1, 0)
    assert np.all(np.isnan(beta[freqs < fc]))
    assert np.all(beta[freqs > fc] > 0)


def test_waveguide_cutoff_ordering():
    wg = RectangularWaveguide(a=0.02286, b=0.01016)
    assert wg.cutoff_frequency(1, 0) < wg.cutoff_frequency(2, 0)
    assert wg.cutoff_frequency(1, 0) < wg.cutoff_frequency(0, 1)


@pytest.mark.parametrize("a,b", [(-0.01, 0.01), (0.0, 0.01)])
def test_non_positive_dimensions_raise(a, b):
    with pytest.raises(ConfigurationError, match="positive"):
        RectangularWaveguide(a=a, b=b)


def test_invalid_mode_type():
    with pytest.raises(ConfigurationError, match="TE"):
        RectangularWaveguide(a=0.02, b=0.01).compute_mode("XX", 1, 0)


def test_tm_mode_requires_mn_ge_1():
    with pytest.raises(ConfigurationError, match="m >= 1"):
        RectangularWaveguide(a=0.02, b=0.01).compute_mode("TM", 0, 1)


# ------------------------------------------------------------------ ports


def test_te10_port_profile():
    eu, ev = ModeSource3D("TE", 1, 0, 1e9, index=4, origin=(1, 1), extent=(16, 8)).profile()
    assert np.all(eu == 0)
    i = np.arange(17)
    want = np.sin(np.pi * i / 16)[:, None] * np.ones((1, 9))
    want[:, [0, 8]] = 0.0
    want[[0, 16], :] = 0.0
    np.testing.assert_allclose(ev, want / want.max(), atol=1e-15)


def test_port_profiles_zero_on_walls_and_orthogonal():
    profs = {}
    for mt, m, n in (("TE", 1, 0), ("TE", 2, 0), ("TE", 0, 1), ("TE", 1, 1), ("TM", 1, 1),
                     ("TM", 2, 1)):
        eu, ev = ModeSource3D(mt, m, n, 1e9, index=0, origin=(0, 0), extent=(20, 12)).profile()
        for p in (eu, ev):
            assert np.all(p[[0, -1], :] == 0) and np.all(p[:, [0, -1]] == 0)
        assert max(np.abs(eu).max(), np.abs(ev).max()) == pytest.approx(1.0)
        profs[(mt, m, n)] = np.concatenate([eu.ravel(), ev.ravel()])
    # distinct TE modes of a rectangular guide are orthogonal on the aperture
    # (up to the half-cell staggering of the Yee samples)
    keys = [("TE", 1, 0), ("TE", 2, 0), ("TE", 0, 1)]
    for x in range(3):
        for y in range(x + 1, 3):
            a, b = profs[keys[x]], profs[keys[y]]
            assert abs(a @ b) / np.linalg.norm(a) / np.linalg.norm(b) < 0.05


@pytest.mark.parametrize("axis", ["x", "y", "z"])
def test_port_point_sources_axes(axis):
    size = (24, 20, 22)
    port = ModeSource3D("TE", 1, 0, 1e9, index=5, origin=(2, 3), extent=(12, 6), axis=axis,
                        amplitude=2.0)
    src = port.point_sources(size)
    w = "xyz".index(axis)
    v = (w + 2) % 3
    assert all(s.position[w] == 5 for s in src)
    assert {s.polarization for s in src} == {"xyz"[v]}   # TE10: E along v only
    assert max(abs(s.amplitude) for s in src) == pytest.approx(2.0)
    assert len(src) == 11 * 5


def test_port_out_of_grid():
    port = ModeSource3D("TE", 1, 0, 1e9, index=5, origin=(2, 3), extent=(12, 6))
    with pytest.raises(ConfigurationError, match="out of grid"):
        port.point_sources((14, 20, 20))
    with pytest.raises(ConfigurationError, match="out of grid"):
        ModeSource3D("TE", 1, 0, 1e9, index=20, origin=(2, 3), extent=(12, 6)).point_sources(
            (20, 20, 20))
    with pytest.raises(ConfigurationError, match="2x2"):
        ModeSource3D("TE", 1, 0, 1e9, index=2, origin=(2, 3), extent=(1, 6)).profile()


def test_port_from_waveguide():
    wg = RectangularWaveguide(a=0.016, b=0.008)
    p = wg.port("TE", 1, 0, 1.5 * wg.cutoff_frequency(1, 0), resolution=0.001, index=3,
                origin=(1, 1))
    assert p.extent == (16, 8)
    with pytest.raises(ConfigurationError):
        wg.port("TM", 1, 0, 1e10, resolution=0.001, index=3, origin=(1, 1))


def test_tube_mask():
    m = tube_mask((30, 20, 40), (23, 10), (2, 3), "z", (5, 35))
    assert m.sum() == 66 * 30
    assert m[2, 3:14, 5].all() and m[25, 3:14, 34].all() and not m[2, 3, 4]
    assert not m[3:25, 4:13, :].any()
    mx = tube_mask((40, 30, 20), (23, 10), (2, 3), "x")
    assert mx.shape == (40, 30, 20) and mx.sum() == 66 * 40 and mx[7, 2, 3:14].all()
    with pytest.raises(ConfigurationError, match="out of grid"):
        tube_mask((20, 20, 20), (23, 10), (2, 3), "z")


def test_grid_conductor_api():
    from jaxphys_b200 import EMGrid3D

    g = EMGrid3D((20, 12, 16), resolution=1.0, boundary="pec")
    wall = tube_mask(g.size, (16, 8), (1, 1), "z")
    g.add_conductor(wall)
    eps = g.epsilon_r()
    assert np.all(np.isinf(eps[wall])) and np.all(eps[~wall] == 1.0)
    with pytest.raises(ConfigurationError, match="doesn't match"):
        g.add_conductor(np.zeros((3, 3, 3), bool))
    g.add_source(ModeSource3D("TE", 1, 0, 1e6, index=4, origin=(1, 1), extent=(16, 8)))
    assert len(g._sources) == 15 * 7


# ------------------------------------------------- oracle: guided propagation

SIZE = (20, 12, 140)
A, B = 16, 8


def oracle_guide(f, steps, dtype=np.float32, every=10):
    """TE10 port at z = 20 of a closed metal guide (walls = +inf permittivity),
    gauss_sine pulse of 100 steps; RMS of Ey on the source plane and 40 cells
    downstream every ``every`` steps, and the downstream plane at its peak."""
    port = ModeSource3D("TE", 1, 0, f, index=20, origin=(1, 1), extent=(A, B),
                        waveform="gauss_sine", width_steps=100, delay_steps=400)
    srcs = [dict(position=s.position, polarization=s.polarization, amplitude=s.amplitude,
                 kind="gauss_sine", frequency=s.frequency, width_steps=100, delay_steps=400)
            for s in port.point_sources(SIZE)]
    eps = np.where(tube_mask(SIZE, (A, B), (1, 1), "z"), np.inf, 1.0)
    o = rn.Oracle3D(rn.Spec3D(size=SIZE, dx=1.0, boundary="pec", eps_r=eps, sources=srcs),
                    dtype=dtype)
    near, far, best = [], [], (0.0, None)
    for k in range(steps):
        o.step()
        if k % every == 0:
            ey = o.f[1]
            near.append(np.sqrt(np.mean(ey[:, :, 20] ** 2)))
            far.append(np.sqrt(np.mean(ey[:, :, 60] ** 2)))
            if far[-1] > best[0]:
                best = (far[-1], ey[:, :, 60].copy())
    return np.array(near), np.array(far), best[1], o


def te10_correlation(plane):
    """|correlation| of an Ey plane inside the guide with sin(pi x / a) (the
    sign depends on the half-cycle the plane was taken at)."""
    prof = plane[2:A + 1, 2:B + 1]
    ref = np.sin(np.pi * (np.arange(2, A + 1) - 1) / A)[:, None] * np.ones((1, B - 1))
    return abs(float(np.sum(prof * ref) / np.linalg.norm(prof) / np.linalg.norm(ref)))


def test_oracle_te10_guided_and_evanescent():
    fc = C0 / (2 * A)
    near, far, plane, o = oracle_guide(1.4 * fc, 900)
    assert far.max() / near.max() > 0.5
    assert te10_correlation(plane) > 0.98
    # metal cells hold zero E
    wall = tube_mask(SIZE, (A, B), (1, 1), "z")
    assert all(np.all(o.f[c][wall] == 0) for c in range(3))
    near, far, _, _ = oracle_guide(0.5 * fc, 900)
    assert far.max() / near.max() < 1e-2


def test_analysis_matches_reference_golden():
    """Cutoffs, propagation constants, mode patterns and dispersion curves of
    three guides against the reference's own waveguides.py executed by
    tests/golden/make_golden.py (bit for bit: the same FP64 operations)."""
    from pathlib import Path

    g = np.load(Path(__file__).resolve().parent / "golden" / "waveguides.npz")
    guides = [(0.02286, 0.01016), (0.02, 0.01), (0.016, 0.008)]
    modes = [("TE", 1, 0), ("TE", 2, 0), ("TE", 0, 1), ("TE", 1, 1), ("TM", 1, 1), ("TM", 2, 1)]
    for gi, (a, b) in enumerate(guides):
        wg = RectangularWaveguide(a=a, b=b)
        for mt, m, n in modes:
            key = f"g{gi}_{mt}{m}{n}"
            assert wg.cutoff_frequency(m, n) == float(g[key + "_fc"])
            beta = [wg.propagation_constant(float(f), m, n) for f in g[key + "_beta_f"]]
            np.testing.assert_array_equal(beta, g[key + "_beta"])
            mode = wg.compute_mode(mt, m, n, n_points=21)
            np.testing.assert_array_equal(mode.field_pattern, g[key + "_pattern"])
            np.testing.assert_array_equal(mode.x, g[key + "_x"])
            np.testing.assert_array_equal(mode.y, g[key + "_y"])
            np.testing.assert_array_equal(wg.dispersion_relation(m, n, g["disp_freqs"]),
                                          g[key + "_disp"])
