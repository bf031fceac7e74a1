"""The CPU oracle against golden vectors produced by the reference's own
FDTD source (tests/golden/make_golden.py).  CPU only."""

import numpy as np
import pytest

from cases import golden, load_cases, oracle2d_from_case, oracle3d_from_case, rn

CASES = load_cases()


@pytest.mark.parametrize("case", CASES["3d"], ids=lambda c: c["name"])
def test_oracle3d_matches_reference(case):
    o, n = oracle3d_from_case(case)
    out = o.run(n, save_every=case["save_every"])
    g = golden("3d", case["name"])
    assert out["t"].shape[0] == int(g["n_saved"])
    np.testing.assert_array_equal(out["t"], g["t"])
    fr = g["frames"]
    for k in ("ex", "ey", "ez", "hx", "hy", "hz"):
        # same FP64 operations in the same order: bit-identical
        np.testing.assert_array_equal(out[k][fr], g[k])
    np.testing.assert_allclose(g["grid_x"], np.arange(case["size"][0]) * case["resolution"])


@pytest.mark.parametrize("case", CASES["2d"], ids=lambda c: c["name"])
def test_oracle2d_matches_reference(case):
    o, n = oracle2d_from_case(case)
    out = o.run(n, save_every=case["save_every"])
    g = golden("2d", case["name"])
    assert out["t"].shape[0] == int(g["n_saved"])
    np.testing.assert_array_equal(out["t"], g["t"])
    fr = g["frames"]
    for k in ("ez", "hx", "hy"):
        np.testing.assert_array_equal(out[k][fr], g[k])


def test_golden_fields_nontrivial():
    """Fixtures carry signal (a zero fixture would pin nothing)."""
    for kind in ("3d", "2d"):
        for case in CASES[kind]:
            g = golden(kind, case["name"])
            assert np.abs(g["ez"][-1]).max() > 1e-3, case["name"]


def test_fp32_oracle_close_to_fp64():
    """FP32 restatement stays within the 1e-5 relative-L2 bar of FP64."""
    case = CASES["3d"][0]
    o64, n = oracle3d_from_case(case, np.float64)
    o32, _ = oracle3d_from_case(case, np.float32)
    a = o64.run(n, save_every=n)
    b = o32.run(n, save_every=n)
    for k in ("ex", "ey", "ez", "hx", "hy", "hz"):
        assert rn.rel_l2(b[k], a[k]) < 1e-5


def test_cpml_oracle_absorbs():
    """Extension semantics sanity: a CPML box keeps far less energy than a
    PEC box after the pulse has left (both FP64, same source)."""
    sz = (24, 24, 24)
    src = [dict(position=(12, 12, 12), polarization="z", amplitude=1.0, kind="gauss_sine",
                frequency=0.05 / rn.default_dt_3d(1.0), width_steps=10, delay_steps=40)]
    energies = {}
    for bnd in ("pec", "cpml"):
        spec = rn.Spec3D(size=sz, dx=1.0, boundary=bnd, pml_layers=6, sources=src)
        o = rn.Oracle3D(spec, dt=rn.default_dt_3d(1.0))
        o.run(300)
        energies[bnd] = sum(float(np.sum(f * f)) for f in o.f[:3])
    assert energies["cpml"] < 1e-3 * energies["pec"]
