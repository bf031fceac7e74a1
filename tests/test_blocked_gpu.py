"""Two-level temporally blocked kernel (fdtd3d_tb.cuh) against the generic
kernel: bit for bit (same operations in the same order; np.array_equal, so
only the sign of an exact zero may differ), fields and probe traces, for
every blocked launch shape, 1-, 3- and 64-plane chunks (chunk seams inside
the two-plane warm-up), ragged tiles, sources on tile and chunk seams and on
the grid faces, duplicate sources on one cell, probes of all six components,
odd step counts (pairs of steps in blocked passes, the last step alone), and
every boundary mode of the TMA path."""

import numpy as np
import pytest

from cases import rn
from gpu_helpers import smooth_eps, to_np

pytestmark = pytest.mark.gpu

COMPS = ("ex", "ey", "ez", "hx", "hy", "hz")
N_TB_CONFIGS = 6


def _gauss(pos, pol="z", amp=1.0, width=10.0):
    dt = rn.default_dt_3d(1.0)
    return dict(frequency=0.05 / dt, position=pos, amplitude=amp, polarization=pol,
                waveform="gauss_sine", width_steps=width)


def _grid(path, size, boundary, eps, sources, probes, n_pml=4, cpml=None):
    from jaxphys_b200 import CPMLSpec, EMGrid3D, PointSource3D

    g = EMGrid3D(size=size, resolution=1.0, boundary=boundary, pml_layers=n_pml, path=path,
                 cpml=cpml or CPMLSpec())
    for s in sources:
        g.add_source(PointSource3D(**s))
    if eps is not None:
        g.set_permittivity(eps)
    for p in probes:
        g.add_probe(p[:3], COMPS[p[3]])
    g.prepare(dt=rn.default_dt_3d(1.0))
    return g


def _run_pair(size, boundary, eps, sources, probes, steps, blocked, n_pml=4, cpml=None,
              split=None, ref_path="generic"):
    """(fields, traces) of the blocked TMA run and of the reference path."""
    from jaxphys_b200 import _native as nat

    lib = nat.load()
    out = []
    for path in ("tma", ref_path):
        g = _grid("tma" if path == "tma" else ref_path, size, boundary, eps, sources, probes,
                  n_pml, cpml)
        if path == "tma":
            cfg, chunk = blocked
            nat.check(lib.jxf_grid3d_set_blocked(g._h, cfg, chunk), "set_blocked")
            if split is not None:
                nat.check(lib.jxf_grid3d_set_axis_split(g._h, split), "set_axis_split")
        elif ref_path == "tma":
            nat.check(lib.jxf_grid3d_set_blocked(g._h, -1, 0), "set_blocked")
        tr = to_np(g.run(steps))
        g.check()
        if path == "tma":
            info = g.info()
            assert info["blocked_config"] == blocked[0]
        out.append(({k: to_np(g.field(k)) for k in COMPS}, tr))
    return out


def _assert_equal(out):
    for k in COMPS:
        assert np.array_equal(out[0][0][k], out[1][0][k]), k
    assert np.array_equal(out[0][1], out[1][1]), "probe traces"
    assert max(np.abs(out[1][0][k]).max() for k in COMPS) > 0


def test_blocked_registry_size(cuda):
    from jaxphys_b200 import _native as nat

    assert nat.load().jxf_num_blocked_configs() == N_TB_CONFIGS


SOURCES = [_gauss((3, 18, 22)), _gauss((6, 0, 43), "x"), _gauss((18, 36, 0), "y"),
           _gauss((9, 15, 31), "z", 0.5), _gauss((9, 15, 31), "z", 0.25),
           _gauss((2, 28, 27), "y", 0.7), _gauss((4, 29, 28), "x", -0.4),
           _gauss((1, 13, 26), "z", 0.3)]
PROBES = [(3, 18, 22, 2), (18, 36, 43, 0), (2, 28, 27, 1), (4, 29, 28, 3), (8, 12, 30, 4),
          (0, 0, 0, 5), (17, 1, 2, 2), (9, 15, 31, 2), (3, 26, 29, 5)]


@pytest.mark.parametrize("cfg", range(N_TB_CONFIGS))
@pytest.mark.parametrize("chunk", [1, 3, 64])
@pytest.mark.parametrize("split", [0, 1])
def test_blocked_cpml_every_shape_bitwise(cuda, cfg, chunk, split):
    size = (19, 37, 44)  # ragged against every tile
    eps = smooth_eps(size, 1.0, 3.0, seed=cfg)
    out = _run_pair(size, "cpml", eps, SOURCES, PROBES, 61, (cfg, chunk), split=split)
    _assert_equal(out)


@pytest.mark.parametrize("cfg", range(N_TB_CONFIGS))
@pytest.mark.parametrize("boundary", ["absorbing", "pec"])
@pytest.mark.parametrize("vacuum", [False, True])
def test_blocked_absorbing_pec_bitwise(cuda, cfg, boundary, vacuum):
    size = (21, 33, 40)
    eps = None if vacuum else smooth_eps(size, 1.0, 4.0, seed=7 + cfg)
    src = [_gauss((10, 16, 20)), _gauss((0, 32, 39), "x"), _gauss((20, 0, 1), "y", 0.5)]
    probes = [(10, 16, 24, 2), (0, 32, 39, 0), (5, 5, 5, 3), (20, 30, 38, 4)]
    out = _run_pair(size, boundary, eps, src, probes, 47, (cfg, 4), n_pml=5)
    _assert_equal(out)


@pytest.mark.parametrize("cfg", range(N_TB_CONFIGS))
def test_blocked_cpml_kappa_cfs_bitwise(cuda, cfg):
    from jaxphys_b200 import CPMLSpec

    size = (24, 30, 32)
    eps = smooth_eps(size, 1.0, 4.0, seed=5)
    cp = CPMLSpec(order=3.0, r0=1e-6, kappa_max=4.0, alpha_max=0.05)
    src = [_gauss((12, 15, 16)), _gauss((3, 3, 3), "y")]
    probes = [(12, 15, 20, 2), (1, 2, 3, 1)]
    out = _run_pair(size, "cpml", eps, src, probes, 80, (cfg, 8), n_pml=8, cpml=cp)
    _assert_equal(out)


def test_blocked_128_cpml_matches_one_step_tma(cuda):
    """A 128^3 CPML grid (10 layers, eps sphere, 16 probes): blocked passes
    equal one-step TMA passes bit for bit over 40 steps."""
    n = 128
    ix, iy, iz = np.ogrid[:n, :n, :n]
    eps = np.where((ix - 70) ** 2 + (iy - 60) ** 2 + (iz - 66) ** 2 <= 400, 4.0, 1.0)
    rng = np.random.default_rng(2)
    probes = [tuple(int(v) for v in rng.integers(16, 112, size=3)) + (2,) for _ in range(16)]
    out = _run_pair((n, n, n), "cpml", eps, [_gauss((64, 64, 64), width=30.0)], probes, 40,
                    (0, 16), n_pml=10, ref_path="tma")
    _assert_equal(out)


def test_blocked_set_blocked_errors(cuda):
    from jaxphys_b200 import EMGrid3D, PointSource3D
    from jaxphys_b200 import _native as nat

    lib = nat.load()
    g = EMGrid3D(size=(16, 16, 16), path="generic")
    g.add_source(PointSource3D(frequency=5e9, position=(8, 8, 8)))
    g.prepare()
    assert lib.jxf_grid3d_set_blocked(g._h, 0, 8) == nat.ERR_INVALID
    t = EMGrid3D(size=(16, 16, 16), path="tma")
    t.add_source(PointSource3D(frequency=5e9, position=(8, 8, 8)))
    t.prepare()
    assert lib.jxf_grid3d_set_blocked(t._h, N_TB_CONFIGS, 8) == nat.ERR_INVALID
    assert lib.jxf_grid3d_set_blocked(t._h, 0, 0) == nat.ERR_INVALID
    nat.check(lib.jxf_grid3d_set_blocked(t._h, -1, 0), "off")
