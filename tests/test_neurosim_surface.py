"""The reference's import surface (``neurosim``, ``neurosim.em``,
``neurosim.em.fdtd3d``, ``neurosim.em.fdtd``, ``neurosim.exceptions``) served
by the CUDA engine, and the reference's own FDTD behaviour tests
(tests/test_fdtd3d.py:16-139, tests/test_em.py:15-79) restated against those
import paths.  The reference's tests build masks with ``jnp`` and reduce with
``jnp.max``; here ``XP`` is ``jax.numpy`` when JAX is importable (then
``simulate`` returns JAX arrays, as the reference does) and NumPy otherwise,
and results are reduced with operations that torch tensors and JAX arrays
share."""

import numpy as np
import pytest

try:
    import jax.numpy as XP

    HAVE_JAX = True
except Exception:  # JAX is optional
    XP = np
    HAVE_JAX = False


def _np(a):
    if hasattr(a, "detach"):
        return a.detach().cpu().numpy()
    return np.asarray(a)


def _amax(a) -> float:
    return float(abs(a).max())


def _mask(shape, from_x):
    m = np.zeros(shape, dtype=bool)
    m[from_x:] = True
    return XP.asarray(m)


# ------------------------------------------------------------------ CPU

def test_import_paths_resolve_to_the_engine():
    import neurosim
    import neurosim.em
    import neurosim.em.fdtd
    import neurosim.em.fdtd3d
    import neurosim.exceptions
    import neurosim.state
    import jaxphys_b200

    assert neurosim.EMGrid3D is neurosim.em.EMGrid3D is neurosim.em.fdtd3d.EMGrid3D
    assert neurosim.EMGrid is neurosim.em.EMGrid is neurosim.em.fdtd.EMGrid
    assert issubclass(neurosim.EMGrid3D, jaxphys_b200.EMGrid3D)
    assert issubclass(neurosim.EMGrid, jaxphys_b200.EMGrid)
    for name in ("PointSource3D", "DielectricRegion"):
        assert getattr(neurosim.em.fdtd3d, name) is getattr(jaxphys_b200, name)
    for name in ("PlaneWave", "Wall"):
        assert getattr(neurosim.em.fdtd, name) is getattr(jaxphys_b200, name)
    assert neurosim.exceptions.ConfigurationError is jaxphys_b200.ConfigurationError
    assert neurosim.state.EMFieldHistory3D is jaxphys_b200.EMFieldHistory3D
    assert issubclass(neurosim.ConfigurationError, neurosim.NeurosimError)
    for name in ("EMGrid", "PlaneWave", "Wall", "EMGrid3D", "PointSource3D",
                 "DielectricRegion", "RectangularWaveguide"):
        assert name in neurosim.em.__all__ and hasattr(neurosim, name)


def test_simulate_defaults_to_reference_result_type():
    import inspect

    from neurosim.em.fdtd import EMGrid
    from neurosim.em.fdtd3d import EMGrid3D

    assert inspect.signature(EMGrid3D.simulate).parameters["output"].default == "auto"
    assert inspect.signature(EMGrid.simulate).parameters["output"].default == "auto"
    from jaxphys_b200.state import resolve_output

    assert resolve_output("auto") == ("jax" if HAVE_JAX else "torch")


def test_output_jax_without_jax_is_a_configuration_error():
    if HAVE_JAX:
        pytest.skip("JAX is importable here")
    from neurosim.em.fdtd3d import EMGrid3D, PointSource3D
    from neurosim.exceptions import ConfigurationError

    g = EMGrid3D(size=(16, 16, 16))
    g.add_source(PointSource3D(frequency=1e9, position=(8, 8, 8)))
    with pytest.raises(ConfigurationError):
        g.simulate(output="jax")


# test_fdtd3d.py:117-133 and test_em.py:42-50 (errors raised before any device work)
def test_3d_no_source_error():
    from neurosim.em.fdtd3d import EMGrid3D
    from neurosim.exceptions import ConfigurationError

    grid = EMGrid3D(size=(16, 16, 16))
    with pytest.raises(ConfigurationError):
        grid.simulate()


def test_3d_small_grid_error():
    from neurosim.em.fdtd3d import EMGrid3D
    from neurosim.exceptions import ConfigurationError

    with pytest.raises(ConfigurationError):
        EMGrid3D(size=(4, 4, 4))


def test_3d_source_out_of_bounds():
    from neurosim.em.fdtd3d import EMGrid3D, PointSource3D
    from neurosim.exceptions import ConfigurationError

    grid = EMGrid3D(size=(16, 16, 16))
    with pytest.raises(ConfigurationError):
        grid.add_source(PointSource3D(frequency=1e9, position=(20, 8, 8)))


def test_3d_material_shape_mismatch():
    from neurosim.em.fdtd3d import DielectricRegion, EMGrid3D
    from neurosim.exceptions import ConfigurationError

    grid = EMGrid3D(size=(16, 16, 16))
    with pytest.raises(ConfigurationError):
        grid.add_material(DielectricRegion(mask=XP.zeros((10, 10, 10), dtype=bool)))


def test_2d_no_source_error():
    from neurosim.em.fdtd import EMGrid
    from neurosim.exceptions import ConfigurationError

    with pytest.raises(ConfigurationError):
        EMGrid(size=(50, 50)).simulate()


def test_2d_small_grid_error():
    from neurosim.em.fdtd import EMGrid
    from neurosim.exceptions import ConfigurationError

    with pytest.raises(ConfigurationError):
        EMGrid(size=(5, 5))


# ------------------------------------------------------------------ GPU
# test_fdtd3d.py:16-115,135-139

@pytest.mark.gpu
def test_3d_basic_simulation(cuda):
    from neurosim.em.fdtd3d import EMGrid3D, PointSource3D

    grid = EMGrid3D(size=(20, 20, 20), resolution=0.01)
    grid.add_source(PointSource3D(frequency=3e9, position=(10, 10, 10)))
    fields = grid.simulate(t_span=(0, 5e-10), save_every=10)
    assert fields.ez.shape[1] == 20 and fields.ez.shape[2] == 20 and fields.ez.shape[3] == 20
    assert fields.t.shape[0] > 0
    if HAVE_JAX:
        import jax

        assert isinstance(fields.ez, jax.Array)


@pytest.mark.gpu
def test_3d_source_excites_field(cuda):
    from neurosim.em.fdtd3d import EMGrid3D, PointSource3D

    grid = EMGrid3D(size=(20, 20, 20), resolution=0.01)
    grid.add_source(PointSource3D(frequency=3e9, position=(10, 10, 10), amplitude=1.0))
    fields = grid.simulate(t_span=(0, 3e-10), save_every=5)
    assert _amax(fields.ez[-1]) > 0.0


@pytest.mark.gpu
def test_3d_all_six_components(cuda):
    from neurosim.em.fdtd3d import EMGrid3D, PointSource3D

    grid = EMGrid3D(size=(16, 16, 16), resolution=0.01)
    grid.add_source(PointSource3D(frequency=5e9, position=(8, 8, 8)))
    fields = grid.simulate(t_span=(0, 2e-10), save_every=5)
    assert fields.ex.shape == fields.ey.shape == fields.ez.shape
    assert fields.hx.shape == fields.hy.shape == fields.hz.shape
    assert tuple(fields.ex.shape[1:]) == (16, 16, 16)


@pytest.mark.gpu
@pytest.mark.parametrize("pol", ["x", "y"])
def test_3d_polarization(cuda, pol):
    from neurosim.em.fdtd3d import EMGrid3D, PointSource3D

    grid = EMGrid3D(size=(16, 16, 16), resolution=0.01)
    grid.add_source(PointSource3D(frequency=3e9, position=(8, 8, 8), polarization=pol))
    fields = grid.simulate(t_span=(0, 2e-10), save_every=5)
    assert _amax(getattr(fields, "e" + pol)[-1]) > 0.0


@pytest.mark.gpu
def test_3d_dielectric_material(cuda):
    from neurosim.em.fdtd3d import DielectricRegion, EMGrid3D, PointSource3D

    grid_free = EMGrid3D(size=(16, 16, 16), resolution=0.01)
    grid_free.add_source(PointSource3D(frequency=5e9, position=(8, 8, 8)))
    grid_diel = EMGrid3D(size=(16, 16, 16), resolution=0.01)
    grid_diel.add_source(PointSource3D(frequency=5e9, position=(8, 8, 8)))
    grid_diel.add_material(DielectricRegion(mask=_mask((16, 16, 16), 10), epsilon_r=4.0))
    a = grid_free.simulate(t_span=(0, 1e-9), save_every=20)
    b = grid_diel.simulate(t_span=(0, 1e-9), save_every=20)
    assert not np.allclose(_np(a.ez[-1]), _np(b.ez[-1]))


@pytest.mark.gpu
def test_3d_periodic_boundary(cuda):
    from neurosim.em.fdtd3d import EMGrid3D, PointSource3D

    ga = EMGrid3D(size=(16, 16, 16), resolution=0.01, boundary="absorbing")
    gp = EMGrid3D(size=(16, 16, 16), resolution=0.01, boundary="periodic", pml_layers=0)
    source = PointSource3D(frequency=5e9, position=(8, 8, 8))
    ga.add_source(source)
    gp.add_source(source)
    a = ga.simulate(t_span=(0, 2e-10), save_every=5)
    p = gp.simulate(t_span=(0, 2e-10), save_every=5)
    assert not np.allclose(_np(a.ez[-1]), _np(p.ez[-1]))


@pytest.mark.gpu
def test_3d_grid_coordinates(cuda):
    from neurosim.em.fdtd3d import EMGrid3D, PointSource3D

    grid = EMGrid3D(size=(16, 16, 16), resolution=0.02)
    grid.add_source(PointSource3D(frequency=1e9, position=(8, 8, 8)))
    fields = grid.simulate(t_span=(0, 1e-10), save_every=5)
    assert tuple(fields.grid_x.shape) == (16,)
    assert float(fields.grid_x[1] - fields.grid_x[0]) == pytest.approx(0.02)


# test_em.py:18-40,52-79

@pytest.mark.gpu
def test_2d_basic_simulation(cuda):
    from neurosim.em.fdtd import EMGrid, PlaneWave

    grid = EMGrid(size=(50, 50), resolution=0.01)
    grid.add_source(PlaneWave(frequency=3e9, y=10))
    fields = grid.simulate(t_span=(0, 1e-9), save_every=10)
    assert fields.ez.shape[1] == 50 and fields.ez.shape[2] == 50
    assert fields.t.shape[0] > 0


@pytest.mark.gpu
def test_2d_with_conductor(cuda):
    from neurosim.em.fdtd import EMGrid, PlaneWave, Wall

    grid = EMGrid(size=(50, 50), resolution=0.01)
    grid.add_source(PlaneWave(frequency=3e9, y=10))
    grid.add_conductor(Wall(y=25, gap_start=20, gap_end=30))
    fields = grid.simulate(t_span=(0, 5e-10), save_every=5)
    assert fields.ez.shape[0] > 0


@pytest.mark.gpu
def test_2d_multiple_sources_are_applied(cuda):
    from neurosim.em.fdtd import EMGrid, PlaneWave

    grid = EMGrid(size=(50, 50), resolution=0.01)
    grid.add_source(PlaneWave(frequency=3e9, y=10, amplitude=1.0))
    grid.add_source(PlaneWave(frequency=5e9, y=35, amplitude=0.5))
    fields = grid.simulate(t_span=(0, 2e-10), save_every=1)
    assert _amax(fields.ez[-1, :, 10]) > 0.0
    assert _amax(fields.ez[-1, :, 35]) > 0.0


@pytest.mark.gpu
def test_2d_boundary_modes_affect_solution(cuda):
    from neurosim.em.fdtd import EMGrid, PlaneWave

    periodic = EMGrid(size=(40, 40), resolution=0.01, boundary="periodic", pml_layers=0)
    reflecting = EMGrid(size=(40, 40), resolution=0.01, boundary="reflecting", pml_layers=0)
    source = PlaneWave(frequency=3e9, y=2, amplitude=1.0)
    periodic.add_source(source)
    reflecting.add_source(source)
    a = periodic.simulate(t_span=(0, 2e-10), save_every=1)
    b = reflecting.simulate(t_span=(0, 2e-10), save_every=1)
    assert not np.allclose(_np(a.ez[-1]), _np(b.ez[-1]))


@pytest.mark.gpu
def test_numpy_and_torch_outputs_agree(cuda):
    """output='numpy' equals output='torch' (and 'jax' when JAX is importable)
    for the same 3D run."""
    from neurosim.em.fdtd3d import EMGrid3D, PointSource3D

    def run(out):
        g = EMGrid3D(size=(16, 16, 16), resolution=0.01)
        g.add_source(PointSource3D(frequency=5e9, position=(8, 8, 8)))
        return g.simulate(t_span=(0, 2e-10), save_every=5, output=out)

    t = run("torch")
    n = run("numpy")
    assert isinstance(n.ez, np.ndarray)
    np.testing.assert_array_equal(_np(t.ez), n.ez)
    if HAVE_JAX:
        j = run("jax")
        np.testing.assert_array_equal(np.asarray(j.ez), n.ez)
