"""Host-side behaviour of the drop-in API that needs no GPU: the reference's
validation cases (tests/test_fdtd3d.py:113-139, tests/test_em.py:41-48,
tests/test_edge_cases.py:1523-1547, tests/test_config.py:69-79)."""

import numpy as np
import pytest
from pydantic import ValidationError

from jaxphys_b200 import (
    ConfigurationError,
    DielectricRegion,
    EMConfig,
    EMGrid,
    EMGrid3D,
    NeurosimError,
    NumericalInstabilityError,
    PlaneWave,
    PointSource3D,
    SimulationError,
    Wall,
)


def test_small_grid_error_3d():
    with pytest.raises(ConfigurationError):
        EMGrid3D(size=(4, 4, 4))


def test_source_out_of_bounds_3d():
    grid = EMGrid3D(size=(16, 16, 16))
    with pytest.raises(ConfigurationError, match="out of grid"):
        grid.add_source(PointSource3D(frequency=1e9, position=(20, 8, 8)))
    with pytest.raises(ConfigurationError):
        grid.add_source(PointSource3D(frequency=1e9, position=(8, -1, 8)))


def test_material_shape_mismatch():
    grid = EMGrid3D(size=(16, 16, 16))
    with pytest.raises(ConfigurationError):
        grid.add_material(DielectricRegion(mask=np.zeros((10, 10, 10), dtype=bool)))


def test_no_source_error_3d():
    grid = EMGrid3D(size=(16, 16, 16))
    with pytest.raises(ConfigurationError):
        grid.simulate()


def test_size_property_and_eps():
    grid = EMGrid3D(size=(16, 12, 10))
    assert grid.size == (16, 12, 10)
    m1 = np.zeros((16, 12, 10), dtype=bool)
    m1[:8] = True
    m2 = np.zeros((16, 12, 10), dtype=bool)
    m2[4:12] = True
    grid.add_material(DielectricRegion(mask=m1, epsilon_r=2.0))
    grid.add_material(DielectricRegion(mask=m2, epsilon_r=5.0))
    eps = grid.epsilon_r()
    assert eps[0, 0, 0] == 2.0 and eps[5, 0, 0] == 5.0 and eps[13, 0, 0] == 1.0


def test_permittivity_override_validation():
    grid = EMGrid3D(size=(8, 8, 8))
    with pytest.raises(ConfigurationError):
        grid.set_permittivity(np.ones((8, 8, 7)))
    with pytest.raises(ConfigurationError):
        grid.set_permittivity(np.zeros((8, 8, 8)))
    grid.set_permittivity(np.full((8, 8, 8), 2.0))
    assert grid.epsilon_r()[0, 0, 0] == 2.0


def test_probe_validation():
    grid = EMGrid3D(size=(8, 8, 8))
    with pytest.raises(ConfigurationError):
        grid.add_probe((8, 0, 0))
    with pytest.raises(ConfigurationError):
        grid.add_probe((0, 0, 0), component="bz")
    assert grid.add_probe((1, 2, 3), "hx") == 0


def test_small_grid_error_2d():
    with pytest.raises(ConfigurationError):
        EMGrid(size=(5, 5))


def test_no_source_error_2d():
    with pytest.raises(ConfigurationError):
        EMGrid(size=(50, 50)).simulate()


def test_out_of_grid_messages_2d():
    grid = EMGrid(size=(50, 50))
    with pytest.raises(ConfigurationError, match="out of grid"):
        grid.add_source(PlaneWave(frequency=1e9, y=100))
    with pytest.raises(ConfigurationError, match="out of grid"):
        grid.add_conductor(Wall(y=100))


def test_grid_properties_2d():
    assert EMGrid(size=(100, 80)).size == (100, 80)


def test_emconfig():
    cfg = EMConfig()
    assert cfg.boundary == "absorbing"
    assert cfg.pml_layers == 10
    with pytest.raises(ValidationError):
        EMConfig(boundary="invalid")
    with pytest.raises(ValidationError):
        EMGrid(size=(20, 20), boundary="bogus")
    # tests/test_edge_cases.py:738-752 of the reference
    with pytest.raises(ValidationError):
        EMConfig(resolution=0.0)
    with pytest.raises(ValidationError):
        EMConfig(courant_number=1.5)


def test_exception_hierarchy():
    assert issubclass(ConfigurationError, NeurosimError)
    assert issubclass(NumericalInstabilityError, SimulationError)


def test_default_dt():
    g3 = EMGrid3D(size=(8, 8, 8), resolution=0.01)
    assert g3.default_dt() == pytest.approx(0.99 * 0.01 / (299792458.0 * np.sqrt(3.0)), rel=1e-15)
    g2 = EMGrid(size=(10, 10), resolution=0.01)
    assert g2.default_dt() == pytest.approx(0.99 * 0.01 / (299792458.0 * np.sqrt(2.0)), rel=1e-15)
