"""Field viewers on the CPU: colour tables, argument errors, and the
reference's behaviour without matplotlib (viz/fields.py:17-29)."""

import numpy as np
import pytest

from jaxphys_b200 import EMFieldHistory, EMFieldHistory3D, VisualizationError
from jaxphys_b200.viz import colour_table, fields as vf


def _hist2d(s=3, nx=12, ny=9):
    rng = np.random.default_rng(0)
    f = lambda: rng.normal(size=(s, nx, ny)).astype(np.float32)
    return EMFieldHistory(t=np.arange(s) * 1e-9, ez=f(), hx=f(), hy=f(),
                          grid_x=np.arange(nx) * 0.01, grid_y=np.arange(ny) * 0.01)


def test_colour_tables():
    rdbu_r = colour_table("RdBu_r")
    assert rdbu_r.shape == (256, 3) and rdbu_r.dtype == np.uint8
    # negative values blue, positive red, white-ish in the middle
    assert tuple(rdbu_r[0]) == (0x05, 0x30, 0x61) and tuple(rdbu_r[255]) == (0x67, 0x00, 0x1F)
    assert np.all(rdbu_r[127:129] > 240)
    np.testing.assert_array_equal(colour_table("RdBu"), rdbu_r[::-1])
    g = colour_table("gray")
    assert np.all(g[:, 0] == g[:, 1]) and np.all(np.diff(g[:, 0].astype(int)) >= 0)
    assert tuple(colour_table("seismic")[255]) == (0x80, 0, 0)
    with pytest.raises(VisualizationError, match="colour map"):
        colour_table("jet")


def test_unknown_component():
    with pytest.raises(VisualizationError, match="Unknown component"):
        vf._component(_hist2d(), "Ex")
    h3 = EMFieldHistory3D(t=np.zeros(1), **{k: np.zeros((1, 8, 8, 8), np.float32)
                                             for k in ("ex", "ey", "ez", "hx", "hy", "hz")},
                          grid_x=None, grid_y=None, grid_z=None)
    assert vf._component(h3, "Hz").shape == (1, 8, 8, 8)


@pytest.mark.skipif(vf.HAS_MATPLOTLIB, reason="matplotlib is installed")
def test_matplotlib_viewers_raise_without_matplotlib():
    with pytest.raises(VisualizationError, match="matplotlib required"):
        vf.plot_field_snapshot(_hist2d())
    with pytest.raises(VisualizationError, match="matplotlib required"):
        vf.animate_field(_hist2d(), save=None)
