"""Field viewers on the GPU: the colour-mapped images against a NumPy
restatement of the same mapping (byte for byte), plane selection in 3D
histories, and the PNG / GIF writers."""

import numpy as np
import pytest

from gpu_helpers import to_np

pytestmark = pytest.mark.gpu


def _rgb_ref(plane, lut, vmax=None):
    """NumPy restatement of the image: imshow(data.T, origin="lower") with
    limits +-vmax, index floor((v/vmax + 1)/2 * 256) clamped, FP32 steps."""
    p = np.asarray(plane, np.float32)
    vm = np.float32(np.abs(p).max() if vmax is None else vmax)
    if not vm > 0:
        vm = np.float32(1.0)
    t = ((p / vm + np.float32(1.0)) * np.float32(0.5)) * np.float32(256.0)
    k = np.clip(np.floor(t), 0, 255).astype(np.int64)
    img = lut[k]                        # (U, V, 3)
    return img.transpose(1, 0, 2)[::-1]  # rows = V from the top, columns = U


def _hist3d():
    from jaxphys_b200 import EMGrid3D, PointSource3D

    g = EMGrid3D((24, 20, 16), resolution=0.01, boundary="cpml", pml_layers=4)
    g.add_source(PointSource3D(frequency=3e9, position=(12, 10, 8), polarization="y"))
    return g.simulate(t_span=(0.0, 60 * g.default_dt()), save_every=20)


def test_snapshot_matches_numpy_mapping(cuda):
    from jaxphys_b200.viz import colour_table, render_snapshot

    h = _hist3d()
    ey = to_np(h.ey)
    for axis, index, plane in (("z", None, ey[-1][:, :, 8]), ("x", 5, ey[-1][5]),
                               ("y", 3, ey[-1][:, 3, :])):
        img = to_np(render_snapshot(h, component="Ey", axis=axis, index=index))
        np.testing.assert_array_equal(img, _rgb_ref(plane, colour_table("RdBu_r")))
    img = to_np(render_snapshot(h, step=1, component="Hz", cmap="seismic", vmax=0.001))
    np.testing.assert_array_equal(img, _rgb_ref(to_np(h.hz)[1][:, :, 8], colour_table("seismic"),
                                                vmax=0.001))


def test_frames_share_one_limit_and_zero_frames(cuda):
    from jaxphys_b200.viz import colour_table, render_frames

    h = _hist3d()
    frames = to_np(render_frames(h, component="Ey", axis="z"))
    data = to_np(h.ey)[:, :, :, 8]
    vmax = np.abs(data).max()
    assert frames.shape == (data.shape[0], 20, 24, 3)
    for f in range(data.shape[0]):
        np.testing.assert_array_equal(frames[f], _rgb_ref(data[f], colour_table("RdBu_r"), vmax))
    # an all-zero plane (Ex on the y = 0 face, never updated) maps to the
    # middle colour (limit 1, reference behaviour)
    assert np.all(to_np(h.ex)[:, :, 0, :] == 0)
    z = to_np(render_frames(h, component="Ex", axis="y", index=0))
    assert np.all(z == colour_table("RdBu_r")[128])


def test_host_history_and_2d(cuda):
    from jaxphys_b200 import EMGrid, PlaneWave
    from jaxphys_b200.viz import colour_table, render_snapshot

    g = EMGrid(size=(40, 30), resolution=0.01)
    g.add_source(PlaneWave(frequency=3e9, y=10))
    h = g.simulate(t_span=(0, 2e-10), save_every=5)
    img = to_np(render_snapshot(h, component="Ez"))
    np.testing.assert_array_equal(img, _rgb_ref(to_np(h.ez)[-1], colour_table("RdBu_r")))
    hn = type(h)(**{k: to_np(getattr(h, k)) for k in ("t", "ez", "hx", "hy", "grid_x",
                                                     "grid_y")})
    np.testing.assert_array_equal(to_np(render_snapshot(hn, component="Ez")), img)


def test_png_and_gif_writers(cuda, tmp_path):
    from PIL import Image

    from jaxphys_b200.viz import render_frames, render_snapshot, save_animation, save_snapshot

    h = _hist3d()
    p = save_snapshot(tmp_path / "ey.png", h, component="Ey", scale=2)
    img = np.asarray(Image.open(p).convert("RGB"))
    want = to_np(render_snapshot(h, component="Ey"))
    np.testing.assert_array_equal(img[::2, ::2], want)
    assert img.shape == (40, 48, 3)
    g = save_animation(tmp_path / "ey.gif", h, component="Ey", fps=10)
    with Image.open(g) as im:
        assert im.n_frames == to_np(render_frames(h, component="Ey")).shape[0]
