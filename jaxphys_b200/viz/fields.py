"""Field viewers (reference: ``src/neurosim/viz/fields.py``).

* ``plot_field_snapshot`` and ``animate_field`` keep the reference's
  matplotlib viewers and arguments (``fields.py:32-167``); as there, they
  raise ``VisualizationError`` when matplotlib is not installed
  (``fields.py:17-29``).
* ``render_snapshot`` / ``render_frames`` build the same picture -- the
  component's values over a plane, mapped through a diverging colour table
  with limits +-max|value| (one frame, or all frames of the history for an
  animation) and shown as ``imshow(data.T, origin="lower")`` -- as RGB bytes
  computed on the GPU from the history's device tensors
  (``csrc/viz_kernels.cuh``).  Only 3 bytes per pixel reach the host.
* ``save_snapshot`` (PNG) and ``save_animation`` (GIF) write those images
  with Pillow; they need no matplotlib.

Histories: ``EMFieldHistory`` (2D: components "Ez", "Hx", "Hy", as the
reference) and ``EMFieldHistory3D`` ("Ex" ... "Hz"; a plane normal to
``axis`` at ``index``, default the middle: axis "z" shows (x, y), "x" shows
(y, z), "y" shows (x, z)).  Tensors may live on the GPU (default), in host
memory (``history="host"``) or be NumPy arrays; host data is copied to the
device once per call.
"""

from __future__ import annotations

from pathlib import Path
from typing import Any

import numpy as np

from .. import _native as nat
from ..exceptions import VisualizationError

try:  # optional, as in the reference
    import matplotlib.pyplot as plt
    from matplotlib import animation

    HAS_MATPLOTLIB = True
except ImportError:
    HAS_MATPLOTLIB = False

# Colour tables: anchor colours spaced evenly over [0, 1], linearly
# interpolated to 256 entries.  RdBu is ColorBrewer's 11-class diverging
# scheme (red for low values); "_r" reverses it.
_ANCHORS = {
    "RdBu": ["#67001f", "#b2182b", "#d6604d", "#f4a582", "#fddbc7", "#f7f7f7", "#d1e5f0",
             "#92c5de", "#4393c3", "#2166ac", "#053061"],
    "seismic": ["#00004c", "#0000ff", "#ffffff", "#ff0000", "#800000"],
    "gray": ["#000000", "#ffffff"],
}
_LUT_CACHE: dict = {}


def _check_matplotlib() -> None:
    if not HAS_MATPLOTLIB:
        raise VisualizationError("matplotlib required. Install with: pip install neurosim[viz]")


def colour_table(cmap: str) -> np.ndarray:
    """256 x 3 uint8 table of a colour map name ("RdBu_r", "RdBu", "seismic",
    "seismic_r", "gray", "gray_r")."""
    base, rev = (cmap[:-2], True) if cmap.endswith("_r") else (cmap, False)
    if base not in _ANCHORS:
        raise VisualizationError(
            f"Unknown colour map '{cmap}'. Available: "
            f"{sorted(list(_ANCHORS) + [k + '_r' for k in _ANCHORS])}")
    hexes = _ANCHORS[base][::-1] if rev else _ANCHORS[base]
    rgb = np.array([[int(h[i:i + 2], 16) for i in (1, 3, 5)] for h in hexes], dtype=np.float64)
    pos = np.linspace(0.0, 1.0, len(rgb))
    x = np.linspace(0.0, 1.0, 256)
    lut = np.stack([np.interp(x, pos, rgb[:, c]) for c in range(3)], axis=1)
    return np.clip(np.rint(lut), 0, 255).astype(np.uint8)


def _device_lut(cmap: str, device):
    import torch

    key = (cmap, str(device))
    if key not in _LUT_CACHE:
        _LUT_CACHE[key] = torch.from_numpy(colour_table(cmap)).to(device)
    return _LUT_CACHE[key]


def _component(fields, component: str):
    if hasattr(fields, "hz"):
        names = {"Ex": fields.ex, "Ey": fields.ey, "Ez": fields.ez, "Hx": fields.hx,
                 "Hy": fields.hy, "Hz": fields.hz}
    else:
        names = {"Ez": fields.ez, "Hx": fields.hx, "Hy": fields.hy}
    if component not in names:
        raise VisualizationError(f"Unknown component '{component}'. Available: {list(names)}")
    return names[component]


def _plane(fields, component: str, axis: str, index: int | None):
    """(S, U, V) view of the component's frames over the displayed plane, on
    the GPU, and the plane's axis names."""
    import torch

    data = _component(fields, component)
    if not isinstance(data, torch.Tensor):
        data = torch.from_numpy(np.ascontiguousarray(data))
    if data.dtype != torch.float32:
        data = data.to(torch.float32)
    if data.dim() == 3:  # 2D history: (S, nx, ny)
        view, names = data, ("x", "y")
    elif data.dim() == 4:
        if axis not in ("x", "y", "z"):
            raise VisualizationError(f"axis must be x, y or z, got {axis!r}")
        w = "xyz".index(axis)
        n = data.shape[1 + w]
        k = n // 2 if index is None else int(index)
        if not 0 <= k < n:
            raise VisualizationError(f"plane index {k} out of range for axis {axis} ({n} cells)")
        view = data.select(1 + w, k)
        names = tuple(a for a in "xyz" if a != axis)
    else:
        raise VisualizationError(f"expected (frames, nx, ny[, nz]) data, got shape "
                                 f"{tuple(data.shape)}")
    if view.shape[0] == 0:
        raise VisualizationError("the history holds no frames")
    if not view.is_cuda:
        view = view.contiguous().to("cuda")
    return view, names


def _rgb(view, cmap: str, vmax: float | None):
    """RGB bytes (S, V, U, 3) of the frames of ``view`` (S, U, V) on the GPU."""
    import torch

    lib = nat.load()
    lut = _device_lut(cmap, view.device)
    s, nu, nv = view.shape
    sf, su, sv = view.stride()
    st = nat.stream_handle()
    vmax_dev = None
    if vmax is None:
        vmax_dev = torch.empty(1, dtype=torch.float32, device=view.device)
        nat.check(lib.jxf_slice_absmax(view.data_ptr(), nu, nv, su, sv, s, sf,
                                       vmax_dev.data_ptr(), st), "slice_absmax")
    out = torch.empty((s, nv, nu, 3), dtype=torch.uint8, device=view.device)
    nat.check(lib.jxf_slice_rgb(view.data_ptr(), nu, nv, su, sv, s, sf,
                                None if vmax_dev is None else vmax_dev.data_ptr(),
                                float(vmax or 0.0), lut.data_ptr(), out.data_ptr(), st),
              "slice_rgb")
    return out


def render_snapshot(fields, step: int = -1, component: str = "Ez", cmap: str = "RdBu_r",
                    axis: str = "z", index: int | None = None, vmax: float | None = None):
    """RGB image (height, width, 3) uint8 on the GPU of one saved frame;
    colour limits +-max|value| of that frame unless ``vmax`` is given."""
    view, _ = _plane(fields, component, axis, index)
    n = view.shape[0]
    k = step + n if step < 0 else step
    if not 0 <= k < n:
        raise VisualizationError(f"step {step} out of range ({n} frames)")
    return _rgb(view[k:k + 1], cmap, vmax)[0]


def render_frames(fields, component: str = "Ez", cmap: str = "RdBu_r", axis: str = "z",
                  index: int | None = None, vmax: float | None = None):
    """RGB images (frames, height, width, 3) uint8 on the GPU of every saved
    frame, with one colour limit +-max|value| over all of them (as the
    reference's animation) unless ``vmax`` is given."""
    view, _ = _plane(fields, component, axis, index)
    return _rgb(view, cmap, vmax)


def _image(rgb, scale: int):
    from PIL import Image

    img = Image.fromarray(np.ascontiguousarray(rgb.cpu().numpy()))
    if scale > 1:
        img = img.resize((img.width * scale, img.height * scale), Image.NEAREST)
    return img


def save_snapshot(path, fields, step: int = -1, component: str = "Ez", cmap: str = "RdBu_r",
                  axis: str = "z", index: int | None = None, scale: int = 1) -> Path:
    """Write ``render_snapshot`` as a PNG (``scale``: integer pixel size)."""
    path = Path(path)
    _image(render_snapshot(fields, step, component, cmap, axis, index), scale).save(path)
    return path


def save_animation(path, fields, component: str = "Ez", fps: int = 30, cmap: str = "RdBu_r",
                   axis: str = "z", index: int | None = None, scale: int = 1) -> Path:
    """Write every frame as an animated GIF at ``fps`` frames per second."""
    path = Path(path)
    frames = render_frames(fields, component, cmap, axis, index).cpu()
    imgs = [_image(f, scale) for f in frames]
    imgs[0].save(path, save_all=True, append_images=imgs[1:], duration=max(1, round(1000 / fps)),
                 loop=0)
    return path


def _host_plane(fields, component: str):
    data = _component(fields, component)
    return data.detach().cpu().numpy() if hasattr(data, "detach") else np.asarray(data)


def plot_field_snapshot(fields, step: int = -1, component: str = "Ez",
                        figsize: tuple[float, float] = (8, 6), cmap: str = "RdBu_r") -> Any:
    """Plot a snapshot of a field component (``fields.py:32-91``): matplotlib
    Figure; ``VisualizationError`` without matplotlib."""
    _check_matplotlib()
    data = _host_plane(fields, component)[step]
    vmax = float(np.max(np.abs(data))) or 1.0
    gx, gy = np.asarray(fields.grid_x), np.asarray(fields.grid_y)
    fig, ax = plt.subplots(figsize=figsize)
    im = ax.imshow(data.T, origin="lower", cmap=cmap, vmin=-vmax, vmax=vmax,
                   extent=(float(gx[0]), float(gx[-1]), float(gy[0]), float(gy[-1])))
    ax.set_xlabel("x (m)", fontsize=12)
    ax.set_ylabel("y (m)", fontsize=12)
    ax.set_title(f"{component} at t = {float(np.asarray(fields.t)[step]):.2e} s", fontsize=13)
    fig.colorbar(im, ax=ax, label=f"{component} (a.u.)")
    fig.tight_layout()
    return fig


def animate_field(fields, component: str = "Ez", save: str | None = None, fps: int = 30,
                  figsize: tuple[float, float] = (8, 6), cmap: str = "RdBu_r") -> Any:
    """Animate a field component (``fields.py:94-167``): matplotlib
    FuncAnimation; ``VisualizationError`` without matplotlib."""
    _check_matplotlib()
    data = _host_plane(fields, component)
    t = np.asarray(fields.t)
    vmax = float(np.max(np.abs(data))) or 1.0
    gx, gy = np.asarray(fields.grid_x), np.asarray(fields.grid_y)
    fig, ax = plt.subplots(figsize=figsize)
    im = ax.imshow(data[0].T, origin="lower", cmap=cmap, vmin=-vmax, vmax=vmax,
                   extent=(float(gx[0]), float(gx[-1]), float(gy[0]), float(gy[-1])))
    ax.set_xlabel("x (m)")
    ax.set_ylabel("y (m)")
    title = ax.set_title(f"{component} at t = 0")
    fig.colorbar(im, ax=ax)

    def update(frame: int) -> list[Any]:
        im.set_data(data[frame].T)
        title.set_text(f"{component} at t = {float(t[frame]):.2e} s")
        return [im, title]

    anim = animation.FuncAnimation(fig, update, frames=data.shape[0], interval=1000 / fps,
                                   blit=False)
    if save:
        anim.save(save, fps=fps, dpi=100)
    return anim
