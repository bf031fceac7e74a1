"""Generate golden vectors by executing the reference's own FDTD sources.

JAX (pinned jax==0.9.2 / jaxlib==0.9.2 in the reference's uv.lock) is not
installable in this environment, so this script runs the reference modules
``src/neurosim/em/fdtd3d.py`` and ``src/neurosim/em/fdtd.py`` -- unmodified,
loaded from the reference checkout -- against a small NumPy-backed stand-in
for the parts of ``jax`` / ``jax.numpy`` / ``jax.lax`` those two files use
(``zeros``, ``ones``, ``where``, ``arange``, ``broadcast_to``, ``roll``,
``exp``, ``sin``, ``sqrt``, ``asarray``, ``newaxis``, ``pi``,
``Array.at[...].set/add`` and ``lax.scan``).  Every stand-in has the
documented JAX semantics for the way these files call it (out-of-place
``.at`` updates, ``scan`` stacking per-step outputs, float64 under
``jax_enable_x64``), so the fixtures are the reference's algorithm executed
op for op in FP64.

The waveguide fixture runs ``src/neurosim/em/waveguides.py`` the same way
(additionally ``linspace``, ``meshgrid``, ``cos`` and ``nan``).

Usage (needs the reference checkout; not run by the tests)::

    python tests/golden/make_golden.py /path/to/jaxphys [--only waveguides]

Writes ``tests/golden/ref3d_<case>.npz`` and ``tests/golden/ref2d_<case>.npz``
plus ``tests/golden/cases.json`` (the inputs of every case), and
``tests/golden/waveguides.npz`` (cutoffs, propagation constants, mode
patterns and dispersion curves of three guides).
"""

from __future__ import annotations

import importlib.util
import json
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


# ---------------------------------------------------------------------------
# NumPy stand-in for the jax surface used by fdtd3d.py / fdtd.py / state.py
# ---------------------------------------------------------------------------


class _AtIndex:
    def __init__(self, arr, idx):
        self._arr = arr
        self._idx = idx

    def set(self, value):
        out = np.array(self._arr, copy=True)
        out[self._idx] = np.asarray(value)
        return out.view(JArray)

    def add(self, value):
        out = np.array(self._arr, copy=True)
        out[self._idx] = out[self._idx] + np.asarray(value)
        return out.view(JArray)


class _At:
    def __init__(self, arr):
        self._arr = arr

    def __getitem__(self, idx):
        return _AtIndex(self._arr, idx)


class JArray(np.ndarray):
    """ndarray with JAX's functional ``.at[idx].set/add``."""

    @property
    def at(self):
        return _At(self)


def _wrap(x):
    if isinstance(x, np.ndarray):
        return x.view(JArray)
    return x


def _make_jax_modules():
    jnp = types.ModuleType("jax.numpy")
    jnp.pi = np.pi
    jnp.newaxis = np.newaxis
    jnp.float64 = np.float64
    jnp.float32 = np.float32
    jnp.bool_ = np.bool_

    def zeros(shape, dtype=None):
        return _wrap(np.zeros(shape, dtype=np.float64 if dtype is None else dtype))

    def ones(shape, dtype=None):
        return _wrap(np.ones(shape, dtype=np.float64 if dtype is None else dtype))

    jnp.zeros = zeros
    jnp.ones = ones
    jnp.where = lambda c, x, y: _wrap(np.where(np.asarray(c), x, y))
    jnp.arange = lambda *a, **k: _wrap(np.arange(*a, **k))
    jnp.broadcast_to = lambda x, s: _wrap(np.array(np.broadcast_to(np.asarray(x), s)))
    jnp.roll = lambda x, shift, axis=None: _wrap(np.roll(np.asarray(x), shift, axis=axis))
    jnp.exp = lambda x: _wrap(np.exp(x))
    jnp.sin = lambda x: _wrap(np.sin(x))
    jnp.cos = lambda x: _wrap(np.cos(x))
    jnp.nan = np.nan
    jnp.linspace = lambda *a, **k: _wrap(np.linspace(*a, **k))
    jnp.meshgrid = lambda *a, **k: tuple(_wrap(m) for m in np.meshgrid(*a, **k))
    jnp.sqrt = lambda x: _wrap(np.sqrt(x))
    jnp.abs = lambda x: _wrap(np.abs(x))
    jnp.max = lambda x, *a, **k: np.max(x, *a, **k)
    jnp.min = lambda x, *a, **k: np.min(x, *a, **k)
    jnp.mean = lambda x, *a, **k: np.mean(x, *a, **k)
    jnp.sum = lambda x, *a, **k: np.sum(x, *a, **k)
    jnp.asarray = lambda x, dtype=None: _wrap(np.asarray(x, dtype=dtype))
    jnp.array = lambda x, dtype=None: _wrap(np.array(x, dtype=dtype))

    lax = types.ModuleType("jax.lax")

    def scan(f, init, xs, length=None):
        carry = init
        ys = []
        n = length if xs is None else len(xs)
        for i in range(n):
            carry, y = f(carry, None if xs is None else xs[i])
            ys.append(y)
        stacked = tuple(_wrap(np.stack([np.asarray(y[j]) for y in ys]))
                        for j in range(len(ys[0])))
        return carry, stacked

    lax.scan = scan

    jax = types.ModuleType("jax")
    jax.numpy = jnp
    jax.lax = lax
    jax.Array = np.ndarray
    cfg = types.SimpleNamespace(update=lambda *a, **k: None)
    jax.config = cfg
    jax.jit = lambda f, *a, **k: f
    return jax, jnp, lax


def load_reference(ref_root: Path):
    """Import the reference's FDTD modules without its package __init__."""
    jax, jnp, lax = _make_jax_modules()
    sys.modules["jax"] = jax
    sys.modules["jax.numpy"] = jnp
    sys.modules["jax.lax"] = lax
    src = ref_root / "src" / "neurosim"
    pkg = types.ModuleType("neurosim")
    pkg.__path__ = [str(src)]
    sys.modules["neurosim"] = pkg
    em = types.ModuleType("neurosim.em")
    em.__path__ = [str(src / "em")]
    sys.modules["neurosim.em"] = em

    def load(name, path):
        spec = importlib.util.spec_from_file_location(name, path)
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
        return mod

    load("neurosim.exceptions", src / "exceptions.py")
    load("neurosim.state", src / "state.py")
    load("neurosim.config", src / "config.py")
    f3 = load("neurosim.em.fdtd3d", src / "em" / "fdtd3d.py")
    f2 = load("neurosim.em.fdtd", src / "em" / "fdtd.py")
    return f3, f2


def load_reference_waveguides(ref_root: Path):
    """The reference's waveguides.py on the same stand-in (after load_reference)."""
    src = ref_root / "src" / "neurosim"
    spec = importlib.util.spec_from_file_location("neurosim.em.waveguides",
                                                  src / "em" / "waveguides.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["neurosim.em.waveguides"] = mod
    spec.loader.exec_module(mod)
    return mod


# guides (a, b) in metres and the modes / frequencies evaluated on each
GUIDES = [(0.02286, 0.01016), (0.02, 0.01), (0.016, 0.008)]
MODES = [("TE", 1, 0), ("TE", 2, 0), ("TE", 0, 1), ("TE", 1, 1), ("TM", 1, 1), ("TM", 2, 1)]


def waveguide_fixture(wg_mod):
    out = {}
    freqs = np.linspace(2e9, 40e9, 77)
    for gi, (a, b) in enumerate(GUIDES):
        wg = wg_mod.RectangularWaveguide(a=a, b=b)
        for mt, m, n in MODES:
            key = f"g{gi}_{mt}{m}{n}"
            out[key + "_fc"] = np.asarray(wg.cutoff_frequency(m, n))
            fc = wg.cutoff_frequency(m, n)
            fs = np.array([1.05 * fc, 1.5 * fc, 3.0 * fc])
            out[key + "_beta"] = np.array([wg.propagation_constant(float(f), m, n) for f in fs])
            out[key + "_beta_f"] = fs
            mode = wg.compute_mode(mt, m, n, n_points=21)
            out[key + "_pattern"] = np.asarray(mode.field_pattern)
            out[key + "_x"] = np.asarray(mode.x)
            out[key + "_y"] = np.asarray(mode.y)
            out[key + "_disp"] = np.asarray(wg.dispersion_relation(m, n, freqs))
    out["disp_freqs"] = freqs
    return out


# ---------------------------------------------------------------------------
# Cases (inputs mirror the reference's own tests/test_fdtd3d.py, tests/test_em.py
# and examples/, plus boundary-cell sources, overlapping masks, non-cubic grids)
# ---------------------------------------------------------------------------

CASES_3D = [
    dict(name="dipole16", size=[16, 16, 16], resolution=0.01, boundary="absorbing",
         pml_layers=8, t_span=[0.0, 1.0e-9], save_every=10,
         sources=[dict(frequency=5e9, position=[8, 8, 8], amplitude=1.0, polarization="z")],
         materials=[]),
    dict(name="slab16", size=[16, 16, 16], resolution=0.01, boundary="absorbing",
         pml_layers=8, t_span=[0.0, 1.0e-9], save_every=20,
         sources=[dict(frequency=5e9, position=[8, 8, 8], amplitude=1.0, polarization="z")],
         materials=[dict(box=[[10, 16], [0, 16], [0, 16]], epsilon_r=4.0)]),
    dict(name="periodic16", size=[16, 16, 16], resolution=0.01, boundary="periodic",
         pml_layers=0, t_span=[0.0, 6.0e-10], save_every=5,
         sources=[dict(frequency=5e9, position=[8, 8, 8], amplitude=1.0, polarization="z"),
                  dict(frequency=3e9, position=[2, 13, 0], amplitude=0.5, polarization="x")],
         materials=[dict(box=[[0, 5], [3, 9], [0, 16]], epsilon_r=2.5)]),
    dict(name="multisrc20", size=[20, 20, 20], resolution=0.01, boundary="absorbing",
         pml_layers=4, t_span=[0.0, 1.2e-9], save_every=7,
         sources=[dict(frequency=3e9, position=[10, 10, 10], amplitude=1.0, polarization="z"),
                  dict(frequency=4e9, position=[0, 5, 7], amplitude=2.0, polarization="y"),
                  dict(frequency=6e9, position=[19, 19, 19], amplitude=1.5, polarization="x"),
                  dict(frequency=4e9, position=[10, 10, 10], amplitude=0.25, polarization="z")],
         materials=[]),
    dict(name="boxes_noncubic", size=[12, 18, 10], resolution=0.02, boundary="absorbing",
         pml_layers=3, t_span=[2.0e-10, 2.2e-9], save_every=9,
         sources=[dict(frequency=2e9, position=[5, 9, 4], amplitude=1.0, polarization="y")],
         materials=[dict(box=[[0, 8], [4, 14], [2, 9]], epsilon_r=3.0),
                    dict(box=[[4, 12], [0, 9], [0, 5]], epsilon_r=6.0)]),
    dict(name="nopml_pec", size=[10, 9, 11], resolution=0.01, boundary="absorbing",
         pml_layers=0, t_span=[0.0, 6.0e-10], save_every=1,
         sources=[dict(frequency=7e9, position=[4, 4, 5], amplitude=1.0, polarization="z")],
         materials=[]),
]

CASES_2D = [
    dict(name="basic50", size=[50, 50], resolution=0.01, boundary="absorbing",
         pml_layers=10, t_span=[0.0, 1.0e-9], save_every=10,
         sources=[dict(frequency=3e9, y=10, amplitude=1.0)], walls=[]),
    dict(name="slit50", size=[50, 50], resolution=0.01, boundary="absorbing",
         pml_layers=10, t_span=[0.0, 5.0e-10], save_every=5,
         sources=[dict(frequency=3e9, y=10, amplitude=1.0)],
         walls=[dict(y=25, gap_start=20, gap_end=30)]),
    dict(name="multisrc50", size=[50, 50], resolution=0.01, boundary="absorbing",
         pml_layers=10, t_span=[0.0, 2.0e-10], save_every=1,
         sources=[dict(frequency=3e9, y=10, amplitude=1.0),
                  dict(frequency=5e9, y=35, amplitude=0.5)], walls=[]),
    dict(name="periodic40", size=[40, 40], resolution=0.01, boundary="periodic",
         pml_layers=0, t_span=[0.0, 6.0e-10], save_every=3,
         sources=[dict(frequency=3e9, y=2, amplitude=1.0)],
         walls=[dict(y=30, gap_start=10, gap_end=18)]),
    dict(name="reflecting40", size=[40, 40], resolution=0.01, boundary="reflecting",
         pml_layers=0, t_span=[0.0, 6.0e-10], save_every=3,
         sources=[dict(frequency=3e9, y=2, amplitude=1.0)], walls=[]),
    dict(name="diffraction60", size=[60, 44], resolution=0.01, boundary="absorbing",
         pml_layers=8, t_span=[0.0, 1.5e-9], save_every=20,
         sources=[dict(frequency=3e9, y=6, amplitude=1.0)],
         walls=[dict(y=30, gap_start=26, gap_end=34), dict(y=40, gap_start=None, gap_end=None)]),
]


def box_mask(shape, box):
    m = np.zeros(shape, dtype=bool)
    (a0, a1), (b0, b1), (c0, c1) = box
    m[a0:a1, b0:b1, c0:c1] = True
    return m


def run_3d(f3, case):
    grid = f3.EMGrid3D(size=tuple(case["size"]), resolution=case["resolution"],
                       boundary=case["boundary"], pml_layers=case["pml_layers"])
    for s in case["sources"]:
        grid.add_source(f3.PointSource3D(frequency=s["frequency"], position=tuple(s["position"]),
                                         amplitude=s["amplitude"],
                                         polarization=s["polarization"]))
    for m in case["materials"]:
        mask = box_mask(tuple(case["size"]), m["box"]).view(JArray)
        grid.add_material(f3.DielectricRegion(mask=mask, epsilon_r=m["epsilon_r"]))
    h = grid.simulate(t_span=tuple(case["t_span"]), save_every=case["save_every"])
    return {k: np.asarray(getattr(h, k)) for k in
            ("t", "ex", "ey", "ez", "hx", "hy", "hz", "grid_x", "grid_y", "grid_z")}


def run_2d(f2, case):
    grid = f2.EMGrid(size=tuple(case["size"]), resolution=case["resolution"],
                     boundary=case["boundary"], pml_layers=case["pml_layers"])
    for s in case["sources"]:
        grid.add_source(f2.PlaneWave(frequency=s["frequency"], y=s["y"], amplitude=s["amplitude"]))
    for w in case["walls"]:
        grid.add_conductor(f2.Wall(y=w["y"], gap_start=w["gap_start"], gap_end=w["gap_end"]))
    h = grid.simulate(t_span=tuple(case["t_span"]), save_every=case["save_every"])
    return {k: np.asarray(getattr(h, k)) for k in ("t", "ez", "hx", "hy", "grid_x", "grid_y")}


def main(argv):
    args = [a for a in argv[1:] if not a.startswith("--")]
    only = argv[argv.index("--only") + 1] if "--only" in argv else None
    if only is not None and only in args:
        args.remove(only)
    if not args:
        raise SystemExit("usage: python tests/golden/make_golden.py <reference checkout> "
                         "[--only waveguides]")
    ref_root = Path(args[0])
    f3, f2 = load_reference(ref_root)
    wg_mod = load_reference_waveguides(ref_root)
    np.savez_compressed(HERE / "waveguides.npz", **waveguide_fixture(wg_mod))
    print("waveguides: saved")
    if only == "waveguides":
        return
    for case in CASES_3D:
        out = run_3d(f3, case)
        # keep the first, a middle and the last saved frame to bound fixture size
        S = out["t"].shape[0]
        keep = sorted({0, S // 2, S - 1})
        save = {"t": out["t"], "frames": np.asarray(keep), "n_saved": np.asarray(S)}
        for k in ("ex", "ey", "ez", "hx", "hy", "hz"):
            save[k] = out[k][keep]
        for k in ("grid_x", "grid_y", "grid_z"):
            save[k] = out[k]
        np.savez_compressed(HERE / f"ref3d_{case['name']}.npz", **save)
        print("3d", case["name"], "saved", S, "frames; kept", keep)
    for case in CASES_2D:
        out = run_2d(f2, case)
        S = out["t"].shape[0]
        keep = sorted({0, S // 2, S - 1})
        save = {"t": out["t"], "frames": np.asarray(keep), "n_saved": np.asarray(S)}
        for k in ("ez", "hx", "hy"):
            save[k] = out[k][keep]
        for k in ("grid_x", "grid_y"):
            save[k] = out[k]
        np.savez_compressed(HERE / f"ref2d_{case['name']}.npz", **save)
        print("2d", case["name"], "saved", S, "frames; kept", keep)
    with open(HERE / "cases.json", "w") as fh:
        json.dump({"3d": CASES_3D, "2d": CASES_2D}, fh, indent=1)


if __name__ == "__main__":
    main(sys.argv)
