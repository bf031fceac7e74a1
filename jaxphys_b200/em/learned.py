"""Learned absorbing band (extension): a per-cell MLP boundary a few cells thick.

A PEC-walled grid whose outer 3 cell layers form the band.  After every
plain Yee step, each cell of the outer layer is corrected by one small
network per face (54 -> 64 -> 64 -> 6, tanh-form GELU, BF16 weights with
FP32 accumulation on the tensor cores, C ABI ``jxf_band_*``):

    X_c <- X_c + s * net_f(v / s)

where v is the 3 x 3 stencil (3 band layers along the face normal x -1, 0, +1
along the face's first tangent axis) of the six components (H scaled by
eta0) and s its RMS.  The networks are trained on the GPU by the engine's own
forward/backward kernels against traces of plain 16-layer CPML runs on padded
domains: for a reference state at step n, the truncated grid takes one plain
step and the target is the reference's state at n + 1 (``collect_traces``).

``LearnedBand``       the 6-face model (parameters, training, evaluation)
``BandCase``          one training / evaluation problem (interior box,
                      permittivity, sources)
``collect_traces``    training rows from padded CPML reference runs
``reflection_db``     boundary error of learned / CPML / bare-PEC runs
                      against a padded reference, in dB
"""

from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from .. import _native as nat
from ..exceptions import ConfigurationError, SimulationError
from .fdtd3d import COMPONENTS, CPMLSpec, EMGrid3D, PointSource3D

N_PARAMS = nat.BAND_PARAMS
N_FACES = nat.BAND_FACES
N_FEATURES = nat.BAND_FEATURES
BAND_LAYERS = 3


def _pad_mask() -> np.ndarray:
    m = np.zeros(N_PARAMS, dtype=bool)
    w1 = slice(0, 64 * 64)
    m[w1] = (np.arange(64 * 64) % 64) >= N_FEATURES
    w3 = 64 * 64 + 64 + 64 * 64 + 64
    m[w3:w3 + 16 * 64] = (np.arange(16 * 64) // 64) >= 6
    m[w3 + 16 * 64:] = np.arange(16) >= 6
    return m


def init_params(seed: int = 0, out_scale: float = 0.1) -> np.ndarray:
    """He-style initial parameters [6, N_PARAMS] (padding entries zero)."""
    rng = np.random.default_rng(seed)
    P = np.zeros((N_FACES, N_PARAMS), dtype=np.float32)
    for f in range(N_FACES):
        w1 = P[f, :4096].reshape(64, 64)
        w2 = P[f, 4160:8256].reshape(64, 64)
        w3 = P[f, 8320:9344].reshape(16, 64)
        w1[:, :N_FEATURES] = rng.normal(0, math.sqrt(2.0 / N_FEATURES), (64, N_FEATURES))
        w2[:] = rng.normal(0, math.sqrt(2.0 / 64), (64, 64))
        w3[:6] = rng.normal(0, out_scale / 8.0, (6, 64))
    return P


WEIGHTS = __import__("pathlib").Path(__file__).resolve().parent / "band_weights.npz"
_DEFAULT: dict = {}


def default_band(device: int | None = None) -> "LearnedBand":
    """The shipped band (``band_weights.npz``, made by ``train_band(seed=0)``),
    one shared instance per device."""
    import torch

    dev = torch.cuda.current_device() if device is None else int(device)
    if dev not in _DEFAULT:
        _DEFAULT[dev] = LearnedBand.load(WEIGHTS, device=dev)
    return _DEFAULT[dev]


def _field_ptrs(g: EMGrid3D):
    lib = nat.load()
    out = (C.c_void_p * 6)()
    for c in range(6):
        p = C.c_void_p()
        nat.check(lib.jxf_grid3d_field_ptr(g._h, c, C.byref(p)), "field_ptr")
        out[c] = p.value
    return out


class LearnedBand:
    """The six per-face networks of a learned absorbing band on one GPU."""

    def __init__(self, params: np.ndarray | None = None, *, seed: int = 0,
                 device: int | None = None):
        import torch

        self.device = torch.cuda.current_device() if device is None else int(device)
        h = C.c_void_p()
        nat.check(nat.load().jxf_band_create(self.device, C.byref(h)), "jxf_band_create")
        self._h = h
        self.params = init_params(seed) if params is None else params

    def close(self) -> None:
        """Free the device copy (refused while a grid or batch still uses it)."""
        if self._h is not None:
            nat.check(nat.load().jxf_band_destroy(self._h), "jxf_band_destroy")
            self._h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    @property
    def params(self) -> np.ndarray:
        out = np.empty((N_FACES, N_PARAMS), dtype=np.float32)
        nat.check(nat.load().jxf_band_get_params(self._h, out.ctypes.data), "get_params")
        return out

    @params.setter
    def params(self, p) -> None:
        p = np.ascontiguousarray(np.asarray(p, dtype=np.float32))
        if p.shape != (N_FACES, N_PARAMS):
            raise ConfigurationError(f"params must have shape {(N_FACES, N_PARAMS)}")
        nat.check(nat.load().jxf_band_set_params(self._h, p.ctypes.data), "set_params")

    def save(self, path) -> None:
        np.savez(path, params=self.params)

    @classmethod
    def load(cls, path, device: int | None = None) -> "LearnedBand":
        with np.load(path) as z:
            return cls(z["params"], device=device)

    # ---------------------------------------------------------------- eval
    def eval(self, feat, face) -> np.ndarray:
        """Network outputs [n, 6] for normalised feature rows [n, 54]."""
        x = np.ascontiguousarray(np.asarray(feat, dtype=np.float32))
        f = np.ascontiguousarray(np.asarray(face, dtype=np.int32))
        if x.ndim != 2 or x.shape[1] != N_FEATURES or f.shape != (x.shape[0],):
            raise ConfigurationError("feat must be [n, 54] and face [n]")
        out = np.empty((x.shape[0], 6), dtype=np.float32)
        nat.check(nat.load().jxf_band_eval(self._h, x.shape[0], x.ctypes.data, f.ctypes.data,
                                           out.ctypes.data), "jxf_band_eval")
        return out

    # ------------------------------------------------------------ dataset
    def collect(self, grid: EMGrid3D, ref: EMGrid3D, offset) -> None:
        """Append rows for ``grid``'s outer cells against ``ref``'s state
        (the box of ``grid``'s size at ``offset`` in ``ref``)."""
        ox, oy, oz = (int(v) for v in offset)
        nx, ny, nz = grid.size
        rx, ry, rz = ref.size
        nat.check(nat.load().jxf_band_collect(self._h, _field_ptrs(grid), nx, ny, nz,
                                              _field_ptrs(ref), rx, ry, rz, ox, oy, oz,
                                              nat.stream_handle()), "jxf_band_collect")

    def dataset_size(self) -> np.ndarray:
        out = np.zeros(N_FACES, dtype=np.int64)
        nat.check(nat.load().jxf_band_dataset_size(self._h, out.ctypes.data), "dataset_size")
        return out

    def clear(self) -> None:
        nat.check(nat.load().jxf_band_dataset_clear(self._h), "dataset_clear")

    def dataset(self, face: int, first: int = 0, count: int | None = None):
        """(features float32 [m, 64] as stored in BF16, targets [m, 6], weights [m])."""
        n = int(self.dataset_size()[face])
        count = n - first if count is None else int(count)
        bits = np.empty((count, 64), dtype=np.uint16)
        tgt = np.empty((count, 6), dtype=np.float32)
        w = np.empty(count, dtype=np.float32)
        nat.check(nat.load().jxf_band_dataset_get(self._h, int(face), int(first), count,
                                                  bits.ctypes.data, tgt.ctypes.data,
                                                  w.ctypes.data), "dataset_get")
        feat = (bits.astype(np.uint32) << 16).view(np.float32)
        return feat, tgt, w

    # ------------------------------------------------------------ training
    def grad(self):
        """(gradient [6, N_PARAMS], loss [6]) over the whole dataset."""
        g = np.empty((N_FACES, N_PARAMS), dtype=np.float32)
        loss = np.empty(N_FACES, dtype=np.float32)
        nat.check(nat.load().jxf_band_grad(self._h, g.ctypes.data, loss.ctypes.data,
                                           nat.stream_handle()), "jxf_band_grad")
        return g, loss

    def train(self, iters: int, batch_rows: int = 8192, lr: float = 1e-3,
              seed: int = 0) -> np.ndarray:
        """Adam steps on random rows (batch_rows per face); per-step loss."""
        loss = np.empty(max(int(iters), 0), dtype=np.float32)
        nat.check(nat.load().jxf_band_train(self._h, int(iters), int(batch_rows), float(lr),
                                            int(seed) & 0xFFFFFFFFFFFFFFFF, loss.ctypes.data,
                                            nat.stream_handle()), "jxf_band_train")
        return loss

    def check(self) -> None:
        nat.check(nat.load().jxf_band_check_error(self._h, nat.stream_handle()), "band")


# ---------------------------------------------------------------------------
# problems, training traces and reflection measurement


@dataclass
class BandCase:
    """An interior box with its permittivity and sources (interior coordinates)."""

    size: tuple[int, int, int]
    eps: np.ndarray | None = None
    sources: list = field(default_factory=list)

    def extra_z(self, pad: int) -> int:
        """Vacuum cells added at the high-z end of a grid with `pad` cells per
        side so that nz is a multiple of 4 (16-byte rows: vector loads of the
        z-face band stencil, and the TMA stencil path)."""
        return (-(int(self.size[2]) + 2 * pad)) % 4

    def grid(self, pad: int, boundary: str, pml_layers: int = 0, resolution: float = 1.0,
             path: str = "generic", cpml: CPMLSpec | None = None,
             extra_z: int | None = None) -> EMGrid3D:
        """This case embedded with `pad` vacuum cells on every side and
        `extra_z` (default: ``self.extra_z(pad)``) more vacuum cells at the
        high-z end; the interior starts at (pad, pad, pad) and any
        `pml_layers` of the boundary are the outermost cells."""
        ez = self.extra_z(pad) if extra_z is None else int(extra_z)
        n = [int(v) + 2 * pad for v in self.size]
        n[2] += ez
        n = tuple(n)
        g = EMGrid3D(n, resolution=resolution, boundary=boundary, pml_layers=pml_layers,
                     cpml=cpml, path=path)
        if self.eps is not None:
            eps = np.ones(n, dtype=np.float32)
            sx, sy, sz = self.size
            eps[pad:pad + sx, pad:pad + sy, pad:pad + sz] = self.eps
            g.set_permittivity(eps)
        for s in self.sources:
            x, y, z = s.position
            g.add_source(PointSource3D(frequency=s.frequency, position=(x + pad, y + pad, z + pad),
                                       amplitude=s.amplitude, polarization=s.polarization,
                                       waveform=s.waveform, width_steps=s.width_steps,
                                       delay_steps=s.delay_steps))
        return g


def smooth_eps(rng: np.random.Generator, shape, lo: float, hi: float,
               sigma: float = 4.0) -> np.ndarray:
    """Gaussian-smoothed uniform noise rescaled to [lo, hi] (float32)."""
    from scipy.ndimage import gaussian_filter

    a = gaussian_filter(rng.random(shape), sigma, mode="nearest")
    a = (a - a.min()) / max(float(a.max() - a.min()), 1e-12)
    return (lo + (hi - lo) * a).astype(np.float32)


def random_case(rng: np.random.Generator, size, eps_range=(1.0, 6.0), n_sources: int = 1,
                margin: int = 4, dt_freq: float = 0.05, width: float = 30.0,
                resolution: float = 1.0) -> BandCase:
    """Random smoothed permittivity and dipoles (random position / orientation)
    driven by a Gaussian-modulated sinusoid of centre frequency dt_freq / dt."""
    size = tuple(int(v) for v in size)
    dt = 0.99 * resolution / (299792458.0 * math.sqrt(3.0))
    eps = smooth_eps(rng, size, *eps_range) if eps_range[1] > eps_range[0] else None
    srcs = []
    for _ in range(n_sources):
        pos = tuple(int(rng.integers(margin, s - margin)) for s in size)
        srcs.append(PointSource3D(frequency=dt_freq / dt, position=pos,
                                  polarization=str(rng.choice(["x", "y", "z"])),
                                  waveform="gauss_sine", width_steps=width))
    return BandCase(size, eps, srcs)


def _copy_box(dst: EMGrid3D, src: EMGrid3D, off) -> None:
    ox, oy, oz = off
    nx, ny, nz = dst.size
    for name in COMPONENTS:
        dst.set_field(name, src.field(name)[ox:ox + nx, oy:oy + ny, oz:oz + nz].contiguous())


def _perturb_band(g: EMGrid3D, rel: float, gen) -> None:
    """Add Gaussian noise of `rel` times the band's RMS field to the band layers."""
    import torch

    nx, ny, nz = g.size
    L = BAND_LAYERS
    mask = torch.ones((nx, ny, nz), dtype=torch.bool, device=f"cuda:{g._h_key[1]}")
    mask[L:nx - L, L:ny - L, L:nz - L] = False
    for name in COMPONENTS:
        f = g.field(name)
        rms = torch.sqrt(torch.mean(f[mask] ** 2))
        noise = torch.randn(f.shape, device=f.device, generator=gen) * (rel * rms)
        g.set_field(name, torch.where(mask, f + noise, f))


def collect_traces(model: LearnedBand, case: BandCase, n_steps: int, every: int = 2,
                   start: int = 0, ref_pml: int = 16, resolution: float = 1.0,
                   noise: float = 0.0, seed: int = 0) -> None:
    """Training rows for `case` (band grid = interior + 3 vacuum layers per side).

    The padded reference grid adds `ref_pml` CPML layers around the band grid.
    Every `every` steps from `start`, the band grid is loaded with the
    reference state, takes one plain (PEC) step, and its outer cells are
    compared with the reference one step later.  With `noise` > 0 the band
    layers of the loaded state are perturbed by Gaussian noise of that size
    relative to their RMS (the target stays the unperturbed reference), which
    teaches the networks to pull a perturbed band back.
    """
    import torch

    ez = case.extra_z(BAND_LAYERS)
    ref = case.grid(BAND_LAYERS + ref_pml, "cpml", ref_pml, resolution, path="auto", extra_z=ez)
    trunc = BandCase(case.size, case.eps, []).grid(BAND_LAYERS, "pec", 0, resolution, extra_z=ez)
    ref.prepare()
    trunc.prepare(ref._dt)
    off = (ref_pml, ref_pml, ref_pml)
    gen = torch.Generator(device=f"cuda:{ref._h_key[1]}").manual_seed(int(seed))
    for n in range(int(n_steps)):
        if n >= start and (n - start) % every == 0:
            _copy_box(trunc, ref, off)
            if noise > 0.0:
                _perturb_band(trunc, noise, gen)
            trunc.step(1)
            ref.step(1)
            model.collect(trunc, ref, off)
        else:
            ref.step(1)
    ref.check()
    model.check()
    ref._release()
    trunc._release()


def collect_onpolicy(model: LearnedBand, case: BandCase, n_steps: int, every: int = 2,
                     resync: int = 80, ref_pml: int = 16, resolution: float = 1.0) -> dict:
    """Training rows from the band's own trajectory (DAgger).

    The band grid runs with `model` in the loop next to the padded CPML
    reference.  Every `every` steps its state X is labelled with the exact
    one-step response given X: a copy of the reference in which the band
    grid's box is replaced by X takes one step, and the outer cells of the
    band grid's plain step from X are compared with it.  Every `resync` steps
    the band grid is reset to the reference state, so the visited states stay
    near the reference trajectory.  Returns {"max_rel": largest ratio of the
    band grid's field norm to the reference's} as a stability indicator.
    """
    import torch

    from .batch import FDTDBatch

    ez = case.extra_z(BAND_LAYERS)
    pad = BAND_LAYERS + ref_pml
    ref = case.grid(pad, "cpml", ref_pml, resolution, path="auto", extra_z=ez)
    hyb = case.grid(pad, "cpml", ref_pml, resolution, path="generic", extra_z=ez)
    live = case.grid(BAND_LAYERS, "pec", 0, resolution, extra_z=ez)
    plain = BandCase(case.size, case.eps, []).grid(BAND_LAYERS, "pec", 0, resolution, extra_z=ez)
    ref.prepare()
    dt = ref._dt
    for g in (hyb, live, plain):
        g.prepare(dt)
    b = FDTDBatch([live])
    b.set_band(model)
    off = (ref_pml, ref_pml, ref_pml)
    nx, ny, nz = live.size
    box = (slice(off[0], off[0] + nx), slice(off[1], off[1] + ny), slice(off[2], off[2] + nz))
    max_rel = 0.0
    for n in range(int(n_steps)):
        if n % resync == 0:
            for name in COMPONENTS:
                live.set_field(name, ref.field(name)[box].contiguous())
        if n % every == 0 and n % resync != 0:
            cur = {name: live.field(name) for name in COMPONENTS}
            for name in COMPONENTS:
                full = ref.field(name)
                full[box] = cur[name]
                hyb.set_field(name, full)
                plain.set_field(name, cur[name])
            hyb.step(1)
            plain.step(1)
            model.collect(plain, hyb, off)
        ref.step(1)
        b.run(1, use_graph=False)
        if n % 20 == 19:
            e_live = float(torch.linalg.vector_norm(live.field("ez")))
            e_ref = float(torch.linalg.vector_norm(ref.field("ez")[box])) + 1e-30
            if not math.isfinite(e_live):
                max_rel = float("inf")
                for name in COMPONENTS:
                    live.set_field(name, ref.field(name)[box].contiguous())
            else:
                max_rel = max(max_rel, e_live / e_ref)
    b.close()
    for g in (ref, hyb, live, plain):
        g._release()
    model.check()
    return {"max_rel": max_rel}


def reflection_db(case: BandCase, n_steps: int, model: LearnedBand | None = None,
                  cpml_layers: tuple = (10,), ref_pml: int = 16, every: int = 10,
                  resolution: float = 1.0, pec: bool = True) -> dict:
    """Boundary error of each method against a padded CPML reference, in dB:

        20 log10( ||E - E_ref|| / ||E_ref|| )

    over the interior box and the steps every, 2 every, ... (E = Ex, Ey, Ez).
    Methods: "learned" (band of 3 layers, `model`), "pec" (the same grid
    without the band), "cpml<k>" (k-layer CPML around the interior).
    """
    import torch

    from .batch import FDTDBatch

    runs = {}
    pad_ref = max(BAND_LAYERS, max(cpml_layers) if cpml_layers else 0) + ref_pml
    ref = case.grid(pad_ref, "cpml", ref_pml, resolution, path="auto")
    ref.prepare()
    dt = ref._dt
    if model is not None:
        g = case.grid(BAND_LAYERS, "pec", 0, resolution)
        g.prepare(dt)
        b = FDTDBatch([g])
        b.set_band(model)
        runs["learned"] = (g, BAND_LAYERS, b)
    if pec:
        g = case.grid(BAND_LAYERS, "pec", 0, resolution)
        g.prepare(dt)
        runs["pec"] = (g, BAND_LAYERS, None)
    for k in cpml_layers:
        g = case.grid(k, "cpml", k, resolution, path="auto")
        g.prepare(dt)
        runs[f"cpml{k}"] = (g, k, None)
    num = {k: 0.0 for k in runs}
    den = 0.0
    sx, sy, sz = case.size

    def interior(g, off):
        return torch.stack([g.field(c)[off:off + sx, off:off + sy, off:off + sz]
                            for c in ("ex", "ey", "ez")]).double()

    done = 0
    while done < n_steps:
        k = min(every, n_steps - done)
        ref.step(k)
        for name, (g, off, b) in runs.items():
            if b is not None:
                b.run(k, use_graph=False)
            else:
                g.step(k)
        done += k
        e_ref = interior(ref, pad_ref)
        den += float((e_ref * e_ref).sum())
        for name, (g, off, b) in runs.items():
            d = interior(g, off) - e_ref
            num[name] += float((d * d).sum())
    out = {}
    for name, (g, off, b) in runs.items():
        if not math.isfinite(num[name]):
            out[name] = float("inf")
        else:
            out[name] = 10.0 * math.log10(max(num[name], 1e-300) / max(den, 1e-300))
        if b is not None:
            b.close()
        g._release()
    ref._release()
    if model is not None:
        model.check()
    return out


def train_band(seed: int = 0, n_cases: int = 8, size_range=(18, 40), n_steps: int = 320,
               noise=(0.03,), schedule=((2e-3, 2000), (1e-3, 2000), (3e-4, 2000),
                                            (1e-4, 1000)),
               dagger_rounds: int = 2, dagger_steps: int = 400,
               dagger_schedule=((3e-4, 1500), (1e-4, 1000)),
               batch_rows: int = 8192, freq_range=(0.035, 0.07), width_range=(20.0, 40.0),
               eps_range=(1.0, 6.0), device: int | None = None, log=None) -> LearnedBand:
    """Train a band from scratch on the GPU (the recipe of the shipped weights).

    `n_cases` random boxes (sides in `size_range`, smoothed permittivity in
    `eps_range`, 1-2 dipoles of random position / orientation driven by
    Gaussian-modulated sinusoids of centre frequency in `freq_range` / dt and
    width in `width_range` steps); for each, one trace pass per entry of
    `noise` (band-state perturbation level); Adam with the piecewise constant
    learning-rate `schedule` of (lr, iterations); then `dagger_rounds` rounds
    of on-policy rows (``collect_onpolicy``, `dagger_steps` steps per case)
    each followed by `dagger_schedule`.
    """
    rng = np.random.default_rng(seed)
    model = LearnedBand(seed=seed, device=device)
    cases = []
    for i in range(int(n_cases)):
        size = tuple(int(v) for v in rng.integers(size_range[0], size_range[1] + 1, 3))
        case = random_case(rng, size, eps_range=eps_range, n_sources=int(rng.integers(1, 3)),
                           dt_freq=float(rng.uniform(*freq_range)),
                           width=float(rng.uniform(*width_range)))
        cases.append(case)
        for k, lvl in enumerate(noise):
            collect_traces(model, case, n_steps=n_steps, every=2, start=k % 2, noise=float(lvl),
                           seed=seed * 1000 + i * 10 + k)
    it = 0

    def fit(sched, tag):
        nonlocal it
        for lr, n in sched:
            h = model.train(int(n), batch_rows=batch_rows, lr=float(lr), seed=seed * 7919 + it)
            it += 1
            if log is not None:
                log(f"{tag} lr {lr:g}: mean loss of the last 100 steps {float(np.mean(h[-100:])):.4g}")

    fit(schedule, "traces")
    for r in range(int(dagger_rounds)):
        worst = 0.0
        for case in cases:
            st = collect_onpolicy(model, case, n_steps=dagger_steps)
            worst = max(worst, st["max_rel"])
        if log is not None:
            log(f"on-policy round {r}: rows {int(model.dataset_size().sum())}, "
                f"largest field-norm ratio to the reference {worst:.3g}")
        fit(dagger_schedule, f"round {r}")
    return model
