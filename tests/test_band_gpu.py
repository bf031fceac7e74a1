"""Learned absorbing band on the GPU against the CPU oracle (oracle/band_mlp.py):
tensor-core inference, training-row collection, full-dataset gradients,
the band step inside a batch, and training on CPML traces."""

import ctypes as C

import numpy as np
import pytest

from oracle import band_mlp as bm
from oracle import ref_numpy as rn

pytestmark = pytest.mark.gpu


def _params(seed, out_scale=1.0):
    rng = np.random.default_rng(seed)
    P = bm.init_params(rng, out_scale=out_scale)
    for f in range(6):
        P[f, bm.B1:bm.W2] = rng.normal(0, 0.1, 64)
        P[f, bm.B2:bm.W3] = rng.normal(0, 0.1, 64)
        P[f, bm.B3:bm.B3 + 6] = rng.normal(0, 0.05, 6)
    return P


def _rows(rng, n):
    x = rng.normal(size=(n, bm.N_IN))
    x /= np.sqrt(np.mean(x * x, axis=1, keepdims=True))
    return x.astype(np.float32)


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def test_eval_matches_oracle(cuda):
    from jaxphys_b200.em.learned import LearnedBand

    P = _params(1)
    m = LearnedBand(P)
    np.testing.assert_array_equal(m.params, P)
    rng = np.random.default_rng(2)
    n = 1500
    x = _rows(rng, n)
    face = rng.integers(0, 6, n).astype(np.int32)
    out = m.eval(x, face)
    ref = np.zeros((n, 6))
    exact = np.zeros((n, 6))
    for f in range(6):
        sel = face == f
        ref[sel] = bm.forward(P[f], x[sel], emulate=True)
        exact[sel] = bm.forward(P[f], x[sel], emulate=False)
    # BF16 operands, FP32 accumulation, hardware tanh: within 5e-3 of the
    # emulated oracle and 3e-2 of exact FP64 arithmetic
    assert _rel(out, ref) < 5e-3, _rel(out, ref)
    assert _rel(out, exact) < 3e-2
    m.close()


def _random_fields(torch, shape, seed, smooth=True):
    g = torch.Generator(device="cuda").manual_seed(seed)
    out = []
    for c in range(6):
        a = torch.randn(shape, device="cuda", generator=g)
        if smooth:
            a = torch.nn.functional.avg_pool3d(a[None, None], 3, 1, 1)[0, 0]
        out.append((a / (376.73 if c >= 3 else 1.0)).contiguous())
    return out


def _collect(m, t_fields, r_fields, off):
    from jaxphys_b200 import _native as nat

    tp = (C.c_void_p * 6)(*[f.data_ptr() for f in t_fields])
    rp = (C.c_void_p * 6)(*[f.data_ptr() for f in r_fields])
    nx, ny, nz = t_fields[0].shape
    rx, ry, rz = r_fields[0].shape
    nat.check(nat.load().jxf_band_collect(m._h, tp, nx, ny, nz, rp, rx, ry, rz, *off,
                                          nat.stream_handle()), "collect")


def test_collect_matches_oracle(cuda):
    import torch

    from jaxphys_b200.em.learned import LearnedBand

    m = LearnedBand(_params(3))
    tf = _random_fields(torch, (12, 10, 14), 5)
    rf = _random_fields(torch, (20, 18, 22), 6)
    off = (4, 3, 5)
    _collect(m, tf, rf, off)
    sizes = m.dataset_size()
    rows = bm.collect([t.cpu().numpy() for t in tf], [r.cpu().numpy() for r in rf], off)
    for f in range(6):
        x, t, w = rows[f]
        assert sizes[f] == len(x)
        gx, gt, gw = m.dataset(f)
        np.testing.assert_array_equal(gx[:, 54:], 0)
        # features are stored as BF16 of the FP32 value
        np.testing.assert_allclose(gx[:, :54], x, rtol=2 ** -7, atol=1e-6)
        np.testing.assert_allclose(gt, t, rtol=1e-4, atol=1e-4)
        np.testing.assert_allclose(gw, w, rtol=1e-5)
    m.close()


def test_grad_matches_oracle(cuda):
    import torch

    from jaxphys_b200.em.learned import LearnedBand

    P = _params(7)
    m = LearnedBand(P)
    for k in range(2):  # two collects append
        _collect(m, _random_fields(torch, (13, 11, 12), 10 + k),
                 _random_fields(torch, (17, 15, 16), 20 + k), (2, 2, 2))
    g, loss = m.grad()
    assert np.all(np.isfinite(g)) and np.all(g[:, bm.pad_mask()] == 0)
    for f in range(6):
        x, t, w = m.dataset(f)
        scale = 1.0 / np.sum(w.astype(np.float64))
        lref, gref = bm.loss_and_grad(P[f], x[:, :54], t, w, scale, emulate=True)
        _, gexact = bm.loss_and_grad(P[f], x[:, :54], t, w, scale, emulate=False)
        assert abs(loss[f] - lref) <= 2e-3 * lref, (f, loss[f], lref)
        assert _rel(g[f], gref) < 2e-2, (f, _rel(g[f], gref))
        assert _rel(g[f], gexact) < 5e-2, (f, _rel(g[f], gexact))
        # every parameter block carries gradient
        for a, b in ((bm.W1, bm.B1), (bm.W2, bm.B2), (bm.W3, bm.B3)):
            assert _rel(g[f, a:b], gref[a:b]) < 3e-2
    m.close()


def test_band_step_in_batch_matches_oracle(cuda):
    from jaxphys_b200 import EMGrid3D
    from jaxphys_b200.em.batch import FDTDBatch
    from jaxphys_b200.em.fdtd3d import COMPONENTS
    from jaxphys_b200.em.learned import LearnedBand

    import torch

    n = (14, 12, 16)
    P = _params(11, out_scale=0.3)
    m = LearnedBand(P)
    g = EMGrid3D(n, resolution=1.0, boundary="pec", path="generic")
    g.prepare()
    init = [t.cpu().numpy() for t in _random_fields(torch, n, 13)]
    for name, a in zip(COMPONENTS, init):
        g.set_field(name, a)
    b = FDTDBatch([g])
    b.set_band(m)
    o = rn.Oracle3D(rn.Spec3D(size=n, dx=1.0, boundary="pec"), dt=g._dt, dtype=np.float32)
    o.f = [a.copy() for a in init]
    for k, steps in enumerate((1, 4)):
        b.run(steps, use_graph=bool(k))
        for _ in range(steps):
            o.step()
            bm.apply_band(o.f, P, emulate=True)
        got = [g.field(c).cpu().numpy() for c in COMPONENTS]
        e = np.concatenate([a.ravel() for a in got[:3]])
        e0 = np.concatenate([a.ravel() for a in o.f[:3]])
        h = np.concatenate([a.ravel() for a in got[3:]])
        h0 = np.concatenate([a.ravel() for a in o.f[3:]])
        tol = 5e-3 if k == 0 else 2e-2
        assert _rel(e, e0) < tol and _rel(h, h0) < tol, (k, _rel(e, e0), _rel(h, h0))
    m.check()
    b.close()
    m.close()


def test_training_reduces_loss(cuda):
    from jaxphys_b200.em.learned import LearnedBand, collect_traces, random_case

    m = LearnedBand(seed=0)
    rng = np.random.default_rng(0)
    case = random_case(rng, (14, 16, 12), eps_range=(1.0, 3.0), margin=5)
    collect_traces(m, case, n_steps=160, every=2, start=20)
    sizes = m.dataset_size()
    assert np.all(sizes > 0)
    _, loss0 = m.grad()
    hist = m.train(300, batch_rows=2048, lr=2e-3, seed=1)
    _, loss1 = m.grad()
    assert np.all(np.isfinite(hist)) and np.all(np.isfinite(m.params))
    assert loss1.sum() < 0.5 * loss0.sum(), (loss0.sum(), loss1.sum())
    m.close()


def test_shipped_band_beats_bare_walls_and_is_stable(cuda):
    """The shipped weights against the same grid without the band (bare PEC
    walls) and against 3- and 4-layer CPML, on a held-out problem."""
    from pathlib import Path

    from jaxphys_b200.em.learned import LearnedBand, random_case, reflection_db

    path = Path(__file__).resolve().parents[1] / "jaxphys_b200" / "em" / "band_weights.npz"
    m = LearnedBand.load(path)
    rng = np.random.default_rng(4242)
    case = random_case(rng, (34, 30, 38), eps_range=(1.0, 6.0), n_sources=1)
    r = reflection_db(case, 500, model=m, cpml_layers=(3, 4), every=10)
    assert np.isfinite(r["learned"])
    # the band removes most of the wall reflection (bare walls: ~ -2 dB)
    assert r["learned"] < r["pec"] - 15.0, r
    # and at 3 cells beats the 3-cell CPML
    assert r["learned"] < r["cpml3"] - 5.0, r
    m.close()


def test_onpolicy_collection_appends_rows(cuda):
    from jaxphys_b200.em.learned import LearnedBand, collect_onpolicy, random_case

    m = LearnedBand(seed=3)
    case = random_case(np.random.default_rng(9), (14, 12, 16), eps_range=(1.0, 2.0), margin=5)
    st = collect_onpolicy(m, case, n_steps=40, every=4, resync=20)
    sizes = m.dataset_size()
    assert np.all(sizes > 0) and "max_rel" in st
    x, t, w = m.dataset(0)
    assert np.all(np.isfinite(x)) and np.all(np.isfinite(t)) and np.all(w >= 0)
    m.close()


def test_learned_boundary_grid_matches_batch(cuda):
    """EMGrid3D(boundary="learned") steps through the single-grid path with
    the band attached to the handle; a batch of one PEC grid with the same band
    gives bit-identical fields and probe traces."""
    import torch

    from jaxphys_b200 import EMGrid3D, PointSource3D
    from jaxphys_b200.em.batch import FDTDBatch
    from jaxphys_b200.em.fdtd3d import COMPONENTS
    from jaxphys_b200.em.learned import default_band

    def make(boundary):
        g = EMGrid3D((22, 20, 24), resolution=1.0, boundary=boundary, path="generic")
        dt = g.default_dt()
        g.add_source(PointSource3D(frequency=0.05 / dt, position=(11, 10, 12), polarization="y",
                                   waveform="gauss_sine", width_steps=12.0))
        g.add_probe((4, 5, 6), "ey")
        g.add_probe((18, 2, 20), "hz")
        g.prepare()
        return g

    a = make("learned")
    ta = a.run(120)
    b = make("pec")
    bb = FDTDBatch([b])
    bb.set_band(default_band())
    tb = bb.run(120, use_graph=True)[0]
    assert torch.equal(ta, tb)
    for c in COMPONENTS:
        assert torch.equal(a.field(c), b.field(c)), c
    assert torch.isfinite(a.field("ey")).all()
    # and the learned batch of learned grids attaches the band itself
    c = make("learned")
    bc = FDTDBatch([c])
    assert bc.band is a._band
    h = a.simulate(t_span=(0.0, 60 * a.default_dt()), save_every=20)
    assert torch.isfinite(h.ey).all()


def test_learned_boundary_on_tma_path(cuda):
    """A learned-band grid on the TMA kernel (the band corrects the buffer set
    each step wrote; one step per pass) equals the same grid on the generic
    kernels bit for bit, and a TMA batch of it equals both."""
    import torch

    from jaxphys_b200 import EMGrid3D, PointSource3D
    from jaxphys_b200.em.batch import FDTDBatch
    from jaxphys_b200.em.fdtd3d import COMPONENTS

    def make(path):
        g = EMGrid3D((22, 20, 24), resolution=1.0, boundary="learned", path=path)
        dt = g.default_dt()
        g.add_source(PointSource3D(frequency=0.05 / dt, position=(11, 10, 12), polarization="z",
                                   waveform="gauss_sine", width_steps=12.0))
        g.add_probe((4, 5, 6), "ez")
        g.add_probe((18, 2, 20), "hx")
        g.prepare()
        return g

    a = make("tma")
    assert a.info()["path"] == 2
    ta = a.run(81)
    b = make("generic")
    tb = b.run(81)
    assert torch.equal(ta, tb)
    for c in COMPONENTS:
        assert torch.equal(a.field(c), b.field(c)), c
    c = make("tma")
    bc = FDTDBatch([c])
    assert bc.path == "tma"
    tc = bc.run(81, use_graph=True)[0]
    assert torch.equal(tc, tb)
    for k in COMPONENTS:
        assert torch.equal(c.field(k), b.field(k)), k
    bc.close()


def test_band_destroy_refused_while_attached(cuda):
    from jaxphys_b200 import EMGrid3D
    from jaxphys_b200.em.batch import FDTDBatch
    from jaxphys_b200.em.learned import LearnedBand
    from jaxphys_b200.exceptions import NeurosimError

    m = LearnedBand(seed=2)
    g = EMGrid3D((12, 12, 12), resolution=1.0, boundary="learned", band=m)
    g.prepare()
    b = FDTDBatch([g])
    with pytest.raises(NeurosimError):
        m.close()
    b.close()
    with pytest.raises(NeurosimError):   # the grid still holds it
        m.close()
    g._release()
    m.close()


def test_band_error_paths(cuda):
    """Invalid uses fail with the library's error status, before any device work."""
    import ctypes as C

    import torch

    from jaxphys_b200 import EMGrid3D
    from jaxphys_b200 import _native as nat
    from jaxphys_b200.em.batch import FDTDBatch
    from jaxphys_b200.em.learned import LearnedBand
    from jaxphys_b200.exceptions import ConfigurationError

    lib = nat.load()
    m = LearnedBand(seed=4)
    # a band needs PEC walls
    g = EMGrid3D((12, 12, 12), resolution=1.0, boundary="cpml", pml_layers=3, path="generic")
    g.prepare()
    b = FDTDBatch([g])
    with pytest.raises(ConfigurationError):
        b.set_band(m)
    b.close()
    # and every side >= 8
    small = EMGrid3D((8, 8, 8), resolution=1.0, boundary="pec", path="generic")
    small.prepare()
    tiny_fields = [torch.zeros((7, 9, 9), device="cuda") for _ in range(6)]
    ptrs = (C.c_void_p * 6)(*[t.data_ptr() for t in tiny_fields])
    assert lib.jxf_band_collect(m._h, ptrs, 7, 9, 9, ptrs, 7, 9, 9, 0, 0, 0, None) == nat.ERR_INVALID
    # a box outside the reference grid
    f = [torch.zeros((10, 10, 10), device="cuda") for _ in range(6)]
    fp = (C.c_void_p * 6)(*[t.data_ptr() for t in f])
    assert lib.jxf_band_collect(m._h, fp, 10, 10, 10, fp, 10, 10, 10, 1, 0, 0, None) == nat.ERR_INVALID
    # bad faces / shapes in eval
    with pytest.raises(ConfigurationError):
        m.eval(np.zeros((3, 54), np.float32), np.array([0, 6, 1], np.int32))
    with pytest.raises(ConfigurationError):
        m.eval(np.zeros((3, 50), np.float32), np.zeros(3, np.int32))
    # parameters of the wrong shape
    with pytest.raises(ConfigurationError):
        m.params = np.zeros((6, 100), np.float32)
    small._release()
    g._release()
    m.check()
    m.close()
