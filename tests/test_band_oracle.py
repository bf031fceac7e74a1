"""CPU checks of the learned-band oracle: gradients against finite
differences, BF16 rounding, face ownership of the outer layer."""

import numpy as np
import pytest

from oracle import band_mlp as bm


def _rows(rng, n):
    x = rng.normal(size=(n, bm.N_IN))
    x /= np.sqrt(np.mean(x * x, axis=1, keepdims=True))
    t = rng.normal(scale=0.3, size=(n, bm.N_OUT))
    w = rng.random(n) + 0.1
    return x, t, w


def test_layout_constants():
    assert bm.N_PARAMS == 9360
    from jaxphys_b200 import _native as nat

    assert nat.BAND_PARAMS == bm.N_PARAMS and nat.BAND_FEATURES == bm.N_IN


def test_grad_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = bm.init_params(rng, out_scale=1.0)[0].astype(np.float64)
    x, t, w = _rows(rng, 40)
    scale = 1.0 / w.sum()
    loss, g = bm.loss_and_grad(p, x, t, w, scale, emulate=False)
    assert loss > 0
    mask = ~bm.pad_mask()
    idx = rng.choice(np.flatnonzero(mask), 60, replace=False)
    idx = np.concatenate([idx, [bm.B1 + 3, bm.B2 + 7, bm.B3 + 2, bm.W3 + 5 * 64 + 9]])
    h = 1e-6
    for k in idx:
        pp = p.copy()
        pm = p.copy()
        pp[k] += h
        pm[k] -= h
        lp, _ = bm.loss_and_grad(pp, x, t, w, scale, emulate=False)
        lm, _ = bm.loss_and_grad(pm, x, t, w, scale, emulate=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 + 1e-5 * abs(fd), (k, fd, g[k])
    assert np.all(g[bm.pad_mask()] == 0)


def test_forward_emulated_close_to_exact():
    rng = np.random.default_rng(4)
    p = bm.init_params(rng, out_scale=1.0)[2]
    x, _, _ = _rows(rng, 200)
    a = bm.forward(p, x, emulate=True)
    b = bm.forward(p, x, emulate=False)
    rel = np.linalg.norm(a - b) / np.linalg.norm(b)
    assert 0 < rel < 2e-2


def test_bf16_rounding():
    vals = np.array([1.0, 1.00390625, 1.005859375, 1.0078125, -3.14159, 0.0, 1e-30],
                    dtype=np.float32)
    r = bm.bf16(vals)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: rounds to even (1.0)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == np.float32(1.0078125) and r[3] == r[2]
    assert abs(r[4] - np.float32(-3.140625)) == 0
    assert r[5] == 0.0
    bits = r.view(np.uint32)
    assert np.all(bits & 0xFFFF == 0)


@pytest.mark.parametrize("n", [(8, 8, 8), (9, 12, 10), (16, 9, 13)])
def test_band_ownership(n):
    per = bm.band_cells(n)
    nx, ny, nz = n
    total = nx * ny * nz - (nx - 2) * (ny - 2) * (nz - 2)
    allc = np.concatenate(per)
    assert len(allc) == total and len(np.unique(allc)) == total
    for f, cells in enumerate(per):
        if f < 4:
            assert np.all(np.diff(cells) > 0)
        else:  # z faces: by (y, x)
            key = ((cells // nz) % ny) * (nx * ny * nz) + cells
            assert np.all(np.diff(key) > 0)
        c = np.stack(np.unravel_index(cells, n), axis=1)
        a, side = f >> 1, f & 1
        assert np.all(c[:, a] == (0 if side == 0 else n[a] - 1))
    # edges: x-y edge -> x face; y-z edge -> y face; z-x edge -> z face; corner -> x face
    assert bm.owner(0, 0, 4, n) == 0
    assert bm.owner(4, ny - 1, 0, n) == 3
    assert bm.owner(nx - 1, 4, nz - 1, n) == 5
    assert bm.owner(0, ny - 1, nz - 1, n) == 0
    assert bm.owner(3, 3, 3, n) == -1


def test_features_of_constant_field():
    n = (10, 9, 8)
    fields = [np.full(n, float(c + 1), np.float32) for c in range(6)]
    per = bm.band_cells(n)
    v, s = bm.features(fields, per[1], 1)   # x-high face, tangent y
    coords = np.stack(np.unravel_index(per[1], n), axis=1)
    inner = (coords[:, 1] > 0) & (coords[:, 1] < n[1] - 1)
    want = np.repeat(np.array([1, 2, 3, 4 * bm.ETA0, 5 * bm.ETA0, 6 * bm.ETA0]), 9)
    np.testing.assert_allclose(v[inner][0], want, rtol=1e-6)
    np.testing.assert_allclose(s[inner][0], np.sqrt(np.mean(want ** 2)), rtol=1e-6)
    # outer tangent positions read zero at the y = 0 edge
    edge = np.flatnonzero(coords[:, 1] == 0)
    if len(edge):
        assert np.all(v[edge[0]][[c * 9 + l * 3 + 0 for c in range(6) for l in range(3)]] == 0)
