"""CPU oracle of the learned absorbing band (test infrastructure only).

The band is an extension: jaxphys has no learned boundary, so this module is
pinned by its own finite-difference tests (tests/test_band_oracle.py) rather
than by a reference file.  It restates, in NumPy, what the CUDA band kernels
compute:

* face ownership of the outer cell layer and the per-face cell lists,
* the 54-value stencil features (Ex..Hz with H scaled by eta0 over the 3
  outermost layers x 3 tangential offsets) and their RMS normalisation,
* the per-face network 54 -> 64 -> 64 -> 6 with tanh-form GELU: BF16
  weights, biases and activations, packed-BF16 GELU arithmetic and wide
  accumulation (``emulate=True``) or exact FP64 arithmetic (``emulate=False``),
* the weighted-MSE loss and its parameter gradients,
* the band correction applied after a plain Yee step.

Parameter layout per face (float32, 9360 values): W1[64][64] (out, in;
inputs 54..63 zero), b1[64], W2[64][64], b2[64], W3[16][64] (rows 6..15 zero),
b3[16].
"""

from __future__ import annotations

import numpy as np

N_IN, N_INP, N_HID, N_OUT, N_OUTP = 54, 64, 64, 6, 16
W1, B1 = 0, 64 * 64
W2 = B1 + 64
B2 = W2 + 64 * 64
W3 = B2 + 64
B3 = W3 + 16 * 64
N_PARAMS = B3 + 16
ETA0 = 376.730313668
GELU_C0 = 0.7978845608028654
GELU_C1 = 0.044715


def bf16(x) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties to even), as float32."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    return np.where(np.isfinite(a), out, a).reshape(a.shape)


def bf16_bits_to_float(bits) -> np.ndarray:
    b = np.asarray(bits, dtype=np.uint16).astype(np.uint32) << 16
    return b.view(np.float32)


def unpack(p: np.ndarray):
    """Views (W1, b1, W2, b2, W3, b3) of one face's parameter vector."""
    return (p[W1:B1].reshape(64, 64), p[B1:W2], p[W2:B2].reshape(64, 64), p[B2:W3],
            p[W3:B3].reshape(16, 64), p[B3:N_PARAMS])


def pad_mask() -> np.ndarray:
    m = np.zeros(N_PARAMS, dtype=bool)
    m[W1:B1] = (np.arange(64 * 64) % 64) >= N_IN
    m[W3:B3] = (np.arange(16 * 64) // 64) >= N_OUT
    m[B3:N_PARAMS] = np.arange(16) >= N_OUT
    return m


def init_params(rng: np.random.Generator, out_scale: float = 0.1) -> np.ndarray:
    """He-style initial parameters for the 6 faces, shape [6, N_PARAMS]."""
    P = np.zeros((6, N_PARAMS), dtype=np.float32)
    for f in range(6):
        w1, b1, w2, b2, w3, b3 = unpack(P[f])
        w1[:, :N_IN] = rng.normal(0, np.sqrt(2.0 / N_IN), (64, N_IN))
        w2[:] = rng.normal(0, np.sqrt(2.0 / 64), (64, 64))
        w3[:N_OUT] = rng.normal(0, out_scale * np.sqrt(1.0 / 64), (N_OUT, 64))
    return P


def gelu(x):
    t = np.tanh(GELU_C0 * (x + GELU_C1 * x ** 3))
    return 0.5 * x * (1.0 + t)


def gelu_grad(x):
    t = np.tanh(GELU_C0 * (x + GELU_C1 * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * GELU_C0 * (1.0 + 3.0 * GELU_C1 * x * x)


def gelu_bf16(z):
    """The kernels' packed-BF16 GELU: x = bf16(z); p = bf16(x^2 * c01 + c0) with
    x^2 rounded first; u = bf16(x p); t = bf16(tanh u); h = x / 2;
    g = bf16(h t + h) (tanh exact here, tanh.approx.bf16x2 on the GPU)."""
    r = lambda a: bf16(a).astype(np.float64)
    c0 = float(bf16(np.float32(GELU_C0)).reshape(-1)[0])
    c01 = float(bf16(np.float32(GELU_C0 * GELU_C1)).reshape(-1)[0])
    x = r(z)
    p = r(r(x * x) * c01 + c0)
    u = r(x * p)
    t = r(np.tanh(u))
    h = x * 0.5
    return r(h * t + h)


def _weights(p, emulate):
    """Weights (BF16 when emulating) and biases (BF16 when emulating: the
    kernels carry them as a BF16 column of the weight image)."""
    w1, b1, w2, b2, w3, b3 = unpack(np.asarray(p, dtype=np.float32 if emulate else np.float64))
    q = bf16 if emulate else (lambda a: np.asarray(a, dtype=np.float64))
    return (q(w1).astype(np.float64), q(b1).astype(np.float64), q(w2).astype(np.float64),
            q(b2).astype(np.float64), q(w3).astype(np.float64), q(b3).astype(np.float64))


def forward(p: np.ndarray, x: np.ndarray, emulate: bool = True):
    """Outputs [n, 6] of one face's network for feature rows x [n, 54 or 64]."""
    X = np.zeros((len(x), N_INP), dtype=np.float64)
    X[:, :x.shape[1]] = x
    X[:, N_IN:] = 0.0
    if emulate:
        X = bf16(X).astype(np.float64)
    w1, b1, w2, b2, w3, b3 = _weights(p, emulate)
    act = gelu_bf16 if emulate else gelu
    z1 = X @ w1.T + b1
    g1 = act(z1)
    z2 = g1 @ w2.T + b2
    g2 = act(z2)
    o = g2 @ w3.T + b3
    return o[:, :N_OUT]


def loss_and_grad(p: np.ndarray, x: np.ndarray, tgt: np.ndarray, w: np.ndarray, scale: float,
                  emulate: bool = True):
    """loss = scale * sum_j w_j |o_j - t_j|^2 and d loss / d p (padding entries 0)."""
    X = np.zeros((len(x), N_INP), dtype=np.float64)
    X[:, :x.shape[1]] = x
    X[:, N_IN:] = 0.0
    q = (lambda a: bf16(a).astype(np.float64)) if emulate else (lambda a: a)
    X = q(X)
    w1, b1, w2, b2, w3, b3 = _weights(p, emulate)
    act = gelu_bf16 if emulate else gelu
    z1 = X @ w1.T + b1
    g1 = act(z1)
    z2 = g1 @ w2.T + b2
    g2 = act(z2)
    o = (g2 @ w3.T + b3)[:, :N_OUT]
    r = o - tgt
    ww = np.asarray(w, dtype=np.float64)[:, None]
    loss = float(scale * np.sum(ww * r * r))
    do = 2.0 * scale * ww * r                      # [n, 6]
    do16 = np.zeros((len(x), 16))
    do16[:, :N_OUT] = do
    dg2 = q(do16) @ w3                            # [n, 64]
    dz2 = dg2 * gelu_grad(z2)
    dg1 = q(dz2) @ w2
    dz1 = dg1 * gelu_grad(z1)
    g = np.zeros(N_PARAMS, dtype=np.float64)
    gw1, gb1, gw2, gb2, gw3, gb3 = unpack(g)
    gw3[:N_OUT] = q(do).T @ g2
    gb3[:N_OUT] = do.sum(0)
    gw2[:] = q(dz2).T @ g1
    gb2[:] = dz2.sum(0)
    gw1[:, :N_IN] = (q(dz1).T @ X)[:, :N_IN]
    gb1[:] = dz1.sum(0)
    return loss, g


# ---------------------------------------------------------------------------
# geometry and features


def owner(x: int, y: int, z: int, n) -> int:
    """Owning face of an outer-layer cell (-1 for inner cells)."""
    c = (x, y, z)
    hits = []
    for a in range(3):
        if c[a] == 0:
            hits.append((a, 0))
        elif c[a] == n[a] - 1:
            hits.append((a, 1))
    if not hits:
        return -1
    if len(hits) in (1, 3):
        a, s = hits[0]
        return 2 * a + s
    (a, sa), (b, sb) = hits
    return 2 * a + sa if b == (a + 1) % 3 else 2 * b + sb


def band_cells(n) -> list[np.ndarray]:
    """Outer-layer cell indices per owning face: x and y faces ascending, z
    faces ordered by (y, x) (the order the kernels process them in)."""
    nx, ny, nz = n
    out = [[] for _ in range(6)]
    for x in range(nx):
        for y in range(ny):
            full = x in (0, nx - 1) or y in (0, ny - 1)
            zs = range(nz) if full else (0, nz - 1)
            for z in zs:
                f = owner(x, y, z, n)
                if f >= 0:
                    out[f].append((x * ny + y) * nz + z)
    res = [np.asarray(v, dtype=np.int64) for v in out]
    for f in (4, 5):
        c = res[f]
        res[f] = c[np.lexsort((c, (c // nz) % ny))]
    return res


def features(fields, cells: np.ndarray, face: int):
    """Raw stencils v [m, 54] (H scaled by eta0) and s [m] of outer cells.

    fields: six float arrays of shape (nx, ny, nz).
    """
    n = fields[0].shape
    a, side = face >> 1, face & 1
    t1 = (a + 1) % 3
    coords = np.stack(np.unravel_index(cells, n), axis=1)
    v = np.zeros((len(cells), N_IN), dtype=np.float64)
    for l in range(3):
        for w in range(3):
            q = coords.copy()
            q[:, a] = coords[:, a] + (-l if side else l)
            q[:, t1] = coords[:, t1] + w - 1
            inside = (q[:, t1] >= 0) & (q[:, t1] < n[t1])
            qq = np.where(inside[:, None], q, 0)
            for comp in range(6):
                val = fields[comp][qq[:, 0], qq[:, 1], qq[:, 2]].astype(np.float64)
                if comp >= 3:
                    val = val * ETA0
                v[:, comp * 9 + l * 3 + w] = np.where(inside, val, 0.0)
    s = np.sqrt(np.mean(v * v, axis=1) + 1e-30)
    return v, s


def apply_band(fields, params: np.ndarray, emulate: bool = True):
    """X_c += s * net_f(v / s) on every outer cell (fields updated in place)."""
    n = fields[0].shape
    per = band_cells(n)
    deltas = []
    for f in range(6):
        if len(per[f]) == 0:
            deltas.append(None)
            continue
        v, s = features(fields, per[f], f)
        o = forward(params[f], v / s[:, None], emulate=emulate)
        deltas.append(o * s[:, None])
    for f in range(6):
        if deltas[f] is None:
            continue
        idx = np.unravel_index(per[f], n)
        for c in range(6):
            d = deltas[f][:, c] / (ETA0 if c >= 3 else 1.0)
            fields[c][idx] = (fields[c][idx] + d).astype(fields[c].dtype)
    return fields


def collect(fields_t, ref_next, offset):
    """Training rows of every face: (features v/s [m, 54], targets [m, 6], weights s^2)."""
    n = fields_t[0].shape
    ox, oy, oz = offset
    per = band_cells(n)
    rows = []
    for f in range(6):
        v, s = features(fields_t, per[f], f)
        coords = np.unravel_index(per[f], n)
        tgt = np.zeros((len(per[f]), N_OUT))
        for c in range(6):
            sc = ETA0 if c >= 3 else 1.0
            r = ref_next[c][coords[0] + ox, coords[1] + oy, coords[2] + oz].astype(np.float64)
            tgt[:, c] = (r * sc - fields_t[c][coords].astype(np.float64) * sc) / s
        rows.append((v / s[:, None], tgt, s * s))
    return rows
