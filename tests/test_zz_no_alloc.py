"""The allocation-free entry point, jxf_grid3d_run_noalloc, through the C ABI.

Some callers cannot call cudaMalloc: code that runs inside another
framework's device memory pool (an XLA custom call, for instance, which must
not take device memory behind the pool's back) or hosts that forbid
allocation at run time.
For them the library keeps a fixed scratch array on every device and steps
the caller's own field buffers with it.  This test checks that entry point
against the regular handle-based one (jxf_grid3d_create / jxf_grid3d_step) on
the same initial fields and permittivity, for two calls in a row (an odd and
an even number of steps, so both the copy-back and the in-place ending run),
to the FP32 tolerance the other GPU tests use.  The file sorts last so a run
that stops at the first failure has already run every other test.
"""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPE = (20, 18, 24)
TOL = 1e-6


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(np.sum((a - b) ** 2)) / max(np.sqrt(np.sum(b * b)), 1e-300))


def _handle_grid(lib, nat, eps, boundary):
    nx, ny, nz = SHAPE
    d = nat.Grid3DDesc(nx=nx, ny=ny, nz=nz, dx=0.01, dt=0.0, boundary=boundary,
                       pml_layers=5, cpml_order=3.0, cpml_r0=1e-6, cpml_kappa_max=1.0,
                       cpml_alpha_max=0.0, path=nat.PATH_TMA, device=0)
    h = C.c_void_p()
    nat.check(lib.jxf_grid3d_create(C.byref(d), C.byref(h)), "create")
    if eps is not None:
        nat.check(lib.jxf_grid3d_set_eps_host(h, eps.ctypes.data), "set_eps")
    return h


@pytest.mark.parametrize("boundary,vacuum", [("absorbing", False), ("pec", False),
                                             ("absorbing", True), ("pec", True)])
def test_noalloc_matches_handle_entry_point(cuda, boundary, vacuum):
    """Absorbing and PEC walls, with a permittivity map (per-cell cb) and in
    vacuum (cb == NULL, the constant coefficient)."""
    import torch

    from jaxphys_b200 import _native as nat

    lib = nat.load()
    bnd = nat.BND_ABSORBING if boundary == "absorbing" else nat.BND_PEC
    nx, ny, nz = SHAPE
    rng = np.random.default_rng(7)
    init = [rng.standard_normal(SHAPE).astype(np.float32) * (1.0 if k < 3 else 2.6e-3)
            for k in range(6)]
    eps = None if vacuum else np.ascontiguousarray(1.0 + 3.0 * rng.random(SHAPE))

    h = _handle_grid(lib, nat, eps, bnd)
    try:
        for k in range(6):
            nat.check(lib.jxf_grid3d_set_field(h, k, init[k].ctypes.data, 1, None), "set_field")
        info = nat.Grid3DInfo()
        nat.check(lib.jxf_grid3d_get_info(h, C.byref(info)), "info")
        cb = None
        if eps is not None:
            cb = torch.from_numpy((info.coef_e / eps).astype(np.float32)).to(cuda)
        cb_ptr = None if cb is None else C.c_void_p(cb.data_ptr())
        fields = [torch.from_numpy(a.copy()).to(cuda) for a in init]
        ptrs = (C.c_void_p * 6)(*[f.data_ptr() for f in fields])
        desc = nat.NoAllocDesc(nx=nx, ny=ny, nz=nz, dx=0.01, dt=0.0, boundary=bnd,
                               pml_layers=5, device=0)
        torch.cuda.synchronize()
        for n_steps in (7, 10):  # two calls in a row: odd, then even
            nat.check(lib.jxf_grid3d_step(h, n_steps, None, None), "step")
            ref = []
            for k in range(6):
                out = np.empty(SHAPE, np.float32)
                nat.check(lib.jxf_grid3d_get_field(h, k, out.ctypes.data, 1, None), "get_field")
                ref.append(out)
            nat.check(lib.jxf_grid3d_run_noalloc(C.byref(desc), ptrs, cb_ptr, n_steps, None),
                      "run_noalloc")
            got = [f.cpu().numpy() for f in fields]
            assert _rel(np.stack(got[:3]), np.stack(ref[:3])) <= TOL
            assert _rel(np.stack(got[3:]), np.stack(ref[3:])) <= TOL
    finally:
        lib.jxf_grid3d_destroy(h)


def test_noalloc_rejects_misaligned_pointers(cuda):
    """TMA needs 16-byte aligned buffers: a field or cb pointer that is not is
    refused on the host, before any copy or launch."""
    import torch

    from jaxphys_b200 import _native as nat

    lib = nat.load()
    nx, ny, nz = 8, 8, 8
    buf = torch.zeros(6 * nx * ny * nz + 16, dtype=torch.float32, device=cuda)
    good = [buf.data_ptr() + 4 * k * nx * ny * nz for k in range(6)]
    desc = nat.NoAllocDesc(nx=nx, ny=ny, nz=nz, dx=0.01, dt=0.0, boundary=nat.BND_PEC,
                           pml_layers=0, device=0)
    bad = list(good)
    bad[3] += 4
    ptrs = (C.c_void_p * 6)(*bad)
    assert lib.jxf_grid3d_run_noalloc(C.byref(desc), ptrs, None, 1, None) == nat.ERR_INVALID
    assert "16-byte aligned" in nat.last_error()
    ptrs = (C.c_void_p * 6)(*good)
    cb_bad = C.c_void_p(buf.data_ptr() + 8)
    assert lib.jxf_grid3d_run_noalloc(C.byref(desc), ptrs, cb_bad, 1, None) == nat.ERR_INVALID
    assert "16-byte aligned" in nat.last_error()


def test_noalloc_rejects_grids_over_the_limit(cuda):
    from jaxphys_b200 import _native as nat

    lib = nat.load()
    ptrs = (C.c_void_p * 6)(*([C.c_void_p(16)] * 6))  # never dereferenced: rejected first
    desc = nat.NoAllocDesc(nx=128, ny=128, nz=128, dx=0.01, dt=0.0, boundary=nat.BND_ABSORBING,
                           pml_layers=5, device=0)
    assert lib.jxf_grid3d_run_noalloc(C.byref(desc), ptrs, None, 1, None) == nat.ERR_INVALID
    assert "allocation-free limit" in nat.last_error()
