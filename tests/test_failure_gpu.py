"""Failure detection without a GPU fault.

* A staged copy that never arrives: JXF_FAULT_DROP_STAGE=l makes every block
  of the TMA step kernels (one-step and two-level blocked) leave its l-th
  staged plane unissued.  The consumers' bounded mbarrier waits run out after
  JXF_WAIT_LIMIT_MS, the blocks record where they gave up, wait (bounded) for
  the copies they did issue and return; jxf_grid3d_check_error reports
  JXF_ERR_TIMEOUT.  The same process then runs the same grid normally and
  gets the generic kernel's result bit for bit: the GPU still answers.  Runs
  in a child process so the short wait limit (read once per process) does
  not reach the other tests.
* A tensor-core step that never completes: JXF_FAULT_DROP_MMA=1 leaves the
  first MMA of every learned-band inference CTA unissued; the waits on its
  commit run out, the kernel frees its tensor memory and returns, and
  jxf_band_check_error reports JXF_ERR_TIMEOUT.
* A device allocation that fails: JXF_FAULT_ALLOC_AFTER=n refuses the
  (n+1)-th allocation of a grid creation; every such creation returns
  JXF_ERR_OOM, returns no handle and gives back what it had allocated.
"""

import ctypes as C
import os
import subprocess
import sys
import textwrap
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]

CHILD = textwrap.dedent("""
    import os, sys
    import numpy as np
    sys.path.insert(0, {root!r})
    from jaxphys_b200 import CPMLSpec, EMGrid3D, PointSource3D, SimulationError
    from jaxphys_b200 import _native as nat

    def make(path, blocked):
        g = EMGrid3D(size=(24, 30, 40), resolution=1.0, boundary="cpml", pml_layers=4,
                     path=path, cpml=CPMLSpec())
        g.add_source(PointSource3D(frequency=5e9, position=(12, 15, 20)))
        g.prepare()
        if path == "tma":
            nat.check(nat.load().jxf_grid3d_set_launch(g._h, 0, 4), "set_launch")
            nat.check(nat.load().jxf_grid3d_set_blocked(g._h, 0 if blocked else -1, 4),
                      "set_blocked")
        return g

    for blocked in (False, True):
        g = make("tma", blocked)
        os.environ["JXF_FAULT_DROP_STAGE"] = "2"
        g.step(2)
        try:
            g.check()
        except SimulationError as e:
            assert "did not arrive" in str(e), str(e)
            print("timeout reported", "blocked" if blocked else "one-step")
        else:
            raise AssertionError("the dropped stage was not reported")
        del os.environ["JXF_FAULT_DROP_STAGE"]
        g.reset()
        g.step(9)
        g.check()
        ref = make("generic", False)
        ref.step(9)
        for k in ("ex", "ey", "ez", "hx", "hy", "hz"):
            a = g.field(k).cpu().numpy()
            b = ref.field(k).cpu().numpy()
            assert np.array_equal(a, b), k
        assert np.abs(ref.field("ez").cpu().numpy()).max() > 0
        print("recovered", "blocked" if blocked else "one-step")
""")


def test_dropped_stage_reports_timeout_and_recovers(cuda):
    env = dict(os.environ, JXF_WAIT_LIMIT_MS="200", JXF_AUTOTUNE="0")
    env.pop("JXF_FAULT_DROP_STAGE", None)
    r = subprocess.run([sys.executable, "-c", CHILD.format(root=str(ROOT))], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    for what in ("one-step", "blocked"):
        assert f"timeout reported {what}" in r.stdout
        assert f"recovered {what}" in r.stdout


def test_allocation_failure_leaves_nothing_behind(cuda, monkeypatch):
    import torch

    from jaxphys_b200 import _native as nat

    lib = nat.load()
    torch.cuda.synchronize()
    desc = nat.Grid3DDesc(nx=96, ny=96, nz=96, dx=0.01, dt=0.0, boundary=nat.BND_CPML,
                          pml_layers=6, cpml_order=3.0, cpml_r0=1e-6, cpml_kappa_max=1.0,
                          cpml_alpha_max=0.0, path=nat.PATH_TMA, device=0)
    free0, _ = torch.cuda.mem_get_info(0)
    refused = 0
    for n in range(0, 200):
        monkeypatch.setenv("JXF_FAULT_ALLOC_AFTER", str(n))
        h = C.c_void_p()
        rc = lib.jxf_grid3d_create(C.byref(desc), C.byref(h))
        if rc == nat.OK:
            assert h.value is not None
            lib.jxf_grid3d_destroy(h)
            break
        assert rc == nat.ERR_OOM, nat.last_error()
        assert "fault injection" in nat.last_error()
        assert h.value is None
        refused += 1
    else:
        raise AssertionError("grid creation never succeeded")
    monkeypatch.delenv("JXF_FAULT_ALLOC_AFTER")
    assert refused > 10  # fields, psi sets, tables and error words were each refused once
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    # every refused creation freed what it had allocated (a field alone is
    # 3.5 MB; allow allocator slack)
    assert free0 - free1 < 16 << 20, (free0, free1)


CHILD_BAND = textwrap.dedent("""
    import os, sys
    import numpy as np
    sys.path.insert(0, {root!r})
    from jaxphys_b200 import EMGrid3D, PointSource3D, SimulationError
    from jaxphys_b200.em.batch import FDTDBatch
    from jaxphys_b200.em.learned import default_band

    def make():
        grids = []
        for i, size in enumerate(((24, 20, 28), (30, 26, 32))):
            g = EMGrid3D(size=size, resolution=1.0, boundary="pec", path="tma")
            g.add_source(PointSource3D(frequency=5e9, position=tuple(s // 2 for s in size)))
            g.prepare()
            grids.append(g)
        b = FDTDBatch(grids)
        b.set_band(default_band())
        return grids, b

    band = default_band()
    grids, b = make()
    os.environ["JXF_FAULT_DROP_MMA"] = "1"
    b.run(1, use_graph=False)
    try:
        band.check()
    except SimulationError as e:
        assert "did not complete" in str(e), str(e)
        print("band timeout reported")
    else:
        raise AssertionError("the dropped MMA was not reported")
    del os.environ["JXF_FAULT_DROP_MMA"]
    b.reset()
    b.run(6, use_graph=False)
    band.check()
    ref_grids, ref = make()
    ref.run(6, use_graph=False)
    band.check()
    for g, r in zip(grids, ref_grids):
        for k in ("ex", "ey", "ez", "hx", "hy", "hz"):
            assert np.array_equal(g.field(k).cpu().numpy(), r.field(k).cpu().numpy()), k
    print("band recovered")
""")


def test_band_mma_timeout_reported_and_recovers(cuda):
    """The learned band's tensor-core step: JXF_FAULT_DROP_MMA=1 leaves the
    first MMA of every CTA's first tile unissued; the bounded waits run out,
    the kernel frees its tensor memory and returns, jxf_band_check_error
    reports JXF_ERR_TIMEOUT, and the next runs on the same GPU equal a fresh
    batch bit for bit."""
    env = dict(os.environ, JXF_WAIT_LIMIT_MS="200", JXF_AUTOTUNE="0")
    env.pop("JXF_FAULT_DROP_MMA", None)
    r = subprocess.run([sys.executable, "-c", CHILD_BAND.format(root=str(ROOT))], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "band timeout reported" in r.stdout and "band recovered" in r.stdout
