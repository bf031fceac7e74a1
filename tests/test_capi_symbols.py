"""The C-ABI library loads on a machine without a GPU and exports every
function declared in include/jaxphys_fdtd.h.  No compute calls."""

import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "jaxphys_fdtd.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(jxf_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "jxf_grid3d_step" in names and "jxf_grid2d_step" in names
    assert len(names) >= 30


def test_library_exports_every_declared_symbol():
    from jaxphys_b200 import _native

    lib = _native.load()
    for name in declared_functions():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", str(_native.LIB_PATH)],
                         capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing


def test_binding_covers_header():
    from jaxphys_b200 import _native

    assert sorted(_native.SIGNATURES) == declared_functions()


def test_version_and_registry():
    from jaxphys_b200 import _native

    lib = _native.load()
    assert lib.jxf_version() >= 100
    assert lib.jxf_num_tma_configs() >= 1


def test_invalid_descriptor_rejected_without_gpu():
    """Argument validation happens on the host before any device call."""
    import ctypes as C

    from jaxphys_b200 import _native

    lib = _native.load()
    d = _native.Grid3DDesc(nx=1, ny=8, nz=8, dx=0.01, dt=0.0, boundary=0, pml_layers=8,
                           cpml_order=3, cpml_r0=1e-6, cpml_kappa_max=1, cpml_alpha_max=0,
                           path=0, device=0)
    h = C.c_void_p()
    assert lib.jxf_grid3d_create(C.byref(d), C.byref(h)) == _native.ERR_INVALID
    assert "at least 2 cells" in _native.last_error()
    d.nx = 8
    d.boundary = 99
    assert lib.jxf_grid3d_create(C.byref(d), C.byref(h)) == _native.ERR_INVALID
    assert lib.jxf_grid3d_step(None, 1, None, None) == _native.ERR_INVALID


@pytest.mark.parametrize("src", ["capi.cu", "fdtd3d_kernels.cuh", "fdtd2d_kernels.cuh"])
def test_sources_have_no_closed_calls(src):
    text = (ROOT / "jaxphys_b200" / "csrc" / src).read_text()
    assert "BatchAsync" not in text
    assert ".multicast::cluster" not in text


STRUCTS = {"jxf_grid3d_desc": "Grid3DDesc", "jxf_grid3d_info": "Grid3DInfo",
           "jxf_noalloc_desc": "NoAllocDesc", "jxf_grid2d_desc": "Grid2DDesc"}


def test_ctypes_structs_match_header_layout(tmp_path):
    """The ctypes mirrors of the header's structs have the C compiler's size
    and field offsets (a C program built from the header prints them)."""
    import ctypes as C
    import shutil

    from jaxphys_b200 import _native

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "jaxphys_fdtd.h"',
             "int main(void) {"]
    for cname, pyname in STRUCTS.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in getattr(_native, pyname)._fields_:
            lines.append(f'  printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {tuple(line.split()[:2]): int(line.split()[2]) for line in out if line}
    for cname, pyname in STRUCTS.items():
        cls = getattr(_native, pyname)
        assert got[(cname, "size")] == C.sizeof(cls), cname
        for field, _ in cls._fields_:
            assert got[(cname, field)] == getattr(cls, field).offset, (cname, field)
