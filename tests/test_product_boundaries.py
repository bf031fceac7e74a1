"""The product package never reaches the CPU oracle, and fails loudly when
its CUDA library is missing (no CPU fallback)."""

import ast
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_package_never_imports_the_oracle():
    paths = list((ROOT / "jaxphys_b200").rglob("*.py")) + list((ROOT / "neurosim").rglob("*.py"))
    for path in paths:
        tree = ast.parse(path.read_text(), filename=str(path))
        for node in ast.walk(tree):
            if isinstance(node, ast.Import):
                names = [a.name for a in node.names]
            elif isinstance(node, ast.ImportFrom):
                names = [node.module or ""]
            else:
                continue
            assert not any(n == "oracle" or n.startswith("oracle.") for n in names), path


def test_missing_library_raises():
    code = ("import os; os.environ['JXF_LIB'] = '/nonexistent/libjaxphys_fdtd.so'\n"
            "from jaxphys_b200 import _native\n"
            "from jaxphys_b200.exceptions import SimulationError\n"
            "try:\n    _native.load()\nexcept SimulationError as e:\n"
            "    print('raised', 'not found' in str(e))\n")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                         cwd=str(ROOT), check=True).stdout
    assert "raised True" in out
