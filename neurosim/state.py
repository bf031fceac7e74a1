"""FDTD result containers under the reference's module path
(``src/neurosim/state.py:271-289,388-414``)."""

from jaxphys_b200.state import EMFieldHistory, EMFieldHistory3D  # noqa: F401
