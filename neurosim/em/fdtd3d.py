"""3D FDTD solver under the reference's module path
(``src/neurosim/em/fdtd3d.py``), running on the CUDA engine.

``EMGrid3D.simulate`` defaults to ``output="auto"``: JAX arrays when JAX is
importable (the reference's result type), torch tensors otherwise.
"""

from __future__ import annotations

from jaxphys_b200.em import fdtd3d as _impl
from jaxphys_b200.em.fdtd3d import DielectricRegion, PointSource3D

__all__ = ["EMGrid3D", "PointSource3D", "DielectricRegion"]


class EMGrid3D(_impl.EMGrid3D):
    __doc__ = _impl.EMGrid3D.__doc__

    def simulate(self, t_span=(0.0, 5e-9), dt=None, save_every=20, output="auto",
                 history="device"):
        """Run the simulation (``fdtd3d.py:169-417``); results as JAX arrays
        when JAX is importable, else torch tensors."""
        return super().simulate(t_span=t_span, dt=dt, save_every=save_every, output=output,
                                history=history)
