"""2D FDTD solver under the reference's module path
(``src/neurosim/em/fdtd.py``), running on the CUDA engine.

``EMGrid.simulate`` defaults to ``output="auto"``: JAX arrays when JAX is
importable (the reference's result type), torch tensors otherwise.
"""

from __future__ import annotations

from jaxphys_b200.em import fdtd as _impl
from jaxphys_b200.em.fdtd import PlaneWave, Wall

__all__ = ["EMGrid", "PlaneWave", "Wall"]


class EMGrid(_impl.EMGrid):
    __doc__ = _impl.EMGrid.__doc__

    def simulate(self, t_span=(0.0, 1e-8), dt=None, save_every=10, output="auto"):
        """Run the simulation (``fdtd.py:193-386``); results as JAX arrays
        when JAX is importable, else torch tensors."""
        return super().simulate(t_span=t_span, dt=dt, save_every=save_every, output=output)
