"""Waveguide analysis under the reference's module path
(``src/neurosim/em/waveguides.py``)."""

from jaxphys_b200.em.waveguides import RectangularWaveguide

__all__ = ["RectangularWaveguide"]
