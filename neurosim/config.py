"""``EMConfig`` under the reference's module path (``src/neurosim/config.py``)."""

from jaxphys_b200.config import EMConfig  # noqa: F401
