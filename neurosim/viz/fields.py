"""Field viewers under the reference's module path (``src/neurosim/viz/fields.py``)."""

from jaxphys_b200.viz.fields import animate_field, plot_field_snapshot  # noqa: F401
