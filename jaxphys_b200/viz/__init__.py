"""Field viewers fed from the solvers' device buffers (reference: ``src/neurosim/viz``)."""

from .fields import (
    animate_field,
    colour_table,
    plot_field_snapshot,
    render_frames,
    render_snapshot,
    save_animation,
    save_snapshot,
)

__all__ = [
    "plot_field_snapshot",
    "animate_field",
    "render_snapshot",
    "render_frames",
    "save_snapshot",
    "save_animation",
    "colour_table",
]
