"""Module path mirroring ``gw_fopt.bubble_gw`` (src/gw_fopt/bubble_gw/__init__.py:4-11)."""
from .. import many_bubbles  # noqa: F401
