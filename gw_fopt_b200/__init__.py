"""gw_fopt_b200: B200-native generalized bulk-flow many-bubble GW spectrum.

Drop-in for gw_fopt's ``bubble_gw.many_bubbles`` bulk-flow path: the C ABI is
in include/bubble_gw.h (+ include/bubble_gw_b200.h for extensions), the
Python surface in ``gw_fopt_b200.many_bubbles`` (also importable as
``gw_fopt_b200.bubble_gw.many_bubbles``).  All spectrum work runs in the
in-tree CUDA library ``libbubble_gw_c.so`` (sm_100a).
"""
from . import many_bubbles  # noqa: F401

__version__ = "0.1.0"
