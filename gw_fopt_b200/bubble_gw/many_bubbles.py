"""``gw_fopt.bubble_gw.many_bubbles`` path for the bulk-flow classes."""
from ..many_bubbles import *  # noqa: F401,F403
from ..many_bubbles import __all__  # noqa: F401
