"""gw_fopt_b200: B200-native generalized bulk-flow many-bubble GW spectrum.

Drop-in for gw_fopt's ``bubble_gw.many_bubbles`` bulk-flow path: the C ABI is
in include/bubble_gw.h (+ include/bubble_gw_b200.h for extensions), the
Python surface in ``gw_fopt_b200.many_bubbles`` (also importable as
``gw_fopt_b200.bubble_gw.many_bubbles``, or under the reference's own module
names after ``install_alias()``).  All spectrum work runs in the in-tree CUDA
library ``libbubble_gw_c.so`` (sm_100a).
"""
import sys
import types

from . import many_bubbles  # noqa: F401

__version__ = "0.2.0"

_REF_EXT = "gw_fopt.bubble_gw._py_bubble_gw"


class _NotProvided(types.ModuleType):
    """A submodule of the reference's extension that this package does not replace."""

    def __getattr__(self, name):
        if name.startswith("__"):
            raise AttributeError(name)
        raise AttributeError(f"{self.__name__}.{name} is not provided by gw_fopt_b200 (bulk-flow path only)")


def install_alias() -> None:
    """Registers ``gw_fopt_b200.many_bubbles`` under the module names of the reference's
    compiled extension, as its PyO3 module registers itself in ``sys.modules``
    (rust/py-bubble-gw/src/lib.rs:41-50): ``gw_fopt.bubble_gw._py_bubble_gw`` and its
    ``many_bubbles`` submodule.  Afterwards unchanged ``from gw_fopt.bubble_gw import
    many_bubbles`` and ``import gw_fopt.bubble_gw.many_bubbles`` load this package's
    classes: through the reference's own pure-Python ``gw_fopt`` package when it is
    importable (its ``bubble_gw/__init__.py`` imports the extension module registered
    here), otherwise through package modules created here.  ``two_bubbles`` and
    ``utils`` of the extension are outside the bulk-flow path and raise on use.
    Call it once, before the first import of ``gw_fopt.bubble_gw``."""
    ext = sys.modules.get(_REF_EXT)
    if ext is None or getattr(ext, "many_bubbles", None) is not many_bubbles:
        ext = types.ModuleType(_REF_EXT, "gw_fopt_b200 stand-in for the reference's compiled extension")
        ext.many_bubbles = many_bubbles
        ext.two_bubbles = _NotProvided(_REF_EXT + ".two_bubbles")
        ext.utils = _NotProvided(_REF_EXT + ".utils")
        sys.modules[_REF_EXT] = ext
        sys.modules[_REF_EXT + ".many_bubbles"] = many_bubbles
    try:
        import gw_fopt.bubble_gw as bg  # the reference's pure-Python package, when installed
    except ImportError:
        top = sys.modules.get("gw_fopt") or types.ModuleType("gw_fopt")
        top.__path__ = getattr(top, "__path__", [])
        bg = types.ModuleType("gw_fopt.bubble_gw")
        bg.__path__ = []
        bg._py_bubble_gw = ext
        bg.two_bubbles, bg.utils = ext.two_bubbles, ext.utils
        top.bubble_gw = bg
        sys.modules.setdefault("gw_fopt", top)
        sys.modules["gw_fopt.bubble_gw"] = bg
    bg.many_bubbles = many_bubbles
    sys.modules["gw_fopt.bubble_gw.many_bubbles"] = many_bubbles
