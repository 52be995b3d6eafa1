"""Minimal stand-in for mpl_toolkits.axes_grid1 (used only by the reference's plotting)."""
import sys
import types

_m = types.ModuleType("mpl_toolkits.axes_grid1")
_m.make_axes_locatable = lambda *a, **k: None
sys.modules["mpl_toolkits.axes_grid1"] = _m
