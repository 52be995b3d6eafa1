"""Minimal stand-in so the reference's plotting imports succeed (plotting is never called)."""
import sys
import types


class _Any:
    def __getattr__(self, name):
        if name.startswith("__"):
            raise AttributeError(name)
        return _Any()

    def __call__(self, *args, **kwargs):
        return _Any()


def _module_getattr(name):
    if name.startswith("__"):
        raise AttributeError(name)
    return _Any()


for _n in ["pyplot", "tri", "cm", "colors", "collections", "patches"]:
    _m = types.ModuleType("matplotlib." + _n)
    _m.__getattr__ = _module_getattr
    sys.modules["matplotlib." + _n] = _m


def __getattr__(name):
    return _module_getattr(name)
