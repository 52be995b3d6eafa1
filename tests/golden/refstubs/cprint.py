"""No-op stand-in for the reference's coloured-print dependency (absent here)."""


def c_print(*args, **kwargs):
    pass
