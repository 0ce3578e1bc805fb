"""Placeholder ``matplotlib.pyplot`` (see the package docstring)."""


def __getattr__(name):
    raise RuntimeError("matplotlib placeholder: plotting unavailable")
