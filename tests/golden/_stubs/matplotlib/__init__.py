"""Placeholder so the reference's ``import matplotlib.pyplot`` succeeds while
fixtures are generated (the reference only plots in its run loop)."""


def __getattr__(name):
    raise RuntimeError("matplotlib placeholder: plotting unavailable")
