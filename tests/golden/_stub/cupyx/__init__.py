"""NumPy stand-in for `cupyx` (golden-fixture generation only)."""
import numpy as _np


def scatter_add(a, idx, v):
    _np.add.at(a, idx, v)
