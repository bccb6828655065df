"""``jax.numpy.linalg`` stand-in."""
import numpy as _np


def solve(a, b):
    from . import ndarray
    return _np.linalg.solve(_np.asarray(a), _np.asarray(b)).view(ndarray)
