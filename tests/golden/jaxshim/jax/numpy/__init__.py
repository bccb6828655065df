"""``jax.numpy`` stand-in on NumPy (see the ``jax`` package docstring).

Every array handed back is a :class:`ndarray`, a NumPy subclass that adds
JAX's functional update syntax ``x.at[idx].set(v)`` / ``.add(v)`` (which
return modified copies and never touch ``x``)."""
import numpy as _np

from . import fft  # noqa: F401
from . import linalg  # noqa: F401


class ndarray(_np.ndarray):
    @property
    def at(self):
        return _AtIndexer(self)


class _AtIndexer:
    def __init__(self, arr):
        self._arr = arr

    def __getitem__(self, idx):
        return _AtRef(self._arr, idx)


def _plain_index(idx):
    if isinstance(idx, tuple):
        return tuple(_plain_index(i) for i in idx)
    if isinstance(idx, _np.ndarray):
        return _np.asarray(idx)
    return idx


class _AtRef:
    def __init__(self, arr, idx):
        self._arr = arr
        self._idx = _plain_index(idx)

    def set(self, val):
        out = _np.array(self._arr, copy=True, order="C")
        out[self._idx] = _np.asarray(val)
        return out.view(ndarray)

    def add(self, val):
        out = _np.array(self._arr, copy=True, order="C")
        out[self._idx] += _np.asarray(val)
        return out.view(ndarray)


def _wrap(x):
    if isinstance(x, _np.ndarray) and not isinstance(x, ndarray):
        return x.view(ndarray)
    if isinstance(x, tuple):
        return tuple(_wrap(e) for e in x)
    return x


def array(obj, dtype=None, copy=True):
    return _np.array(obj, dtype=dtype, order="C").view(ndarray)


def asarray(obj, dtype=None):
    return _np.array(obj, dtype=dtype, order="C").view(ndarray)


def __getattr__(name):
    attr = getattr(_np, name)
    if callable(attr) and not isinstance(attr, type):
        def wrapped(*args, **kwargs):
            return _wrap(attr(*args, **kwargs))
        wrapped.__name__ = name
        return wrapped
    return attr
