"""A NumPy-backed stand-in for the small part of the ``jax`` API that the
JAX-ALFA reference sources use, so that those sources can be executed in a
container where JAX is not installed.

Test infrastructure only: it is put on ``sys.path`` by
``tests/golden/make_golden.py`` (and nowhere else) to run the reference's own
``src/Main.py`` and hot-path functions and record golden vectors.

Semantics kept from JAX:
  * ``jit`` is the identity (the reference's functions are pure);
  * arrays are immutable from the reference's point of view: ``x.at[i].set(v)``
    returns a modified copy (``jax.numpy.ndarray`` below);
  * ``vmap``/``lax.scan``/``lax.while_loop``/``lax.cond`` run as Python loops
    with the same carry/stack semantics;
  * x64 is enabled (every reference golden run here is FP64), so NumPy's
    float64/complex128 defaults are the JAX x64 defaults.
Arithmetic differences to real JAX are roundoff only: NumPy's pocketfft in
place of XLA's ducc/cuFFT, NumPy's pairwise sums in place of XLA reductions.
"""
import numpy as _np

from . import numpy  # noqa: F401  (jax.numpy)
from . import lax    # noqa: F401  (jax.lax)
from .numpy import _wrap


class _Config:
    jax_enable_x64 = True

    def update(self, name, value):
        setattr(self, name, value)


config = _Config()


def jit(fun=None, **_kwargs):
    if fun is None:
        return lambda f: f
    return fun


def devices():
    return ["cpu:0 (numpy stand-in)"]


def _take(x, i, axis):
    if axis is None:
        return x
    return _wrap(_np.take(_np.asarray(x), i, axis=axis))


def vmap(fun, in_axes=0, out_axes=0):
    """Map ``fun`` over an axis of its arguments with a Python loop and stack
    the results along ``out_axes`` (tuples of results stack element-wise)."""

    def mapped(*args):
        axes = in_axes if isinstance(in_axes, (tuple, list)) else (in_axes,) * len(args)
        n = None
        for a, ax in zip(args, axes):
            if ax is not None:
                n = _np.shape(a)[ax]
                break
        results = [fun(*[_take(a, i, ax) for a, ax in zip(args, axes)]) for i in range(n)]
        if isinstance(results[0], tuple):
            oax = out_axes if isinstance(out_axes, (tuple, list)) else (out_axes,) * len(results[0])
            return tuple(_wrap(_np.stack([r[j] for r in results], axis=oax[j]))
                         for j in range(len(results[0])))
        return _wrap(_np.stack(results, axis=out_axes))

    return mapped
