"""``jax.numpy.fft`` stand-in: NumPy's pocketfft (FP64 in, FP64 out)."""
import numpy as _np


def _w(x):
    from . import ndarray
    return _np.ascontiguousarray(x).view(ndarray)


def rfft2(a, s=None, axes=(-2, -1), norm=None):
    return _w(_np.fft.rfft2(_np.asarray(a), s=s, axes=axes, norm=norm))


def irfft2(a, s=None, axes=(-2, -1), norm=None):
    return _w(_np.fft.irfft2(_np.asarray(a), s=s, axes=axes, norm=norm))


def fftfreq(n, d=1.0):
    return _w(_np.fft.fftfreq(n, d))


def rfftfreq(n, d=1.0):
    return _w(_np.fft.rfftfreq(n, d))
