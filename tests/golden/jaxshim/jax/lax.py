"""``jax.lax`` stand-in (see the package docstring): control flow as Python
loops, and the 2-D 'VALID' correlation that ``Imfilter`` uses."""
import numpy as _np

from .numpy import _wrap

_MISSING = object()


def cond(pred, true_fun, false_fun, *operands, operand=_MISSING):
    if operand is not _MISSING:
        operands = (operand,)
    return true_fun(*operands) if bool(pred) else false_fun(*operands)


def while_loop(cond_fun, body_fun, init_val):
    val = init_val
    while bool(cond_fun(val)):
        val = body_fun(val)
    return val


def _tree_index(xs, i):
    if xs is None:
        return None
    if isinstance(xs, tuple):
        return tuple(_tree_index(x, i) for x in xs)
    return _wrap(_np.asarray(xs)[i])


def _tree_stack(ys):
    if ys[0] is None:
        return None
    if isinstance(ys[0], tuple):
        return tuple(_tree_stack([y[j] for y in ys]) for j in range(len(ys[0])))
    return _wrap(_np.stack([_np.asarray(y) for y in ys]))


def _leading_len(xs):
    if isinstance(xs, tuple):
        return _leading_len(xs[0])
    return _np.shape(xs)[0]


def scan(f, init, xs=None, length=None, reverse=False, unroll=1):
    n = length if xs is None else _leading_len(xs)
    order = range(n - 1, -1, -1) if reverse else range(n)
    carry, ys = init, []
    for i in order:
        carry, y = f(carry, _tree_index(xs, i))
        ys.append(y)
    if reverse:
        ys = ys[::-1]
    return carry, (_tree_stack(ys) if ys else None)


def conv_general_dilated(lhs, rhs, window_strides, padding, *args, **kwargs):
    """NCHW x OIHW cross-correlation, stride 1, 'VALID' padding only."""
    assert tuple(window_strides) == (1, 1) and padding == "VALID"
    lhs = _np.asarray(lhs)
    rhs = _np.asarray(rhs)
    kh, kw = rhs.shape[2], rhs.shape[3]
    oh, ow = lhs.shape[2] - kh + 1, lhs.shape[3] - kw + 1
    out = _np.zeros((lhs.shape[0], rhs.shape[0], oh, ow), dtype=_np.result_type(lhs, rhs))
    for a in range(kh):
        for b in range(kw):
            out[:, 0] += lhs[:, 0, a:a + oh, b:b + ow] * rhs[0, 0, a, b]
    return _wrap(out)
