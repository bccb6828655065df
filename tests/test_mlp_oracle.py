"""CPU checks of the NumPy restatement of the learned-coefficient network:
its backpropagated gradient against central finite differences."""
import numpy as np

from oracle import alfa_mlp_oracle as mo


def test_backprop_matches_finite_differences():
    rng = np.random.default_rng(7)
    p = rng.standard_normal(mo.NPARAM) * 0.3
    X = rng.standard_normal((40, mo.NIN))
    T = rng.standard_normal((40, 2))
    norm = np.concatenate([rng.standard_normal(12) * 0.1, 0.5 + rng.random(12)])
    _, g = mo.loss_and_grad(p, X, T, norm)
    h = 1e-6
    for q in rng.choice(mo.NPARAM, 60, replace=False):
        e = np.zeros_like(p)
        e[q] = h
        fd = (mo.loss_and_grad(p + e, X, T, norm)[0] - mo.loss_and_grad(p - e, X, T, norm)[0]) / (2 * h)
        assert abs(fd - g[q]) <= 1e-7 + 1e-6 * abs(g[q]), (q, fd, g[q])
