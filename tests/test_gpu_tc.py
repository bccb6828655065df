"""The split-BF16 tensor-core line pass (alfa_tc_line_apply) against the
same line operator applied in FP64 with NumPy's FFT.

The operator of each map is built here from its spectral definition (the
maps of the FP64 line passes: truncation k < cut or k >= n - cut + 1; i*k
with the Nyquist mode zeroed; the 3/2 pad repeating the Nyquist row; the
unpad dropping it), column by column as ifft(map(fft(e_i))).  Tolerance:
the split keeps ~16 significant bits per product and accumulates in FP32,
so the result is held to 3e-5 of the output's maximum."""
import numpy as np
import pytest

from jax_alfa_b200 import cases

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
TOL = 3e-5


def mapped_spectrum(F, name, n_out, cut):
    n = F.shape[0]
    k = np.arange(n)
    if name == "identity":
        return F
    if name == "truncate":
        keep = (k < cut) | (k >= n - cut + 1)
        return F * keep[:, None]
    if name == "derivative":
        kk = np.where(k < n // 2, k, np.where(k == n // 2, 0, k - n))
        return F * (1j * kk)[:, None]
    out = np.zeros((n_out,) + F.shape[1:], dtype=complex)
    if name == "pad":
        h = n // 2
        out[:h + 1] = F[:h + 1]
        out[n_out - h:] = F[n - h:]
        return out
    h = n_out // 2  # unpad
    out[:h] = F[:h]
    out[h + 1:] = F[h + 1 - n_out + n:]
    return out


def operator(name, n_in, n_out, cut):
    I = np.eye(n_in)
    return np.real(np.fft.ifft(mapped_spectrum(np.fft.fft(I, axis=0), name, n_out, cut), axis=0))


@pytest.mark.parametrize("name,n_in,n_out,cut", [
    ("derivative", 256, 256, 0), ("truncate", 256, 256, 64), ("pad", 256, 384, 0),
    ("unpad", 384, 256, 0), ("identity", 128, 128, 0)])
def test_tc_line_pass_matches_fp64_operator(name, n_in, n_out, cut):
    from jax_alfa_b200.api import Alfa
    a = Alfa(cases.neutral(16, 16, 8, nsteps=1))
    rng = np.random.default_rng(7)
    X = rng.standard_normal((n_in, 4, 128)).astype(np.float32)  # 512 columns
    Y = a.tc_line_apply(torch.from_numpy(X).cuda(), name, n_out=n_out, cut=cut)
    got = Y.cpu().numpy().astype(np.float64).reshape(n_out, -1)
    ref = operator(name, n_in, n_out, cut) @ X.astype(np.float64).reshape(n_in, -1)
    err = float(np.abs(got - ref).max() / np.abs(ref).max())
    print(f"{name} {n_in}->{n_out}: max rel err {err:.2e}")
    assert err <= TOL, err
    a.close()


def test_tc_line_pass_rejects_unaligned_shapes():
    from jax_alfa_b200 import _lib
    from jax_alfa_b200.api import Alfa
    a = Alfa(cases.neutral(16, 16, 8, nsteps=1))
    X = torch.zeros((256, 100), dtype=torch.float32, device="cuda")
    with pytest.raises(_lib.AlfaError):
        a.tc_line_apply(X, "derivative")
    a.close()


def test_tc_wait_limit_returns_timeout_and_context_recovers():
    """A wait limit of one mbarrier poll makes the kernel's waits for its own
    products give up: the call returns ALFA_E_TIMEOUT (the kernel waited at
    the full limit for the products in flight and freed its tensor memory).
    With the default limit restored, the same context computes the operator
    correctly."""
    from jax_alfa_b200 import _lib
    from jax_alfa_b200.api import Alfa
    a = Alfa(cases.neutral(16, 16, 8, nsteps=1))
    rng = np.random.default_rng(3)
    X = rng.standard_normal((256, 4, 128)).astype(np.float32)
    Xd = torch.from_numpy(X).cuda()
    assert a.lib.alfa_set_tc_spin_limit(a.ctx, 1) == 0
    with pytest.raises(_lib.AlfaError) as ei:
        a.tc_line_apply(Xd, "derivative")
    assert "(-5)" in str(ei.value) and "gave up" in str(ei.value)
    assert a.lib.alfa_set_tc_spin_limit(a.ctx, 0) == 0
    Y = a.tc_line_apply(Xd, "derivative")
    got = Y.cpu().numpy().astype(np.float64).reshape(256, -1)
    ref = operator("derivative", 256, 256, 0) @ X.astype(np.float64).reshape(256, -1)
    assert float(np.abs(got - ref).max() / np.abs(ref).max()) <= TOL
    a.close()
