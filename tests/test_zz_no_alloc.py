"""alfa_PlanarMean_noalloc, the plane mean for callers that may not allocate
device memory (for example a JAX/XLA custom call, where XLA owns the GPU's
memory), against the context entry point alfa_PlanarMean.

The no-allocation variant keeps its partial sums in a fixed array inside
the library shared by every call on a device, so the test makes two calls in
a row on different fields and checks that the second result does not carry
anything over from the first.  Runs alone or after the other tests."""
import ctypes

import numpy as np
import pytest

from jax_alfa_b200 import _lib, cases

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-12


def _noalloc(lib, F, nx, ny, nz, out):
    stream = torch.cuda.current_stream().cuda_stream
    return lib.alfa_PlanarMean_noalloc(ctypes.c_void_p(F.data_ptr()), nx, ny, nz,
                                       ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))


def test_noalloc_matches_context_entry_on_two_calls_in_a_row():
    from jax_alfa_b200.api import Alfa
    nx, ny, nz = 48, 24, 40
    a = Alfa(cases.neutral(nx, ny, nz, nsteps=1))
    lib = _lib.load()
    g = torch.Generator(device="cuda").manual_seed(7)
    F1 = torch.randn((nx, ny, nz), dtype=torch.float64, device="cuda", generator=g)
    F2 = torch.randn((nx, ny, nz), dtype=torch.float64, device="cuda", generator=g) * 3.0 + 1.0
    ref1 = a.PlanarMean(F1)
    ref2 = a.PlanarMean(F2)
    out1 = torch.full((nz,), np.nan, dtype=torch.float64, device="cuda")
    out2 = torch.full((nz,), np.nan, dtype=torch.float64, device="cuda")
    assert _noalloc(lib, F1, nx, ny, nz, out1) == 0
    assert _noalloc(lib, F2, nx, ny, nz, out2) == 0
    torch.cuda.synchronize()
    for out, ref in ((out1, ref1), (out2, ref2)):
        o, r = out.cpu().numpy(), ref.cpu().numpy()
        err = np.max(np.abs(o - r)) / np.max(np.abs(r))
        assert err <= TOL, err
    # and against the plain definition (mean over the horizontal plane)
    host = F2.cpu().numpy().mean(axis=(0, 1))
    assert np.max(np.abs(out2.cpu().numpy() - host)) <= 1e-12 * np.max(np.abs(host))
    a.close()


def test_noalloc_rejects_levels_above_its_limit():
    lib = _lib.load()
    F = torch.zeros((2, 2, 4), dtype=torch.float64, device="cuda")
    out = torch.zeros((4,), dtype=torch.float64, device="cuda")
    # nz above the 2048-level limit is refused on the host, before any launch
    rc = _noalloc(lib, F, 2, 2, 4096, out)
    assert rc == -7
