"""Failure reporting of the whole-step entry points, with the failure made on
the host (no device fault): a NaN planted in the initial velocity must come
back from alfa_get_diag as ALFA_E_NUMERIC after a step, in every precision,
and the context must stay usable (a reset with finite fields steps
normally).  The device-side wait limit is covered by
test_gpu_tc.py::test_tc_wait_limit_returns_timeout_and_context_recovers."""
import ctypes

import numpy as np
import pytest

from jax_alfa_b200 import _lib, cases

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

ALFA_E_NUMERIC = -4


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_nan_state_is_reported_and_context_recovers(prec):
    from jax_alfa_b200.api import Simulation
    cfg = cases.neutral(16, 16, 12, nsteps=4, precision=prec)
    u, v, w, th = cases.initial_fields(cfg, 0)
    bad = u.copy()
    bad[3, 5, 2] = np.nan
    sim = Simulation(cfg, bad, v, w, th, adv_series=cases.adv_forcing_series(cfg))
    sim.step(1)
    a = sim.alfa
    a.lib.alfa_set_stream(a.ctx, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    d = _lib.AlfaDiag()
    rc = a.lib.alfa_get_diag(a.ctx, ctypes.byref(d))
    assert rc == ALFA_E_NUMERIC, rc
    assert b"non-finite" in a.lib.alfa_last_error(a.ctx)
    sim.reset(u, v, w, th)
    sim.step(2)
    assert np.isfinite(sim.diag()["CFL"])
    a.close()
