"""GPU tests of the statistics accumulator (src/utilities/Statistics.py:47-380)
and of checkpoint / restart of the whole-step engine."""
import os

import numpy as np
import pytest
import torch

from jax_alfa_b200 import cases
from tests.golden import replay

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-12

# statistics in the same units; a statistic near zero (the plane mean of w,
# zero up to the flow's own fluctuations) is measured against a thousandth of
# the largest statistic of its group
GROUPS = (("U", "V", "W"), ("dUdz", "dVdz"),
          ("u2", "v2", "w2", "uv", "uw", "vw", "txy", "txz", "tyz"),
          ("uTH", "vTH", "wTH", "qz"), ("Cs2_1", "Cs2_2", "Cs2PrRatio", "Beta1", "Beta2"),
          ("wQ", "qHz"))


def stats_err(got, exp, key):
    group = next((g for g in GROUPS if key in g), (key,))
    gmax = max(float(np.abs(np.asarray(exp[k], dtype=np.float64)).max()) for k in group)
    e = np.asarray(exp[key], dtype=np.float64)
    g = np.asarray(got[key], dtype=np.float64)
    scale = max(float(np.abs(e).max()), 1e-3 * gmax, 1e-300)
    return float(np.abs(g - e).max()) / scale


def test_compute_stats_matches_reference():
    """Two accumulated samples (moisture entries included) and a reset through
    alfa_ComputeStats against the reference's own ComputeStats outputs."""
    from jax_alfa_b200.api import Alfa, STATS_PROFILE_KEYS, STATS_SCALAR_KEYS
    z = np.load(os.path.join(GOLDEN, "ref_stats.npz"))
    a = Alfa(cases.stable(12, 16, 8, nsteps=1))
    dev = a.device
    t = lambda x: torch.as_tensor(np.ascontiguousarray(x), dtype=torch.float64, device=dev)
    st = a.InitializeStats()
    for s in (1, 2):
        d = {k[len(f"in{s}."):]: z[k] for k in z.files if k.startswith(f"in{s}.")}
        st = a.ComputeStats(t(d["u"]), t(d["v"]), t(d["w"]), t(d["TH"]), t(d["Q"]),
                            t(d["dudz"]), t(d["dvdz"]), t(d["dTHdz"]), t(d["dQdz"]),
                            t(d["M_sfc_loc"]), t(d["ustar"]), float(d["qz_sfc_avg"]),
                            float(d["qm_sfc_avg"]), t(d["txy"]), t(d["txz"]), t(d["tyz"]),
                            t(d["qz"]), t(d["qHz_q"]), t(d["Cs2_1D_avg1"]),
                            t(d["Cs2_1D_avg2"]), t(d["Cs2PrRatio_1D"]), t(d["beta1_1D"]),
                            t(d["beta2_1D"]), st, 0)
        exp = {k: z[f"acc{s}.{k}"] for k in STATS_PROFILE_KEYS + STATS_SCALAR_KEYS}
        for k in exp:
            if not np.any(exp[k]):
                assert not np.any(st[k]), (s, k)
                continue
            err = stats_err(st, exp, k)
            assert err <= TOL, (s, k, err)
    st = a.ComputeStats(*([None] * 23), st, 1)
    for k in STATS_PROFILE_KEYS + STATS_SCALAR_KEYS:
        assert not np.any(st[k]), k
    a.close()


def _sim(cfg):
    from jax_alfa_b200.api import Simulation
    u, v, w, th = cases.initial_fields(cfg, 0)
    adv = cases.adv_forcing_series(cfg) if cfg["optAdvection"] else None
    sfc = cases.surface_bc_series(cfg) if cfg["optSurfBC"] else None
    return Simulation(cfg, u, v, w, th, surface_series=sfc, adv_series=adv)


def test_stats_sample_matches_oracle_run():
    """The engine's statistics sample after each step (Main.py:547-558)
    against the oracle's time loop with the same arguments."""
    from oracle.alfa_oracle import OracleRun, InitializeStats
    from jax_alfa_b200.api import STATS_PROFILE_KEYS, STATS_SCALAR_KEYS, stats_to_dict
    cfg = cases.convective(24, 24, 16, nsteps=4)
    sim = _sim(cfg)
    u, v, w, th = cases.initial_fields(cfg, 0)
    r = OracleRun(cfg, u, v, w, th, adv=None)
    acc = None
    st = InitializeStats(r.o, 16)
    with np.errstate(all="ignore"):
        for _ in range(3):
            sim.step(1)
            acc = sim.stats_sample(acc)
            r.step()
            st = r.stats_sample(st)
    got = stats_to_dict(acc, 16, cfg["Ugal"])
    for k in STATS_PROFILE_KEYS + STATS_SCALAR_KEYS:
        if not np.any(st[k]):
            assert not np.any(got[k]), k
            continue
        err = stats_err(got, st, k)
        print(f"{k}: {err:.2e}")
        assert err <= 1e-10, (k, err)


def test_moist_stats_sample_matches_oracle_run():
    """The same with optMoisture = 1: Q, dQdz, Q2, wQ, qHz and qm_sfc from the
    engine's state (heterogeneous prescribed surface humidity)."""
    from oracle.alfa_oracle import OracleRun, InitializeStats
    from jax_alfa_b200.api import Simulation, STATS_PROFILE_KEYS, STATS_SCALAR_KEYS, stats_to_dict
    cfg = cases.convective(24, 24, 16, nsteps=4, optMoisture=1, optMoistureSurfBC=2)
    u, v, w, th = cases.initial_fields(cfg, 0)
    Q, ms = cases.initial_moisture(cfg, 0), cases.moisture_surface_series(cfg)
    sim = Simulation(cfg, u, v, w, th, Q=Q, moisture_series=ms)
    r = OracleRun(cfg, u, v, w, th, Q=Q, moisture_series=ms)
    acc = None
    st = InitializeStats(r.o, 16)
    with np.errstate(all="ignore"):
        for _ in range(3):
            sim.step(1)
            acc = sim.stats_sample(acc)
            r.step()
            st = r.stats_sample(st)
    got = stats_to_dict(acc, 16, cfg["Ugal"])
    for k in ("Q", "dQdz", "Q2", "wQ", "qHz", "qm_sfc"):
        assert np.any(st[k]), k
    for k in STATS_PROFILE_KEYS + STATS_SCALAR_KEYS:
        if not np.any(st[k]):
            assert not np.any(got[k]), k
            continue
        err = stats_err(got, st, k)
        print(f"{k}: {err:.2e}")
        assert err <= 1e-10, (k, err)


def test_checkpoint_restart_is_bitwise(tmp_path):
    """4 steps straight == 2 steps, checkpoint to a file, restore in a fresh
    context, 2 more steps (dynamic procedure every 2nd step, so the cached
    coefficients and profiles cross the restart)."""
    cfg = cases.convective(24, 24, 16, nsteps=4, dynamicSGS_call_time=2)
    a = _sim(cfg).step(4)
    ref = {k: t.cpu().numpy() for k, t in a.state().items()}
    b = _sim(cfg).step(2)
    path = b.save(os.path.join(tmp_path, "ckpt.npz"))
    del b
    c = _sim(cfg).load(path).step(2)
    got = {k: t.cpu().numpy() for k, t in c.state().items()}
    for k in ref:
        assert np.array_equal(ref[k], got[k]), k
    assert c.diag()["iteration"] == a.diag()["iteration"]


def test_moist_checkpoint_restart_is_bitwise(tmp_path):
    """The same with optMoisture = 1 (Q and its RHS cross the restart) and a
    prescribed surface humidity series."""
    from jax_alfa_b200.api import Simulation
    cfg = cases.convective(24, 24, 16, nsteps=4, dynamicSGS_call_time=2, optMoisture=1,
                           optMoistureSurfBC=2)
    u, v, w, th = cases.initial_fields(cfg, 0)
    kw = dict(Q=cases.initial_moisture(cfg, 0),
              moisture_series=cases.moisture_surface_series(cfg))

    def sim():
        return Simulation(cfg, u, v, w, th, **kw)
    a = sim().step(4)
    ref = {k: t.cpu().numpy() for k, t in a.state().items()}
    assert "Q" in ref
    b = sim().step(2)
    path = b.save(os.path.join(tmp_path, "ckpt.npz"))
    del b
    c = sim().load(path).step(2)
    got = {k: t.cpu().numpy() for k, t in c.state().items()}
    for k in ref:
        assert np.array_equal(ref[k], got[k]), k
