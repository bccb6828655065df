"""GPU tests of the CUDA-graph step (alfa_step_graph) and of ensembles of
independent simulations stepped by one graph launch per step."""
import numpy as np
import pytest

from jax_alfa_b200 import cases

pytestmark = pytest.mark.gpu


def _sim(cfg, seed=0):
    from jax_alfa_b200.api import Simulation
    u, v, w, th = cases.initial_fields(cfg, seed)
    adv = cases.adv_forcing_series(cfg) if cfg["optAdvection"] else None
    sfc = cases.surface_bc_series(cfg) if cfg["optSurfBC"] else None
    geo = cases.geowind_series(cfg) if cfg["optGeoWind"] else None
    moist = {}
    if cfg["optMoisture"]:
        moist["Q"] = cases.initial_moisture(cfg, seed)
        if cfg["optMoistureSurfBC"]:
            moist["moisture_series"] = cases.moisture_surface_series(cfg)
        if adv is not None:
            adv = adv + (cases.adv_moisture_series(cfg),)
    return Simulation(cfg, u, v, w, th, surface_series=sfc, adv_series=adv, geowind_series=geo,
                      **moist)


def _state(sim):
    return {k: t.cpu().numpy() for k, t in sim.state().items()}


@pytest.mark.parametrize("case,grid,over", [
    ("neutral", (32, 32, 32), {}),                                # advection forcing series
    ("stable", (24, 24, 16), {}),                                 # surface temperature series
    ("convective", (24, 24, 16), {"dynamicSGS_call_time": 3}),    # dynamic and static steps
    ("stable", (24, 24, 16), {"optGeoWind": 1}),                  # geostrophic wind series
    ("neutral", (24, 24, 16), {"optMoisture": 1, "optMoistureSurfBC": 1,
                               "MoistureFlux": 5e-5}),            # moisture with Qadv
])
def test_graph_step_equals_direct_step(case, grid, over):
    cfg = cases.CASES[case](*grid, nsteps=7, **over)
    a = _sim(cfg).step(7)
    b = _sim(cfg).step(7, graph=True)
    sa, sb = _state(a), _state(b)
    for k in sa:
        assert np.array_equal(sa[k], sb[k]), (case, k)
    assert a.diag()["iteration"] == b.diag()["iteration"]


def test_ensemble_equals_members_run_alone():
    from jax_alfa_b200.api import Ensemble
    grids = [(16, 16, 16), (24, 24, 16), (32, 32, 24)]
    cfgs = [cases.neutral(*g, nsteps=5) for g in grids]
    alone = [_state(_sim(c, seed=i).step(5)) for i, c in enumerate(cfgs)]
    ens = Ensemble([_sim(c, seed=i) for i, c in enumerate(cfgs)])
    ens.step(5)
    for i, st in enumerate(ens.states()):
        got = {k: t.cpu().numpy() for k, t in st.items()}
        for k in got:
            assert np.array_equal(got[k], alone[i][k]), (i, k)
    ens.close()


@pytest.mark.parametrize("grid", [(48, 48, 32), (256, 256, 16)])
def test_autotune_picks_the_fastest_equivalent_variant(grid):
    cfg = cases.neutral(*grid, nsteps=4)
    base = _state(_sim(cfg).step(4))
    sim = _sim(cfg)
    cands = sim.autotune(reps=3)
    shapes = {}
    for c in cands:
        shapes.setdefault(c["shape"], []).append(c)
    assert len(shapes) == 8
    for name, cs in shapes.items():
        assert [c["variant"] for c in cs][0] == "default"
        chosen = [c for c in cs if c["chosen"]]
        assert len(chosen) == 1, name
        assert chosen[0]["equal"], name
        assert chosen[0]["ms"] == min(c["ms"] for c in cs if c["equal"]), name
        # the compile-time candidate exists only where a phase-split pass does
        phase = name.endswith("pad") and grid[0] == 256
        assert any(c["variant"] == "compile-time" for c in cs) == phase, name
    tuned = _state(sim.step(4))
    for k in base:
        scale = max(np.abs(base[k]).max(), 1e-300)
        assert np.abs(tuned[k] - base[k]).max() <= 1e-12 * scale, k
    # graphs captured after tuning replay the tuned passes
    g = _sim(cfg)
    g.autotune(reps=1)
    graphed = _state(g.step(4, graph=True))
    for k in base:
        scale = max(np.abs(base[k]).max(), 1e-300)
        assert np.abs(graphed[k] - base[k]).max() <= 1e-12 * scale, k


def test_reset_restarts_the_run_bitwise():
    """Simulation.reset (alfa_init_state on a used context) starts the same
    run again: the buffers return to their carved arrangement, so the steps
    (and the step graphs captured before the reset) repeat bit for bit."""
    cfg = cases.neutral(24, 24, 16, nsteps=6, optMoisture=1, MoistureFlux=5e-5)
    u, v, w, th = cases.initial_fields(cfg, 0)
    q = cases.initial_moisture(cfg, 0)
    fresh = _state(_sim(cfg).step(5, graph=True))
    s = _sim(cfg).step(3, graph=True)
    s.reset(u, v, w, th, Q=q)
    again = _state(s.step(5, graph=True))
    for k in fresh:
        assert np.array_equal(fresh[k], again[k]), k


def test_fp32_ensemble_with_member_draws_equals_members_alone():
    """Members of the ensemble workload (cases.ensemble_members: own seed,
    u* ~ U[0.3, 0.6] m/s, z0 log-uniform in [0.01, 0.5] m; FP32 with the FP64
    tridiagonal solve), two of each size, 100 steps together against each
    run alone: bit for bit (the bar of the workload is 1e-6 relative)."""
    import torch

    from jax_alfa_b200.api import Ensemble
    steps = 100
    pick = [0, 1, 32, 33, 48, 49]
    members = [cases.ensemble_members(nsteps=steps + 1)[i] for i in pick]
    assert len({round(c["ustar"], 6) for c, _ in members}) == len(pick)
    alone = [_state(_sim(c, seed=s).step(1).step(steps - 1, graph=True)) for c, s in members]
    ens = Ensemble([_sim(c, seed=s) for c, s in members])
    ts = torch.cuda.Stream()
    ens.set_stream(ts)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(ts)
    ens.step(steps)
    ev1.record(ts)
    torch.cuda.synchronize()
    # events on the ordering stream bracket the steps: at least a few
    # microseconds of device time per step of 6 members
    assert ev0.elapsed_time(ev1) / steps > 0.05
    for i, st in enumerate(ens.states()):
        got = {k: t.cpu().numpy() for k, t in st.items()}
        for k in got:
            assert np.array_equal(got[k], alone[i][k]), (i, k)
    ens.close()
