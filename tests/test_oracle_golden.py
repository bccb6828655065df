"""The NumPy oracle against golden vectors recorded from the reference's own
sources (``tests/golden/make_golden.py``, ``make_golden_kats.py``)."""
import ast
import os

import numpy as np
import pytest

from jax_alfa_b200 import cases
from oracle.alfa_oracle import AlfaOracle, OracleRun
from tests.golden import replay

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CALL_FIXTURES = [
    ("ref_neutral_16x16x12.npz", "neutral"),
    ("ref_convective_12x12x8.npz", "convective"),
    ("ref_convective_flux_12x12x8.npz", "convective"),
    ("ref_convective_fluxhet_12x12x8.npz", "convective"),
    ("ref_stable_lu_12x12x8.npz", "stable"),
    ("ref_stable_het_12x12x8.npz", "stable"),
    ("ref_convective_fgr2_12x12x8.npz", "convective"),  # FGR = 2: no dealiasing
    ("ref_stable_fgr2_12x12x8.npz", "stable"),
    ("ref_convective_wl_12x12x8.npz", "convective"),  # LASDD-WL (optSgs = 2)
    ("ref_stable_wl4_12x12x8.npz", "stable"),  # LAD-WL (optSgs = 4)
    ("ref_convective_wl_fgr2_12x12x8.npz", "convective"),  # LASDD-WL, FGR = 2
    ("ref_stable_geo_12x12x8.npz", "stable"),  # time/height-varying geostrophic wind
    ("ref_convective_moist_12x12x8.npz", "convective"),  # moisture, constant flux, Qadv
    ("ref_stable_moistq_12x12x8.npz", "stable"),  # moisture, prescribed surface Q
    ("ref_convective_moistq_12x12x8.npz", "convective"),  # heterogeneous surface Q
    ("ref_convective_moistwl_12x12x8.npz", "convective"),  # flux series, LAD-WL, FGR 2
]
MOIST_FIXTURES = [f for f in CALL_FIXTURES if "moist" in f[0]]
# The oracle restates the reference operation for operation; on the same
# NumPy FFT it reproduces the recorded results to the last bit.  The bound
# leaves room for a different NumPy build's pairwise-sum order.
TOL = 1e-13


def _cfg_of(g, case):
    grid = tuple(int(x) for x in g["meta.grid"])
    over = dict(ast.literal_eval(str(g["meta.overrides"])))
    return cases.CASES[case](*grid, nsteps=int(g["meta.steps"]), **over)


@pytest.mark.parametrize("fname,case", CALL_FIXTURES)
def test_every_recorded_call(fname, case):
    g = replay.load(os.path.join(GOLDEN, fname))
    o = AlfaOracle(_cfg_of(g, case))
    recorded = replay.calls(g)
    assert recorded
    with np.errstate(all="ignore"):
        for (fn, c), rec in sorted(recorded.items()):
            res = getattr(o, fn)(*rec["in"])
            res = res if isinstance(res, tuple) else (res,)
            got = dict(replay.flat(res))
            for k, exp in replay.flat(rec["out"]):
                assert k in got, (fn, c, k)
                err = replay.rel_err(got[k], exp)
                assert err <= TOL, f"{fn} call {c} out{k}: rel err {err:.3e}"


def test_fixture_coverage():
    seen = set()
    for fname, case in CALL_FIXTURES:
        g = replay.load(os.path.join(GOLDEN, fname))
        seen |= {fn for fn, _ in replay.calls(g)}
    need = {"Filtering_Explicit", "velocityGradients", "potentialTemperatureGradients",
            "Advection", "ScalarAdvection", "BuoyancyOpt1", "BuoyancyOpt2",
            "DivStressDynamicSGS", "DivFluxDynamicSGS", "DivStressStaticSGS",
            "DivFluxStaticSGS", "RHS_Momentum", "RHS_Scalar", "PressureRC",
            "ThomasPressureSolve", "PressureSolve", "AB2_uvw", "AB2_TH",
            "SurfaceFlux_HomogeneousConstantFlux", "SurfaceFlux_HeterogeneousConstantFlux",
            "SurfaceFlux_HomogeneousVaryingFlux", "SurfaceFlux_HeterogeneousVaryingFlux",
            "SurfaceFlux_HomogeneousPrescribedTemperature",
            "SurfaceFlux_HeterogeneousPrescribedTemperature"}
    assert need <= seen, need - seen


def _run(steps):
    cfg = cases.neutral(32, 32, 32, nsteps=steps)
    o = AlfaOracle(cfg)
    u, v, w, th = cases.initial_fields(cfg, 0)
    r = OracleRun(cfg, u, v, w, th, adv=o.adv_series(*cases.adv_forcing_series(cfg)))
    with np.errstate(all="ignore"):
        for _ in range(steps):
            r.step()
    return r


def test_time_loop_one_step_matches_reference_main():
    g = replay.load(os.path.join(GOLDEN, "ref_neutral_32_step1.npz"))
    r = _run(1)
    for name in ("u", "v", "w", "TH", "p", "beta1_1D", "beta2_1D", "Cs2_1D_avg2"):
        assert replay.rel_err(getattr(r, name), g["final." + name]) <= TOL, name


def test_time_loop_varying_geowind_matches_reference_main():
    """optGeoWind = 1: the geostrophic wind row of each iteration
    (``Main.py:170-174``) reaches the momentum RHS."""
    g = replay.load(os.path.join(GOLDEN, "ref_stable_geo_12x12x8.npz"))
    cfg = _cfg_of(g, "stable")
    steps = cases.nsteps_of(cfg)  # Main.py runs ceil(SimTime / dt) steps
    o = AlfaOracle(cfg)
    u, v, w, th = cases.initial_fields(cfg, int(g["meta.seed"]))
    r = OracleRun(cfg, u, v, w, th,
                  surface_series=o.surface_series(cases.surface_bc_series(cfg)),
                  geowind=o.geowind_series(*cases.geowind_series(cfg)))
    with np.errstate(all="ignore"):
        for _ in range(steps):
            r.step()
    for name in ("u", "v", "w", "TH", "p"):
        assert replay.rel_err(getattr(r, name), g["final." + name]) <= TOL, name


def moist_run_inputs(cfg, o, seed):
    """OracleRun keyword arguments for a moist case (the reference's input
    files as ``cases.write_run_dir`` writes them, non-dimensionalised)."""
    kw = {"Q": cases.initial_moisture(cfg, seed)}
    if cfg["optMoistureSurfBC"] >= 1:
        kw["moisture_series"] = cases.moisture_surface_series(cfg)  # u_scale = Q_scale = 1
    if cfg["optSurfBC"] >= 1:
        kw["surface_series"] = o.surface_series(cases.surface_bc_series(cfg))
    if cfg["optAdvection"] >= 1:
        kw["adv"] = o.adv_series(*cases.adv_forcing_series(cfg)) + (
            cases.adv_moisture_series(cfg) * o.z_scale,)
    return kw


@pytest.mark.parametrize("fname,case", MOIST_FIXTURES)
def test_time_loop_with_moisture_matches_reference_main(fname, case):
    """optMoisture = 1 (Main.py:71-76, 164-198, 246-369, 474-528): the
    humidity and every other state variable after the recorded steps."""
    g = replay.load(os.path.join(GOLDEN, fname))
    cfg = _cfg_of(g, case)
    o = AlfaOracle(cfg)
    seed = int(g["meta.seed"])
    u, v, w, th = cases.initial_fields(cfg, seed)
    r = OracleRun(cfg, u, v, w, th, **moist_run_inputs(cfg, o, seed))
    with np.errstate(all="ignore"):
        for _ in range(cases.nsteps_of(cfg)):  # Main.py runs ceil(SimTime / dt) steps
            r.step()
    for name in ("u", "v", "w", "TH", "Q", "p"):
        assert replay.rel_err(getattr(r, name), g["final." + name]) <= TOL, name


@pytest.mark.slow
def test_time_loop_200_steps_matches_reference_main():
    g = replay.load(os.path.join(GOLDEN, "ref_neutral_32_step200.npz"))
    r = _run(200)
    for name in ("u", "v", "w", "TH", "p"):
        assert replay.rel_err(getattr(r, name), g["final." + name]) <= 1e-12, name


def test_roots_and_beta_kats():
    z = np.load(os.path.join(GOLDEN, "ref_kats.npz"))
    for i in range(4):
        got = AlfaOracle.Roots(z[f"testroot{i}.coeffs"], z[f"testroot{i}.guess"])
        assert abs(got - z[f"testroot{i}.root"]) <= 1e-14 * max(1, abs(got))
    q = z["quintic.coeffs"]
    got = AlfaOracle.Roots(q[:, None, :], np.array(AlfaOracle.BETA_GUESSES)[None, :])
    ref = z["quintic.roots"]
    assert (np.isnan(got) == np.isnan(ref)).all()
    ok = ~np.isnan(ref)
    assert np.max(np.abs(got[ok] - ref[ok])) <= 1e-13
    o = AlfaOracle(cases.neutral(8, 8, 8, nsteps=1))
    c = z["beta.coeffs"]
    assert np.array_equal(o.ComputeBeta1(*c), z["beta1"])
    assert np.array_equal(o.ComputeBeta2(*c), z["beta2"])
    assert np.max(np.abs(AlfaOracle.Imfilter(z["imfilter.in"]) - z["imfilter.out"])) <= 1e-15


def test_thomas_matches_dense_lu():
    """Reference claim (docs Config_Reference.ipynb:310): the Thomas solver
    reproduces the dense solve for all non-singular modes."""
    cfg = cases.neutral(12, 10, 9, nsteps=1)
    o = AlfaOracle(cfg)
    rng = np.random.default_rng(3)
    RCr = rng.standard_normal((o.nx, o.ny_rfft, o.nz + 1))
    RCi = rng.standard_normal((o.nx, o.ny_rfft, o.nz + 1))
    fRz = rng.standard_normal((o.nx, o.ny_rfft, o.nz))
    kr2, kc2, a, b, c, bt, mt = o.ThomasPressureInit()
    pt = o.ThomasPressureSolve(RCr, RCi, fRz, bt, mt, c)
    pl = o.PressureSolve(RCr, RCi, fRz, a, b, c)
    for x, y in zip(pt, pl):
        assert replay.rel_err(x, y) <= 1e-11


def test_dealias_triple_product_quirk():
    """Dealias1 output carries the (nx ny)/(mx my) = 4/9 factor and Dealias2
    undoes it once, so padded triple products come back scaled by 4/9
    (``src/operations/Dealiasing.py:76,112``)."""
    o = AlfaOracle(cases.neutral(16, 16, 4, nsteps=1))
    rng = np.random.default_rng(0)
    f = []
    for _ in range(3):
        F = o.FFT(rng.standard_normal((16, 16, 4)))
        kx = np.fft.fftfreq(16, 1 / 16)[:, None, None]
        ky = np.fft.rfftfreq(16, 1 / 16)[None, :, None]
        F[np.broadcast_to((np.abs(kx) >= 3) | (ky >= 3), F.shape)] = 0
        f.append(np.fft.irfft2(F, axes=(0, 1), s=(16, 16)))
    P = [o.Dealias1(o.FFT(x)) for x in f]
    two = o.Dealias2(o.FFT(P[0] * P[1]))
    three = o.Dealias2(o.FFT(P[0] * P[1] * P[2]))
    assert replay.rel_err(two, f[0] * f[1]) < 1e-13
    assert replay.rel_err(three, (4 / 9) * f[0] * f[1] * f[2]) < 1e-13


def test_statistics_match_reference():
    """ComputeStats / InitializeStats (Statistics.py:47-380): two accumulated
    samples (moisture entries included) and a reset, against the reference's
    own outputs."""
    from oracle import alfa_oracle
    z = np.load(os.path.join(GOLDEN, "ref_stats.npz"))
    o = alfa_oracle.AlfaOracle(cases.stable(12, 16, 8, nsteps=1))
    st = alfa_oracle.InitializeStats(o, 8)
    keys = alfa_oracle.STATS_PROFILE_KEYS + alfa_oracle.STATS_SCALAR_KEYS
    for s in (1, 2):
        d = {k[len(f"in{s}."):]: z[k] for k in z.files if k.startswith(f"in{s}.")}
        st = alfa_oracle.ComputeStats(
            o, d["u"], d["v"], d["w"], d["TH"], d["Q"], d["dudz"], d["dvdz"], d["dTHdz"],
            d["dQdz"], d["M_sfc_loc"], d["ustar"], float(d["qz_sfc_avg"]),
            float(d["qm_sfc_avg"]), d["txy"], d["txz"], d["tyz"], d["qz"], d["qHz_q"],
            d["Cs2_1D_avg1"], d["Cs2_1D_avg2"], d["Cs2PrRatio_1D"], d["beta1_1D"],
            d["beta2_1D"], st, 0)
        for k in keys:
            np.testing.assert_allclose(st[k], z[f"acc{s}.{k}"], rtol=1e-13, atol=1e-15,
                                       err_msg=f"sample {s} {k}")
    st = alfa_oracle.ComputeStats(o, *([None] * 23), st, 1)
    for k in keys:
        np.testing.assert_array_equal(st[k], z[f"reset.{k}"])
