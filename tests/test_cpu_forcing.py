"""Host-side loading of the time/height-varying geostrophic wind
(``Initialization.py:163-246``): both file forms, and the reference's
rejections of a mismatched file."""
import numpy as np
import pytest

from jax_alfa_b200 import cases
from jax_alfa_b200.api import load_geowind


def _cfg(**over):
    return cases.stable(8, 8, 6, nsteps=10, optGeoWind=1, **over)


def test_per_step_series_round_trip(tmp_path):
    cfg = _cfg()
    cases.write_run_dir(cfg, str(tmp_path))
    Ug, Vg = load_geowind(str(tmp_path / "input" / "GeoWind.npz"), cfg)
    eU, eV = cases.geowind_series(cfg)
    assert np.array_equal(Ug, eU) and np.array_equal(Vg, eV)
    assert Ug.shape == (cases.nsteps_of(cfg) + 1, cfg["nz"])


def test_compact_profiles_are_interpolated_per_level(tmp_path):
    cfg = _cfg()
    nz = cfg["nz"]
    t = np.array([0.0, 0.4, 1.2])
    Up = np.stack([np.linspace(1, 2, nz), np.linspace(3, 5, nz), np.linspace(0, 1, nz)])
    Vp = -Up
    f = tmp_path / "g.npz"
    np.savez(f, dt_geo=cfg["dt"], optGeoWind=np.int32(1), t_profile=t, Ug_profile=Up,
             Vg_profile=Vp)
    Ug, Vg = load_geowind(str(f), cfg)
    tt = np.arange(cases.nsteps_of(cfg) + 1) * cfg["dt"]
    for k in range(nz):
        assert np.allclose(Ug[:, k], np.interp(tt, t, Up[:, k]), rtol=0, atol=1e-15)
    assert np.array_equal(Vg, -Ug)


@pytest.mark.parametrize("bad", ["dt", "opt", "len", "nz", "cover"])
def test_mismatched_files_are_rejected(tmp_path, bad):
    cfg = _cfg()
    n, nz = cases.nsteps_of(cfg) + 1, cfg["nz"]
    kw = dict(dt_geo=cfg["dt"] * (2 if bad == "dt" else 1),
              optGeoWind=np.int32(2 if bad == "opt" else 1))
    if bad == "cover":
        kw.update(t_profile=np.array([0.0, 0.5]), Ug_profile=np.zeros((2, nz)),
                  Vg_profile=np.zeros((2, nz)))
    else:
        shape = (n + (1 if bad == "len" else 0), nz + (1 if bad == "nz" else 0))
        kw.update(Ug_series=np.zeros(shape), Vg_series=np.zeros(shape))
    f = tmp_path / "g.npz"
    np.savez(f, **kw)
    with pytest.raises(ValueError):
        load_geowind(str(f), cfg)
