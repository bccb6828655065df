"""Workload definitions: run configurations and seeded initial conditions.

Each case is a dict whose keys are the reference's ``Config.py`` option names
(see ``src/config/ConfigLoader.py:70-157`` for the defaults and
``examples/NBL_A94/runs/*/Config.py`` for a complete file), plus the seeded
initial fields in the reference's input-file convention
(``src/initialization/Initialization.py:58-100``: ``vel.npy`` holds total
u, v, w as Fortran-flattened columns, ``TH.npy`` absolute theta).

Cases (all FP64, 3/2-rule dealiased, FGR=1):
  neutral     32x32x32, pressure-gradient-driven neutral ABL (log-law u,
              u*=0.45 m/s, z0=0.1 m, Coriolis off), LASDD-SM, dt=0.5 s.
              The large-scale forcing is the reference's advective tendency
              (optAdvection=1, ``src/pde/NSE_AllTerms.py:86-88``) held at
              Uadv = u*^2 / Lz.
  nbl_a94     the reference's own neutral-boundary-layer benchmark after
              Andren et al. (1994): a neutral Ekman layer under a 5 m/s
              geostrophic wind, f = 1e-4 1/s, 4000 m cube, Ugal = 3 m/s,
              z0 = 0.01 m, LASDD-SM, dt = 0.75 s, Rayleigh damping above
              2500 m (examples/NBL_A94/runs/256x256x256_LASDD_SM_DP/
              Config.py), the configuration of the reference's A100 256^3
              throughput figures and this build's throughput workload.  (The
              neutral case's own domain at 256^3 is not a usable workload:
              its 7.8 m spacing at dt = 0.5 s puts the spectral CFL number
              near 0.7, where AB2 is unstable.)
  convective  128^3 CBL: 0.24 K m/s surface flux, z0=0.16 m, inversion,
              0.03 m/s velocity noise below 200 m.
  stable      256x256x192 SBL: prescribed surface cooling 0.5 K/h from
              265 K, geostrophic wind 8 m/s, LAD-SM (dynamic Smagorinsky).
"""
import numpy as np

VONK = 0.4

_BASE = dict(
    use_double_precision=True, optGPU=1, GPU_ID=0,
    istep=1, Ugal=0.0,
    optSurfFlux=0, optSurfBC=0, z0m=0.1, z0T=0.1, zTemperature=0.0,
    SensibleHeatFlux=0.0, SurfaceBCFile="input/SurfaceBC.npz",
    optGeoWind=0, Ug2=0.0, Vg2=0.0, GeoWindFile="input/GeoWind.npz",
    f_coriolis=0.0, inversion=0.0, optBuoyancy=1, T_0=300.0,
    optSgs=1, dynamicSGS_call_time=1, FGR=1,
    Cs2=0.1 ** 2, Cwl=0.1 ** 2, Cs2PrRatio=0.1 ** 2, CwlPrRatio=0.1 ** 2,
    optDamping=0, RelaxTime=300.0,
    SampleInterval_sec=1.0e9, OutputInterval_sec=1.0e9, Output3DInterval_sec=1.0e9,
    optAdvection=0, AdvectionFile="input/AdvForcing.npz",
    optMoisture=0, zMoisture=0.0, MoistureFlux=0.0, optMoistureSurfBC=0,
    MoistureSurfaceBCFile="input/MoistureSurfaceBC.npz", q_inversion=0.0,
    optPressureSolver=1,
)

USTAR_NEUTRAL = 0.45


def neutral(nx=32, ny=32, nz=32, nsteps=200, **over):
    """The neutral channel-like ABL driven by a constant pressure-gradient
    forcing u*^2 / l_z (``ustar``, default 0.45 m/s), log-law initial wind
    over roughness z0m."""
    cfg = dict(_BASE, l_x=2000.0, l_y=2000.0, l_z=1000.0, nx=nx, ny=ny, nz=nz,
               dt=0.5, optSgs=1, z0m=0.1, z0T=0.1, optAdvection=1,
               z_damping=800.0, optDamping=0, ustar=USTAR_NEUTRAL)
    cfg["case"] = "neutral"
    cfg.update(over)
    cfg.setdefault("SimTime", nsteps * cfg["dt"])
    cfg.setdefault("Uadv_const", cfg["ustar"] ** 2 / cfg["l_z"])   # m s^-2
    return cfg


def ensemble_members(nsteps=500, precision="fp32", seed=2024):
    """The ensemble workload: 64 independent neutral members of uneven sizes
    (32 of 32^3, 16 of 48^3, 16 of 64^3), each with its own seed for the
    initial perturbation, friction velocity u* ~ U[0.3, 0.6] m/s (forcing
    and initial log law) and roughness z0 (= z0m = z0T) log-uniform in
    [0.01, 0.5] m, drawn from one seeded generator.  The time step scales
    with the grid spacing, dt = 0.5 s x 32 / nx, so every member runs at the
    advective CFL number of the 32^3 neutral case (<= 0.13 here): at dt =
    0.5 s the 64^3 members reach CFL ~0.27, where the AB2 growth of the
    highest resolved modes (|amplification| - 1 ~ (pi CFL)^4 / 4 per step)
    outruns the SGS dissipation and the run diverges within a few hundred
    steps, in FP64 as in FP32.  Returns a list of (config, initial-field
    seed)."""
    rng = np.random.default_rng(seed)
    grids = [(32, 32, 32)] * 32 + [(48, 48, 48)] * 16 + [(64, 64, 64)] * 16
    out = []
    for i, g in enumerate(grids):
        ustar = float(rng.uniform(0.3, 0.6))
        z0 = float(np.exp(rng.uniform(np.log(0.01), np.log(0.5))))
        out.append((neutral(*g, nsteps=nsteps, ustar=ustar, z0m=z0, z0T=z0,
                            dt=0.5 * 32 / g[0], precision=precision), 1000 + i))
    return out


def nbl_a94(nx=256, ny=256, nz=256, nsteps=400000, **over):
    cfg = dict(_BASE, l_x=4000.0, l_y=4000.0, l_z=4000.0, nx=nx, ny=ny, nz=nz,
               dt=0.75, Ugal=3.0, optSgs=1, z0m=0.01, z0T=0.01, Ug2=5.0, Vg2=0.0,
               f_coriolis=1.0e-4, inversion=0.0, optDamping=1, z_damping=2500.0,
               RelaxTime=300.0, optAdvection=0)
    cfg["SimTime"] = nsteps * cfg["dt"]
    cfg["case"] = "nbl_a94"
    cfg.update(over)
    return cfg


def convective(nx=128, ny=128, nz=128, nsteps=2000, **over):
    cfg = dict(_BASE, l_x=5120.0, l_y=5120.0, l_z=2048.0, nx=nx, ny=ny, nz=nz,
               dt=0.5, optSgs=1, z0m=0.16, z0T=0.16, optSurfFlux=1,
               SensibleHeatFlux=0.24, f_coriolis=1.0e-4, inversion=3.0 / 1000,
               optDamping=1, z_damping=1650.0, RelaxTime=300.0)
    cfg["SimTime"] = nsteps * cfg["dt"]
    cfg["case"] = "convective"
    cfg.update(over)
    return cfg


def stable(nx=256, ny=256, nz=192, nsteps=1000, **over):
    cfg = dict(_BASE, l_x=400.0, l_y=400.0, l_z=400.0, nx=nx, ny=ny, nz=nz,
               dt=0.1, optSgs=3, z0m=0.1, z0T=0.1, optSurfBC=2, Ug2=8.0,
               Vg2=0.0, Ugal=5.0, f_coriolis=1.4e-4, T_0=265.0,
               inversion=0.01, optDamping=1, z_damping=300.0, RelaxTime=60.0)
    cfg["SimTime"] = nsteps * cfg["dt"]
    cfg["case"] = "stable"
    cfg.update(over)
    return cfg


CASES = {"neutral": neutral, "nbl_a94": nbl_a94,
         "convective": convective, "stable": stable}


def nsteps_of(cfg):
    """``src/config/DerivedVars.py:90``."""
    return int(np.ceil(cfg["SimTime"] / cfg["dt"]))


def z_uvp(cfg):
    """Cell-centre heights (m) as the reference's input generators use them
    (``examples/NBL_A94/runs/*/CreateInputs_NBL_A94.py``: z_k=(k+1/2)dz,
    dz=Lz/(nz-1))."""
    dz = cfg["l_z"] / (cfg["nz"] - 1)
    return (np.arange(cfg["nz"]) + 0.5) * dz


def initial_fields(cfg, seed=0):
    """Dimensional initial (u, v, w, theta), each (nx, ny, nz) C-order, u
    total (Ugal included), theta absolute."""
    nx, ny, nz = cfg["nx"], cfg["ny"], cfg["nz"]
    z = z_uvp(cfg)
    rng = np.random.default_rng(seed)
    u = np.zeros((nx, ny, nz))
    v = np.zeros((nx, ny, nz))
    w = np.zeros((nx, ny, nz))
    th = np.full((nx, ny, nz), float(cfg["T_0"]))
    case = cfg["case"]
    if case == "nbl_a94":
        # CreateInputs_NBL_A94.py: u = Ug, v = w = 0, theta = T_0, with
        # Gaussian noise of 0.03 m/s in u and 1e-3 K in theta below 200 m
        u[:] = cfg["Ug2"]
        for k in range(nz):
            if z[k] <= 200.0:
                u[:, :, k] += 0.03 * rng.standard_normal((nx, ny))
                th[:, :, k] += 1.0e-3 * rng.standard_normal((nx, ny))
    elif case == "neutral":
        prof = (cfg.get("ustar", USTAR_NEUTRAL) / VONK) * np.log(z / cfg["z0m"])
        u[:] = prof[None, None, :]
        for k in range(nz):
            if z[k] < 500.0:
                u[:, :, k] += 0.005 * u[:, :, k] * rng.uniform(-1.0, 1.0, (nx, ny))
                v[:, :, k] += 0.005 * u[:, :, k] * rng.uniform(-1.0, 1.0, (nx, ny))
        th[:] = 300.0
    elif case == "convective":
        prof = np.where(z <= 1350.0, 300.0,
                        np.where(z <= 1450.0, 300.0 + 5.0 * (z - 1350.0) / 100.0,
                                 305.0 + 3.0e-3 * (z - 1450.0)))
        th[:] = prof[None, None, :]
        for k in range(nz):
            if z[k] < 1000.0:
                th[:, :, k] += 0.1 * rng.uniform(-1.0, 1.0, (nx, ny))
        # u = v = 0 everywhere would make the near-surface wind speed zero and
        # the reference's wall boundary value 0/0 (src/operations/
        # Derivatives.py:224-229); like the reference's own CBL generator
        # (examples/CBL_N91/runs/*/CreateInputs_CBL_N91.py) seed 0.03 m/s
        # noise into u and w below 200 m.
        for k in range(nz):
            if z[k] <= 200.0:
                r = 0.03 * rng.standard_normal((nx, ny))
                u[:, :, k] += r
                w[:, :, k] += r
    elif case == "stable":
        u[:] = cfg["Ug2"]
        prof = np.where(z <= 100.0, 265.0, 265.0 + 0.01 * (z - 100.0))
        th[:] = prof[None, None, :]
        for k in range(nz):
            if z[k] < 50.0:
                th[:, :, k] += 0.1 * rng.uniform(-1.0, 1.0, (nx, ny))
    else:
        raise ValueError(case)
    return u, v, w, th


def initial_moisture(cfg, seed=0):
    """Initial specific humidity (kg/kg, absolute; ``Initialize_Q``), (nx,
    ny, nz) C-order: 8 g/kg at the surface drying by 2 g/kg over the domain
    depth, with 0.1 g/kg seeded noise in the lower third."""
    nx, ny, nz = cfg["nx"], cfg["ny"], cfg["nz"]
    z = z_uvp(cfg)
    rng = np.random.default_rng(1000 + seed)
    q = np.empty((nx, ny, nz))
    q[:] = (8.0e-3 - 2.0e-3 * z / cfg["l_z"])[None, None, :]
    for k in range(nz):
        if z[k] < cfg["l_z"] / 3:
            q[:, :, k] += 1.0e-4 * rng.uniform(-1.0, 1.0, (nx, ny))
    return q


def moisture_surface_series(cfg):
    """The moisture surface series at every step (``Initialization.py:
    344-388`` format): for ``optMoistureSurfBC=1`` a flux (kg/kg m/s)
    oscillating about MoistureFlux, for ``=2`` the surface humidity (kg/kg)
    near 10 g/kg."""
    n = nsteps_of(cfg) + 1
    ph = 2 * np.pi * np.arange(n) / 5.0
    if cfg["optMoistureSurfBC"] == 1:
        return cfg["MoistureFlux"] + 2.0e-5 * np.sin(ph)
    return 1.0e-2 + 5.0e-4 * np.sin(ph)


def adv_moisture_series(cfg):
    """Qadv (kg/kg s^-1) at every step and level for the AdvForcing file."""
    n = nsteps_of(cfg) + 1
    zh = (np.arange(cfg["nz"]) + 0.5) / cfg["nz"]
    return np.broadcast_to(-2.0e-8 * (1.0 - zh)[None, :], (n, cfg["nz"])).copy()


def surface_bc_series(cfg):
    """Surface boundary series at every step, t=0..SimTime, in the
    ``Initialization.py:107-160`` format: for ``optSurfBC=2`` the surface
    temperature (K), cooling linearly at 0.5 K/h from 265 K; for
    ``optSurfBC=1`` a heat flux (K m/s) oscillating about the case's
    SensibleHeatFlux."""
    n = nsteps_of(cfg) + 1
    t = np.arange(n) * cfg["dt"]
    if cfg["optSurfBC"] == 1:
        return cfg["SensibleHeatFlux"] + 0.02 * np.sin(2 * np.pi * t / 3600.0)
    return 265.0 - 0.5 * t / 3600.0


def adv_forcing_series(cfg):
    """(Uadv, Vadv, THadv) in m s^-2 / K s^-1 at every step and level
    (``Initialization.py:253-323`` format)."""
    n = nsteps_of(cfg) + 1
    nz = cfg["nz"]
    U = np.full((n, nz), cfg.get("Uadv_const", 0.0))
    return U, np.zeros((n, nz)), np.zeros((n, nz))


def geowind_series(cfg):
    """Time- and height-varying geostrophic wind (Ug, Vg) in m/s at every
    step and level, (nsteps+1, nz) each (``Initialization.py:173-246``
    per-step format): a height shear about (Ug2, Vg2) plus an oscillation
    with a period of seven steps, so every step's row differs."""
    n = nsteps_of(cfg) + 1
    nz = cfg["nz"]
    zh = (np.arange(nz) + 0.5) / nz
    ph = 2 * np.pi * np.arange(n)[:, None] / 7.0
    Ug = cfg["Ug2"] + 1.5 * zh[None, :] + 0.8 * np.sin(ph) * (1.0 - zh[None, :])
    Vg = cfg["Vg2"] - 0.6 * zh[None, :] + 0.5 * np.cos(ph) * zh[None, :]
    return Ug, Vg


def to_reference_files(cfg, u, v, w, th):
    """Arrays in the layout of the reference's ``vel.npy`` / ``TH.npy``."""
    vel = np.column_stack([u.reshape(-1, order="F"), v.reshape(-1, order="F"),
                           w.reshape(-1, order="F")])
    return vel, th.reshape(-1, order="F")


def config_py_text(cfg):
    """A ``Config.py`` for the reference holding this case's options."""
    lines = ["import numpy as np"]
    skip = {"case", "Uadv_const"}
    for k, v in cfg.items():
        if k in skip:
            continue
        lines.append(f"{k} = {v!r}")
    return "\n".join(lines) + "\n"


def write_run_dir(cfg, path, seed=0):
    """Write ``Config.py`` and ``input/`` files the reference's Main.py loads."""
    import os
    os.makedirs(os.path.join(path, "input"), exist_ok=True)
    with open(os.path.join(path, "Config.py"), "w") as f:
        f.write(config_py_text(cfg))
    u, v, w, th = initial_fields(cfg, seed)
    vel, thf = to_reference_files(cfg, u, v, w, th)
    np.save(os.path.join(path, "input", "vel.npy"), vel)
    np.save(os.path.join(path, "input", "TH.npy"), thf)
    if cfg["optSurfBC"] >= 1:
        np.savez(os.path.join(path, cfg["SurfaceBCFile"]), dt_surf=cfg["dt"],
                 optSurfBC=np.int32(cfg["optSurfBC"]), data_series=surface_bc_series(cfg))
    moist = cfg.get("optMoisture", 0) >= 1
    if moist:
        q = initial_moisture(cfg, seed)
        np.save(os.path.join(path, "input", "Q.npy"), q.reshape(-1, order="F"))
        if cfg["optMoistureSurfBC"] >= 1:
            np.savez(os.path.join(path, cfg["MoistureSurfaceBCFile"]), dt_moist=cfg["dt"],
                     optMoistureSurfBC=np.int32(cfg["optMoistureSurfBC"]),
                     data_series=moisture_surface_series(cfg))
    if cfg.get("optGeoWind", 0) >= 1:
        Ug, Vg = geowind_series(cfg)
        np.savez(os.path.join(path, cfg["GeoWindFile"]), dt_geo=cfg["dt"],
                 optGeoWind=np.int32(cfg["optGeoWind"]), Ug_series=Ug, Vg_series=Vg)
    if cfg["optAdvection"] >= 1:
        U, V, T = adv_forcing_series(cfg)
        extra = {"Qadv_series": adv_moisture_series(cfg)} if moist else {}
        np.savez(os.path.join(path, cfg["AdvectionFile"]), dt_adv=cfg["dt"],
                 optAdvection=np.int32(cfg["optAdvection"]),
                 Uadv_series=U, Vadv_series=V, THadv_series=T, **extra)


def gp_per_step(cfg):
    return cfg["nx"] * cfg["ny"] * cfg["nz"]


__all__ = ["CASES", "neutral", "nbl_a94", "convective", "stable",
           "initial_fields", "write_run_dir", "nsteps_of", "surface_bc_series",
           "adv_forcing_series", "geowind_series", "initial_moisture",
           "moisture_surface_series", "adv_moisture_series", "gp_per_step"]
