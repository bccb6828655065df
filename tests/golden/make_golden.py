"""Generate golden vectors by executing the JAX-ALFA reference's own sources.

JAX is not installed in this image, so the reference's ``src/Main.py`` runs
here on the NumPy-backed stand-in for ``jax`` in ``tests/golden/jaxshim``.
Everything else is the reference's code, unmodified and read in place from
the reference checkout: its config loader, initialisation, the full step
loop of ``src/Main.py:156-541`` and every hot-path function it calls.

Two stub modules stand in for ``src/pde/NSE_SGSTerms_STABSM.py`` and
``src/pde/SCL_SGSTerms_STABSM.py``; the reference's ``.gitignore:2-6``
excludes them from its repository but ``src/config/Imports.py:140-141``
imports them unconditionally.  They are only called when optSgs == 5, which
no case here uses.

While ``Main.py`` runs, the hot-path functions it calls are wrapped ("tapped")
so that their inputs and outputs at selected iterations are recorded.  The
result is one ``.npz`` per case:
  ``<fn>.<call>.in<i>[.<j>]`` / ``<fn>.<call>.out<i>[.<j>]`` arrays for every
  tapped call made during the recorded iterations, ``<call>`` counting that
  function's calls from the start of the run;
  ``final.<name>`` for the model state after the last step.

Usage (from the repository root; the reference checkout is given by --reference or
$ALFA_REFERENCE_DIR):
    python tests/golden/make_golden.py --case neutral --grid 16 16 12 \
        --steps 2 --record 1 2 --out tests/golden/ref_neutral_16x16x12.npz
"""
import argparse
import os
import runpy
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
# the reference checkout: --reference DIR, else $ALFA_REFERENCE_DIR (no default)
REFERENCE = os.environ.get("ALFA_REFERENCE_DIR")

TAPPED = {
    "src.operations.Filtering": ["Filtering_Explicit"],
    "src.surface.SurfaceFlux": [
        "SurfaceFlux_HomogeneousConstantFlux", "SurfaceFlux_HeterogeneousConstantFlux",
        "SurfaceFlux_HomogeneousVaryingFlux", "SurfaceFlux_HeterogeneousVaryingFlux",
        "SurfaceFlux_HomogeneousPrescribedTemperature",
        "SurfaceFlux_HeterogeneousPrescribedTemperature",
        "SurfaceMoistureFlux_HomogeneousPrescribedQ",
        "SurfaceMoistureFlux_HeterogeneousPrescribedQ"],
    "src.operations.Derivatives": ["velocityGradients", "potentialTemperatureGradients",
                                   "moistureGradients"],
    "src.pde.NSE_AdvectionTerms": ["Advection"],
    "src.pde.SCL_AdvectionTerms": ["ScalarAdvection"],
    "src.pde.NSE_BuoyancyTerms": ["BuoyancyOpt1", "BuoyancyOpt2"],
    "src.pde.NSE_SGSTerms": ["DivStressDynamicSGS", "DivStressStaticSGS"],
    "src.pde.SCL_SGSTerms": ["DivFluxDynamicSGS", "DivFluxStaticSGS"],
    "src.pde.NSE_AllTerms": ["RHS_Momentum"],
    "src.pde.SCL_AllTerms": ["RHS_Scalar", "RHS_Moisture"],
    "src.pde.NSE_PressureTerms": ["PressureRC", "PressureSolve"],
    "src.pde.NSE_PressureTerms_Thomas": ["ThomasPressureSolve"],
    "src.pde.NSE_TimeAdvancement": ["AB2_uvw"],
    "src.pde.SCL_TimeAdvancement": ["AB2_TH", "AB2_Q"],
}

FINAL_NAMES = ["u", "v", "w", "TH", "Q", "p", "dpdx", "dpdy", "dpdz",
               "RHS_u", "RHS_v", "RHS_w", "RHS_TH", "Cs2_3D", "Cs2PrRatio_3D",
               "beta1_1D", "beta2_1D", "Cs2_1D_avg1", "Cs2_1D_avg2", "Cs2PrRatio_1D",
               "ustar", "M_sfc_loc", "qz_sfc_avg", "psi2D_m", "psi2D_m0",
               "MOSTfunctions"]


def _flatten(prefix, obj, out):
    if isinstance(obj, (tuple, list)):
        for j, e in enumerate(obj):
            _flatten(f"{prefix}.{j}", e, out)
    elif obj is None:
        return
    else:
        a = np.asarray(obj)
        if a.dtype.kind in "fcib":
            out[prefix] = np.array(a)


def run(case, grid, steps, record, out_path, seed, overrides, final_names=FINAL_NAMES):
    sys.path.insert(0, os.path.join(HERE, "jaxshim"))
    sys.path.insert(0, REFERENCE)
    sys.path.insert(0, REPO)
    from jax_alfa_b200 import cases

    nx, ny, nz = grid
    cfg = cases.CASES[case](nx, ny, nz, nsteps=steps, **overrides)
    rundir = tempfile.mkdtemp(prefix="alfa_golden_")
    cases.write_run_dir(cfg, rundir, seed=seed)
    os.environ["JAXALFA_RUNDIR"] = rundir

    for name, fn in (("src.pde.NSE_SGSTerms_STABSM", "DivStressStaticSGS_STABSM"),
                     ("src.pde.SCL_SGSTerms_STABSM", "DivFluxStaticSGS_STABSM")):
        mod = types.ModuleType(name)

        def _unavailable(*a, **k):
            raise RuntimeError("STAB-SM sources are not part of the reference repository")
        setattr(mod, fn, _unavailable)
        sys.modules[name] = mod

    import importlib
    state = {"iteration": 1}
    # the last state update of an iteration (Main.py:522-528)
    last_update = "AB2_Q" if int(cfg.get("optMoisture", 0)) >= 1 else "AB2_TH"
    calls = {}
    rec = {}

    def tap(fname, f):
        def wrapped(*args, **kwargs):
            res = f(*args, **kwargs)
            c = calls.get(fname, 0)
            calls[fname] = c + 1
            if state["iteration"] in record:
                d = {}
                for i, a in enumerate(args):
                    _flatten(f"{fname}.{c}.in{i}", a, d)
                _flatten(f"{fname}.{c}.out", res if isinstance(res, tuple) else (res,), d)
                rec.update({k.replace(".out.", ".out"): v for k, v in d.items()})
                rec[f"{fname}.{c}.iteration"] = np.array(state["iteration"])
            if fname == last_update:
                state["iteration"] += 1
            return res
        return wrapped

    for modname, fns in TAPPED.items():
        mod = importlib.import_module(modname)
        for fn in fns:
            setattr(mod, fn, tap(fn, getattr(mod, fn)))

    g = runpy.run_module("src.Main", run_name="src.Main")
    for name in final_names:
        if name in g:
            _flatten(f"final.{name}", g[name], rec)
    rec["meta.steps"] = np.array(steps)
    rec["meta.grid"] = np.array(grid)
    rec["meta.seed"] = np.array(seed)
    rec["meta.case"] = np.array(case)
    rec["meta.overrides"] = np.array(repr(sorted(overrides.items())))
    # Many recorded arguments repeat (the same field passed to several
    # functions, zero buffers, broadcast wavenumbers): store each distinct
    # array once and an index from key to blob.
    import hashlib
    import json
    blobs, index, seen = {}, {}, {}
    for k, v in rec.items():
        v = np.array(v, order="C")
        h = hashlib.sha1(v.tobytes() + str((v.shape, v.dtype.str)).encode()).hexdigest()
        if h not in seen:
            seen[h] = f"blob{len(seen)}"
            blobs[seen[h]] = v
        index[k] = seen[h]
    blobs["index"] = np.array(json.dumps(index))
    np.savez_compressed(out_path, **blobs)
    print(f"wrote {out_path}: {len(rec)} keys, {len(seen)} distinct arrays, "
          f"{sum(v.nbytes for v in blobs.values()) / 1e6:.2f} MB uncompressed")


def main():
    global REFERENCE
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default="neutral")
    ap.add_argument("--grid", type=int, nargs=3, default=[16, 16, 12])
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--record", type=int, nargs="*", default=[1, 2])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--set", nargs="*", default=[],
                    help="config overrides key=value (Python literals)")
    ap.add_argument("--final", nargs="*", default=FINAL_NAMES,
                    help="model-state names kept after the last step")
    ap.add_argument("--out", required=True)
    ap.add_argument("--reference", default=REFERENCE,
                    help="the JAX-ALFA checkout (default: $ALFA_REFERENCE_DIR)")
    a = ap.parse_args()
    if not a.reference or not os.path.isdir(os.path.join(a.reference, "src")):
        ap.error("give the JAX-ALFA checkout with --reference DIR or ALFA_REFERENCE_DIR")
    REFERENCE = a.reference
    import ast
    over = {}
    for kv in a.set:
        k, v = kv.split("=", 1)
        over[k] = ast.literal_eval(v)
    run(a.case, a.grid, a.steps, set(a.record), a.out, a.seed, over, a.final)


if __name__ == "__main__":
    main()
