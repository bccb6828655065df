"""Known-answer vectors for the statistics accumulator, produced by the
reference's own ``ComputeStats`` / ``InitializeStats``
(``src/utilities/Statistics.py:47-380``) on the NumPy stand-in for ``jax``
(see ``make_golden.py``), for seeded synthetic inputs of the stable case's
configuration (Galilean velocity Ugal = 5 m/s), moisture entries included:

  ``in<s>.<name>``  inputs of sample s = 1, 2 (fields, planes, profiles);
  ``acc<s>.<key>``  the statistics dictionary after accumulating samples
                    1..s from ``InitializeStats``;
  ``reset.<key>``   the dictionary after a call with ResetFlag = 1.

Usage:  python tests/golden/make_golden_stats.py --out tests/golden/ref_stats.npz
"""
import argparse
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
# the reference checkout: --reference DIR, else $ALFA_REFERENCE_DIR (no default)
REFERENCE = os.environ.get("ALFA_REFERENCE_DIR")

GRID = (12, 16, 8)
FIELDS = ("u", "v", "w", "TH", "dudz", "dvdz", "dTHdz", "txy", "txz", "tyz", "qz",
          "Q", "dQdz", "qHz_q")
PLANES = ("M_sfc_loc", "ustar")
PROFILES = ("Cs2_1D_avg1", "Cs2_1D_avg2", "Cs2PrRatio_1D", "beta1_1D", "beta2_1D")


def sample_inputs(rng, nx, ny, nz):
    d = {k: rng.standard_normal((nx, ny, nz)) for k in FIELDS}
    d["TH"] = 0.5 * d["TH"] + np.linspace(0.0, 3.0, nz)   # anomaly with a mean profile
    d["u"] = d["u"] + 2.0
    d["Q"] = 8.0e-3 + 1.0e-4 * d["Q"] - 1.0e-4 * np.linspace(0.0, 1.0, nz)  # specific humidity
    d["dQdz"] = 1.0e-5 * d["dQdz"]
    d["qHz_q"] = 1.0e-5 * d["qHz_q"]
    for k in PLANES:
        d[k] = 0.2 + rng.random((nx, ny))
    for k in PROFILES:
        d[k] = rng.random(nz)
    d["qz_sfc_avg"] = np.array(rng.standard_normal() * 1e-3)
    d["qm_sfc_avg"] = np.array(rng.standard_normal() * 1e-5)
    return d


def main():
    global REFERENCE
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--reference", default=REFERENCE,
                    help="the JAX-ALFA checkout (default: $ALFA_REFERENCE_DIR)")
    a = ap.parse_args()
    if not a.reference or not os.path.isdir(os.path.join(a.reference, "src")):
        ap.error("give the JAX-ALFA checkout with --reference DIR or ALFA_REFERENCE_DIR")
    REFERENCE = a.reference
    sys.path.insert(0, os.path.join(HERE, "jaxshim"))
    sys.path.insert(0, REFERENCE)
    sys.path.insert(0, REPO)
    from jax_alfa_b200 import cases
    rundir = tempfile.mkdtemp(prefix="alfa_stats_")
    cases.write_run_dir(cases.stable(*GRID, nsteps=1), rundir)
    os.environ["JAXALFA_RUNDIR"] = rundir
    import jax.numpy as jnp
    from src.utilities.Statistics import ComputeStats, InitializeStats

    nx, ny, nz = GRID
    zero3 = jnp.zeros((nx, ny, nz))
    stats = InitializeStats(jnp.zeros(nz))
    rng = np.random.default_rng(2024)
    out = {}

    def call(d, stats, reset):
        return ComputeStats(d["u"], d["v"], d["w"], d["TH"], d["Q"],
                            d["dudz"], d["dvdz"], d["dTHdz"], d["dQdz"],
                            d["M_sfc_loc"], d["ustar"], float(d["qz_sfc_avg"]),
                            float(d["qm_sfc_avg"]),
                            d["txy"], d["txz"], d["tyz"], d["qz"], d["qHz_q"],
                            d["Cs2_1D_avg1"], d["Cs2_1D_avg2"], d["Cs2PrRatio_1D"],
                            d["beta1_1D"], d["beta2_1D"], stats, reset, zero3)

    for s in (1, 2):
        d = sample_inputs(rng, nx, ny, nz)
        for k, v in d.items():
            out[f"in{s}.{k}"] = np.asarray(v)
        stats = call(d, stats, 0)
        for k, v in stats.items():
            out[f"acc{s}.{k}"] = np.asarray(v)
    stats = call(d, stats, 1)
    for k, v in stats.items():
        out[f"reset.{k}"] = np.asarray(v)
    np.savez_compressed(a.out, **out)
    print(f"wrote {a.out}: {len(out)} arrays")


if __name__ == "__main__":
    main()
