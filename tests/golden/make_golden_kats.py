"""Known-answer vectors for the root finder and beta selection, produced by
the reference's own functions on the NumPy stand-in for ``jax`` (see
``make_golden.py``):

  * ``Roots`` (``src/utilities/Utilities.py:123-241``) on the polynomials the
    reference's scratch test uses (``src/utilities/TEST_Root.py:164-170``)
    and on 64 seeded random quintics from each of the 8 beta guesses;
  * ``ComputeBeta1`` / ``ComputeBeta2`` (``DynamicSGS_LASDD_SM.py:53-95``,
    ``DynamicSGS_ScalarLASDD_SM.py:54-96``) on 64 seeded coefficient sets;
  * ``Imfilter`` (``Utilities.py:87-115``) on a seeded 12x10 plane.

Usage:  python tests/golden/make_golden_kats.py --out tests/golden/ref_kats.npz
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

TEST_ROOT_CASES = [([1.0, 0.0, -4.0], 1.0), ([1.0, 0.0, 0.0, -1.0], 0.5),
                   ([1.0, -3.0], 1.0), ([0.1, 0.3, 0.6, 0.1, 2.0, 1.0], 1.0)]
GUESSES = [0.5, 0.75, 1.0, 1.25, 1.5, 2.0, 3.0, 4.5]


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
    rundir = tempfile.mkdtemp(prefix="alfa_kats_")
    cases.write_run_dir(cases.neutral(8, 8, 8, nsteps=1), rundir)
    os.environ["JAXALFA_RUNDIR"] = rundir
    import jax.numpy as jnp
    from src.utilities.Utilities import Roots, Imfilter
    from src.subgridscale.DynamicSGS_LASDD_SM import ComputeBeta1
    from src.subgridscale.DynamicSGS_ScalarLASDD_SM import ComputeBeta2

    out = {}
    for i, (c, g) in enumerate(TEST_ROOT_CASES):
        out[f"testroot{i}.coeffs"] = np.array(c)
        out[f"testroot{i}.guess"] = np.array(g)
        out[f"testroot{i}.root"] = np.asarray(Roots(jnp.array(c), init_guess=g))
    rng = np.random.default_rng(1234)
    quint = rng.standard_normal((64, 6))
    quint[:16] *= np.array([1e-3, 1e-2, 1.0, 1.0, 1.0, 1.0])   # near-degenerate leading terms
    roots = np.array([[np.asarray(Roots(jnp.array(q), init_guess=g)) for g in GUESSES] for q in quint])
    out["quintic.coeffs"] = quint
    out["quintic.roots"] = roots
    coef = rng.standard_normal((6, 64))
    out["beta.coeffs"] = coef
    out["beta1"] = np.asarray(ComputeBeta1(*[jnp.array(x) for x in coef]))
    out["beta2"] = np.asarray(ComputeBeta2(*[jnp.array(x) for x in coef]))
    plane = rng.standard_normal((12, 10))
    out["imfilter.in"] = plane
    out["imfilter.out"] = np.asarray(Imfilter(jnp.array(plane)))
    np.savez_compressed(a.out, **out)
    print(f"wrote {a.out}")


if __name__ == "__main__":
    main()
