"""A few whole steps of the NBL_A94 workload (the reference's neutral
boundary-layer benchmark case) for profilers: the bootstrap step, then graph
steps, nothing else on the device.  The kernel launch lists and ncu captures
under profiles/ name this command.

    python -m jax_alfa_b200.profile_step --precision mixed --grid 256 256 256 --steps 3 \
        --variant two-lane
"""
import argparse
import sys


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--precision", default="mixed", choices=["fp64", "fp32", "mixed"])
    ap.add_argument("--grid", type=int, nargs=3, default=[256, 256, 256])
    ap.add_argument("--steps", type=int, default=3, help="graph steps after the bootstrap step")
    ap.add_argument("--tune", action="store_true", help="run the line-pass autotuner first")
    ap.add_argument("--learned", action="store_true",
                    help="instead: the convective case at --grid in FP64, one dynamic step, a "
                         "network trained one epoch on it, then two learned steps (the "
                         "tensor-core inference of alfa_step_learned)")
    ap.add_argument("--variant", default=None,
                    help="set this line-pass variant (a TUNE_VARIANTS name) on every pass "
                         "shape that takes it, without timing")
    args = ap.parse_args(argv)
    import torch

    from jax_alfa_b200 import cases
    from jax_alfa_b200.api import Learned, Simulation
    if args.learned:
        cfg = cases.convective(*args.grid, nsteps=8)
        u, v, w, th = cases.initial_fields(cfg, 0)
        sim = Simulation(cfg, u, v, w, th)
        sim.step(1)
        net = Learned(sim, capacity=8192, seed=1)
        net.collect(8192)
        net.train(epochs=1, batch=1024, lr=1e-3)
        rep = net.step(2, judge_every=1000, tol=1e9)
        torch.cuda.synchronize()
        print("ok", rep, flush=True)
        return 0
    cfg = cases.nbl_a94(*args.grid, nsteps=args.steps + 2, precision=args.precision)
    u, v, w, th = cases.initial_fields(cfg, 0)
    sim = Simulation(cfg, u, v, w, th)
    sim.step(1)
    if args.variant:
        from jax_alfa_b200._lib import AlfaError
        for shape in sim.alfa.tune_shapes():
            try:
                sim.set_line_variant(shape, args.variant)
                print(f"{shape['shape']}: {args.variant}")
            except AlfaError:
                print(f"{shape['shape']}: default ({args.variant} does not apply)")
    if args.tune:
        for c in sim.autotune(reps=3):
            if c["chosen"]:
                print(f"{c['shape']}: {c['variant']} {c['ms']:.4f} ms")
    sim.step(args.steps, graph=True)
    torch.cuda.synchronize()
    print("ok", sim.diag(), flush=True)


if __name__ == "__main__":
    sys.exit(main())
