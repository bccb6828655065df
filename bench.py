"""Throughput of the LES step on B200: grid-point-steps per second.

Workload: the reference's own neutral-boundary-layer benchmark (NBL_A94,
Andren et al. 1994) at 256^3: a neutral Ekman layer under a 5 m/s
geostrophic wind in a 4000 m cube, Ugal = 3 m/s, LASDD-SM dynamic SGS every
step, 3/2-rule dealiasing, Thomas pressure solve, AB2 at dt = 0.75 s
(examples/NBL_A94/runs/256x256x256_LASDD_SM_DP/Config.py, the configuration
of the reference's A100 figures).  Seeded synthetic initial fields of that
case's form (u = 5 m/s, theta = 300 K, Gaussian noise below 200 m).  Every
field (4 or 8 B x 16.8 M points) is larger than L2 (126 MB), so no flush is
needed between steps.

The metric compares the mixed-precision step with the plain FP64 drop-in on
the same GPU:
  value   : the mixed-precision step (FP32 fields and transforms, split-BF16
            tensor-core line passes where the autotuner measures them faster,
            FP64 pressure tridiagonal solve, zero mode, plane means, beta
            roots and surface layer), device-timed CUDA-graph steps with the
            state resident in HBM, CUDA events on the launching stream, max
            over ranks;
  fp64    : the same for the FP64 drop-in, with the speed-up of the mixed
            step over it and the mixed state's error against the FP64 state
            after the same steps from the same initial fields;
  e2e     : the mixed step through the whole-step C-ABI with the state from
            and to pinned host memory and the CFL diagnostics read back every
            step, all inside the timed region;
  cpu_baseline / --impl reference : the reference's algorithm on the host
            (the NumPy FP64 port of it, scipy.fft on every host thread) on
            the same 256^3 workload, a bounded number of steps.

Multi-GPU: ``replicas only`` -- each rank advances its own independent
simulation (no data-path collective); scaling is weak.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# the reference's A100 JAX figures for NBL_A94 256^3 LASDD-SM
A100_FP64 = 93.4e6   # gp-steps/s, FP64
A100_FP32 = 166.8e6  # gp-steps/s, FP32
METRIC = "LES grid-point-steps/s at 256^3: mixed-prec vs plain FP64 on B200, err vs FP64"
DTYPES = {"mixed": "f32 fields + split-bf16 tensor-core line passes + f64 solves/means",
          "fp32": "f32 fields + f64 solves/means", "fp64": "f64"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default 20; 500 with --ensemble)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="alfa", choices=["alfa", "reference"])
    ap.add_argument("--grid", type=int, nargs=3, default=[256, 256, 256])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp32", "fp64"],
                    help="the form timed as the headline value")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 comparison run")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=60.0,
                    help="seconds of host time for the cpu_baseline sample")
    ap.add_argument("--epochs", type=int, default=40,
                    help="training epochs of the learned closure (--learned)")
    ap.add_argument("--no-tune", action="store_true",
                    help="skip the line-pass autotuner (default dispatch)")
    ap.add_argument("--learned", action="store_true",
                    help="the learned SGS coefficient on the 192x192x128 convective case: "
                         "train on the dynamic procedure, then time and compare learned, "
                         "dynamic and fixed-coefficient steps")
    ap.add_argument("--ensemble", action="store_true",
                    help="time the 64-member uneven ensemble (32x32^3, 16x48^3, 16x64^3) "
                         "against its members stepped one at a time")
    ap.add_argument("--no-ensemble", action="store_true",
                    help="skip the short ensemble run of the default line")
    ap.add_argument("--no-workloads", action="store_true",
                    help="skip the convective 128^3 and stable 256x256x192 runs of the "
                         "default line")
    ap.add_argument("--ens-precision", default="fp32", choices=["fp32", "fp64"],
                    help="storage precision of the ensemble members")
    ap.add_argument("--spinup", type=int, default=3000,
                    help="dynamic steps before the learned closure collects samples")
    args = ap.parse_args()
    if args.steps is None:
        args.steps = 500 if args.ensemble else (200 if args.learned else 20)
    return args


def workload_config(grid, nsteps, precision="fp64"):
    from jax_alfa_b200 import cases
    return cases.nbl_a94(*grid, nsteps=nsteps, precision=precision)


def config_block(grid, world, precision):
    return {"workload": f"NBL_A94 neutral Ekman layer {grid[0]}x{grid[1]}x{grid[2]} (the "
                        "reference's 256^3 benchmark case), LASDD-SM dynamic SGS, 3/2-rule "
                        "dealiasing, Thomas pressure, AB2, dt 0.75 s",
            "grid": list(grid), "sgs": "LASDD-SM (optSgs=1, dynamic every step)",
            "precision": precision, "l2": "every field exceeds L2 (126 MB); no flush",
            "step": "one CUDA graph replay per step (alfa_step_graph)",
            "parallelism": f"replicas x{world} (no sharding)",
            "baseline": "A100 JAX NBL_A94 256^3 LASDD-SM: FP32 166.8 M, FP64 93.4 M gp-steps/s"}


def cpu_info():
    """Host threads and the CPU model (lscpu)."""
    model = None
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
        for ln in out.splitlines():
            if ln.startswith("Model name:"):
                model = ln.split(":", 1)[1].strip()
                break
    except (OSError, subprocess.SubprocessError):
        pass
    return os.cpu_count() or 1, model


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.idx)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def measured_bf16_peak():
    """Dense BF16 TFLOP/s (burst) from MEASURED_PEAKS.json, else the
    fallback figure of this pool."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        if "bf16_tflops" in d:
            return float(d["bf16_tflops"]), "measured"
    return 1590.0, "fallback"


def ncu_traffic():
    """DRAM bytes per launch of the dominant kernel from the committed ncu
    summary (profiles/), or None."""
    p = os.path.join(ROOT, "profiles", "dominant_kernel_traffic.txt")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        for ln in f:
            if ln.startswith("{"):
                return json.loads(ln)
    return None


def oracle_steps(grid, threads, warmup, steps, budget_s):
    """The NumPy FP64 port of the reference's step on the host: `warmup`
    untimed steps, then timed steps until `steps` are done or the next one
    would pass `budget_s` seconds.  Returns (timed steps, seconds)."""
    from jax_alfa_b200 import cases
    from oracle import alfa_oracle
    from oracle.alfa_oracle import OracleRun
    alfa_oracle.set_fft_workers(threads)
    cfg = workload_config(grid, warmup + steps + 1)
    u, v, w, th = cases.initial_fields(cfg, 0)
    r = OracleRun(cfg, u, v, w, th)  # no forcing series: NBL_A94 has none
    with np.errstate(all="ignore"):
        for _ in range(warmup):
            r.step()
        n, t0 = 0, time.perf_counter()
        while n < steps:
            r.step()
            n += 1
            el = time.perf_counter() - t0
            if el * (n + 1) / n > budget_s:
                break
    return n, time.perf_counter() - t0


def rank_max(x, dist, device=None):
    """The largest of x over the ranks of the process group (x itself when
    there is none): the device time of a replicated step is the slowest
    rank's."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_seed(rank):
    """Each rank's replica starts from its own seeded initial fields."""
    return rank


def run_reference(args, rank, world):
    if rank != 0:  # the host arm runs once, on rank 0; the other ranks do no work
        return
    threads, model = cpu_info()
    grid = tuple(args.grid)
    # one warm-up step (the first step allocates the port's temporaries), then
    # as many of the requested steps as fit in about 150 s of host time
    n, dt = oracle_steps(grid, threads, 1, args.steps, 150.0)
    npts = grid[0] * grid[1] * grid[2]
    value = npts * n / dt
    sample = (f"{n} of the {args.steps} requested steps (after 1 warm-up step) of the same "
              f"{grid[0]}x{grid[1]}x{grid[2]} workload, {dt / n:.2f} s/step: NumPy FP64 port of "
              f"the reference's step with scipy.fft on {threads} host threads ({model})")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "gp-steps/s",
        "n_gpus": world, "steps": n, "warmup": 1, "steps_requested": args.steps,
        "ms_per_step": 1e3 * dt / n, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_block(grid, world, "FP64 reference algorithm on the host"),
        "cpu_baseline": {"value": value, "unit": "gp-steps/s", "cores": threads,
                         "cpu_model": model, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "gp-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


def run_alfa(args, rank, world, dist):
    import ctypes

    import torch
    from jax_alfa_b200 import _lib, cases
    from jax_alfa_b200.api import Simulation, stats_to_dict

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    grid = tuple(args.grid)
    n_gp = grid[0] * grid[1] * grid[2]
    total = args.warmup + args.steps + 2
    u, v, w, th = cases.initial_fields(workload_config(grid, total), replica_seed(rank))
    lib = _lib.load()
    stream = torch.cuda.current_stream(dev)

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        return rank_max(x, dist, dev)

    def timed(prec, keep=False):
        """Warm-up (the bootstrap step, the line-pass autotuner, graph
        captures of both iteration parities), then args.steps graph steps
        timed with CUDA events on this stream, clocks sampled meanwhile."""
        sim = Simulation(workload_config(grid, total, prec), u, v, w, th)
        sim.step(1)
        tune = sim.autotune(reps=3) if not args.no_tune else []
        sim.step(max(args.warmup - 1, 2), graph=True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        clocks = ClockSampler(local)
        torch.cuda.synchronize(dev)
        barrier()
        torch.cuda.synchronize(dev)
        clocks.start()
        n0 = lib.alfa_launch_count()
        e0.record(stream)
        sim.step(args.steps, graph=True)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        n1 = lib.alfa_launch_count()
        barrier()
        torch.cuda.synchronize(dev)
        clk = clocks.stop()
        ms = max_over_ranks(e0.elapsed_time(e1))
        if not np.isfinite(sim.diag()["CFL"]):
            raise RuntimeError(f"non-finite state in the timed {prec} run")
        st = {k: t.cpu().numpy() for k, t in sim.state().items()}
        # the beta profiles of the last step (the dynamic procedure's quintic roots)
        prof = stats_to_dict(sim.stats_sample(None), grid[2], sim.alfa.cfg["Ugal"])
        st["beta"] = np.stack([prof["Beta1"], prof["Beta2"]])
        out = {"ms": ms, "tune": tune, "launches": int(n1 - n0), "clocks": clk, "state": st}
        if keep:
            out["sim"] = sim
        else:
            del sim
            torch.cuda.empty_cache()
        return out

    head = timed(args.precision, keep=True)
    sim = head["sim"]
    ms = head["ms"]
    value = n_gp * args.steps * world / (ms / 1e3)
    fp64 = None
    if args.precision != "fp64" and not args.no_fp64:
        sim_keep = sim
        ref = timed("fp64")
        st, rs = head["state"], ref["state"]
        vmax = max(float(np.abs(rs[k]).max()) for k in ("u", "v", "w"))
        err = {k: float(np.abs(st[k] - rs[k]).max()) / vmax for k in ("u", "v", "w")}
        for k in ("TH", "p"):
            err[k] = float(np.abs(st[k] - rs[k]).max()) / max(float(np.abs(rs[k]).max()), 1e-300)
        # the same per level: the median over levels shows the round-off floor,
        # the maximum the levels where the beta root selection went the other way
        lev = np.max(np.stack([np.abs(st[k] - rs[k]).max(axis=(0, 1)) for k in ("u", "v", "w")]),
                     axis=0) / vmax
        beta_flips = int(np.sum(np.any(np.abs(st["beta"] - rs["beta"]) > 0.1, axis=0)))
        fp64 = {"value": n_gp * args.steps * world / (ref["ms"] / 1e3),
                "ms_per_step": ref["ms"] / args.steps,
                "speedup": ref["ms"] / ms,
                "vs_a100_fp64": n_gp * args.steps * world / (ref["ms"] / 1e3) / A100_FP64,
                "err_vs_fp64": err,
                "velocity_err_per_level": {"median": float(np.median(lev)),
                                           "max": float(lev.max()),
                                           "worst_level": int(np.argmax(lev))},
                "levels_with_other_beta_root": beta_flips,
                "err_definition": (f"max |x - x_fp64| after {1 + max(args.warmup - 1, 2) + args.steps} "
                                   "steps from the same initial fields: u, v, w relative to the "
                                   "largest FP64 velocity component, TH and p relative to their "
                                   "own largest FP64 value (TH is theta - T_0)"),
                "gpu_launches": ref["launches"], "clocks": ref["clocks"]}
        sim = sim_keep
    del head["state"]
    clk_head, launches_head, tune_head = head["clocks"], head["launches"], head["tune"]

    # ---- dominant kernel and the other line passes, live ------------------
    roof = None
    peak, peak_kind = measured_peaks()
    t_ms, t_bytes = ctypes.c_double(), ctypes.c_double()
    a = sim.alfa
    a.lib.alfa_set_stream(a.ctx, ctypes.c_void_p(stream.cuda_stream))
    nx_, ny_, nz_ = grid
    names = {0: f"k_pad3 (y pad pass {ny_} -> {3 * ny_ // 2}, phase-split 3/2 rule)",
             1: f"k_pad3 (x pad pass {nx_} -> {3 * nx_ // 2}, phase-split 3/2 rule)",
             2: f"k_unpad3 (x unpad pass {3 * nx_ // 2} -> {nx_})",
             3: f"k_unpad3 (y unpad pass {3 * ny_ // 2} -> {ny_})",
             4: "k_line_rr (x derivative line pass)",
             5: "k_y_fwd (2-D path: real rows -> half spectrum)",
             6: "k_x (2-D path: x columns, forward FFT + two i*k outputs)",
             7: "k_y_inv (2-D path: half spectrum -> real rows)"}
    probes = {}
    for which in names:
        if a.lib.alfa_time_kernel(a.ctx, which, 20, ctypes.byref(t_ms), ctypes.byref(t_bytes)) == 0:
            gbs = t_bytes.value / (t_ms.value * 1e-3) / 1e9
            probes[which] = {"kernel": names[which], "avg_launch_ms": t_ms.value,
                             "alg_bytes_per_launch": t_bytes.value, "achieved_gbs": gbs,
                             "frac": gbs / peak}
    chosen = {c["shape"]: c["variant"] for c in head["tune"] if c["chosen"]}
    for which, shape in ((0, "y pad"), (1, "x pad"), (2, "x unpad"), (3, "y unpad"),
                         (4, "x derivative")):
        if which in probes and chosen.get(shape, "default") != "default":
            probes[which]["kernel"] = (f"{shape} line pass, autotuned variant "
                                       f"'{chosen[shape]}'")
    # the split-BF16 tensor-core line pass (FP32 x derivative of a field of
    # this grid): issued tensor flops and bytes per launch
    tc = None
    if a.lib.alfa_time_kernel(a.ctx, 8, 20, ctypes.byref(t_ms), ctypes.byref(t_bytes)) == 0:
        flops = 3 * 2.0 * nx_ * nx_ * ny_ * nz_
        tflops = flops / (t_ms.value * 1e-3) / 1e12
        bf16_peak, bf16_kind = measured_bf16_peak()
        gbs = t_bytes.value / (t_ms.value * 1e-3) / 1e9
        tc = {"kernel": "k_line_gemm_bf16x3 (x derivative, FP32 lines, split BF16 on tcgen05)",
              "avg_launch_ms": t_ms.value, "alg_bytes_per_launch": t_bytes.value,
              "achieved_gbs": gbs, "hbm_frac": gbs / peak, "issued_tflops": tflops,
              "tensor_frac": tflops / bf16_peak,
              "tensor_peak": f"{bf16_kind} {bf16_peak:.0f} TFLOP/s bf16 dense (burst)"}
    dom = 1  # the x pad pass holds the largest share of the step (profiles/)
    if dom in probes:
        tr = ncu_traffic()
        p1 = probes[dom]
        roof = {"kernel": p1["kernel"], "bound": "hbm", "achieved": p1["achieved_gbs"],
                "peak": peak, "unit": "GB/s", "frac": p1["frac"],
                "peak_source": f"{peak_kind} hbm_gbs (burst copy)",
                "alg_bytes_per_launch": p1["alg_bytes_per_launch"],
                "avg_launch_ms": p1["avg_launch_ms"],
                "traffic": (tr or {}).get(args.precision, {}).get("dram_bytes_per_launch"),
                "traffic_source": "profiles/dominant_kernel_traffic.txt (one ncu capture)",
                "other_kernels": [probes[k] for k in names if k in probes and k != dom]}
    del sim, head
    torch.cuda.empty_cache()

    # ---- end to end through the C-ABI with host buffers -----------------
    # The whole-step entry (alfa_init_state / alfa_step_graph / alfa_get_diag
    # / alfa_get_state) on a context created beforehand: the state comes in
    # from pinned host memory (FP64, as the reference's arrays), every step
    # reads its CFL diagnostics back to the host (Main.py:534-540 checks CFL
    # every step), and the final state goes back to pinned host memory, all
    # inside the timed region.
    e2e = None
    if not args.no_e2e:
        host = [torch.from_numpy(np.ascontiguousarray(x)).pin_memory() for x in (u, v, w, th)]
        outs = [torch.empty(x.shape, dtype=torch.float64).pin_memory() for x in host]
        sim_e = Simulation(workload_config(grid, 2 * total, args.precision), u, v, w, th)
        if not args.no_tune:
            sim_e.autotune(reps=3)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

        def run_e2e():
            sim_e.reset(*host)
            for _ in range(args.steps):
                sim_e.step(1, graph=True)
                sim_e.diag()  # synchronises: the step's CFL on the host
            st = sim_e.state()
            for o, k in zip(outs, ("u", "v", "w", "TH")):
                o.copy_(st[k], non_blocking=True)
        run_e2e()  # captures the step graphs of this sequence
        torch.cuda.synchronize(dev)
        barrier()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        e0.record(stream)
        run_e2e()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        barrier()
        e2e_ms = max_over_ranks(e0.elapsed_time(e1))
        state_bytes = 4 * 8 * n_gp
        e2e = {"value": n_gp * args.steps * world / (e2e_ms / 1e3), "unit": "gp-steps/s",
               "h2d_bytes_per_step": state_bytes / args.steps,
               # per step: CFL (3), qz_sfc_avg (1) and the ustar plane of alfa_get_diag
               "d2h_bytes_per_step": state_bytes / args.steps + 8 * (4 + grid[0] * grid[1]),
               "path": f"whole-step C-ABI, precision {args.precision} (alfa_init_state, "
                       "alfa_step_graph, alfa_get_diag every step, alfa_get_state): FP64 state "
                       "from and to pinned host memory inside the timed region",
               "host_wall_ms": 1e3 * (time.perf_counter() - t0)}
        del sim_e
        torch.cuda.empty_cache()

    # the ensemble workload, a short run beside the headline (`--ensemble`
    # gives its full 500-step line)
    # (rank 0 only: no collective follows, the line is rank 0's)
    ens = None
    if not args.no_ensemble and rank == 0:
        ens = ensemble_measure(50, args.warmup, "fp32")
    # the convective and stable configurations, short
    wl = None
    if not args.no_workloads and rank == 0:
        wl = workloads_measure()

    cpu = None
    if rank == 0 and not args.no_cpu:
        threads, model = cpu_info()
        n, dt = oracle_steps(grid, threads, 1, 3, args.cpu_budget)
        cpu = {"value": n_gp * n / dt, "unit": "gp-steps/s", "cores": threads, "cpu_model": model,
               "kind": "port",
               "sample": f"{n} step(s) after 1 warm-up of the same {grid[0]}x{grid[1]}x{grid[2]} "
                         f"workload, {dt / n:.1f} s/step: NumPy FP64 port of the reference's "
                         f"step, scipy.fft on {threads} threads"}
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": "gp-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak",
            "vs_baseline": value / (A100_FP64 if args.precision == "fp64" else A100_FP32),
            "vs_baseline_ref": ("A100 JAX NBL_A94 256^3 LASDD-SM "
                                + ("FP64 93.4 M" if args.precision == "fp64" else "FP32 166.8 M")
                                + " gp-steps/s (BASELINE.md)"),
            "dtype": DTYPES[args.precision], "data": "synthetic",
            "config": config_block(grid, world, args.precision),
            "clocks": clk_head, "gpu_launches": launches_head,
            "fp64": fp64, "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
            "tensor_core_line_pass": tc,
            "ensemble": ens,
            "workloads": wl,
            # the chosen variant of each pass shape, and the tensor-core
            # candidate's time beside it (mixed precision)
            "autotune": [{k: c[k] for k in ("shape", "variant", "ms", "equal", "chosen")}
                         for c in tune_head if c["chosen"] or c["variant"] == "tensor-core"],
        }), flush=True)


def ensemble_measure(steps, warmup, precision):
    """The ensemble workload (cases.ensemble_members: 64 independent neutral
    members of uneven sizes, 32 of 32^3, 16 of 48^3, 16 of 64^3, each with its
    own seed, u* ~ U[0.3, 0.6] m/s and z0 log-uniform in [0.01, 0.5] m) stepped
    together (one CUDA graph launch per step across the members' streams)
    against the same members stepped one after another.  Both timed with CUDA
    events on this stream (the ensemble's steps are ordered on it,
    alfa_ensemble_set_stream); every member's final state is compared with
    the same member run alone."""
    import torch

    from jax_alfa_b200 import cases
    from jax_alfa_b200.api import Ensemble, Simulation
    total = warmup + steps + 2
    members = cases.ensemble_members(nsteps=total, precision=precision)
    n_gp = int(sum(c["nx"] * c["ny"] * c["nz"] for c, _ in members))
    stream = torch.cuda.current_stream()
    n_warm = 1 + max(warmup - 1, 2)

    def make(c, seed):
        u, v, w, th = cases.initial_fields(c, seed)
        return Simulation(c, u, v, w, th, adv_series=cases.adv_forcing_series(c))

    def state(sim):
        return {k: t.cpu().numpy() for k, t in sim.state().items()}

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sims = [make(c, seed) for c, seed in members]
    for s_ in sims:  # the bootstrap step, then graph captures of both parities
        s_.step(1)
        s_.step(n_warm - 1, graph=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        for s_ in sims:
            s_.step(1, graph=True)
    e1.record(stream)
    torch.cuda.synchronize()
    t_seq = e0.elapsed_time(e1) / steps
    alone = [state(s_) for s_ in sims]
    del sims
    torch.cuda.empty_cache()

    # the ensemble's steps ordered on a stream of their own (the legacy
    # default stream cannot be handed over: its handle is the null stream)
    tstream = torch.cuda.Stream()
    ens = Ensemble([make(c, seed) for c, seed in members]).set_stream(tstream)
    ens.step(n_warm)
    torch.cuda.synchronize()
    e0.record(tstream)
    ens.step(steps)
    e1.record(tstream)
    torch.cuda.synchronize()
    t_ens = e0.elapsed_time(e1) / steps
    errs, exact = [], 0
    finite = sum(all(np.isfinite(r[k]).all() for k in r) for r in alone)
    for st, ref in zip(ens.states(), alone):
        got = {k: t.cpu().numpy() for k, t in st.items()}
        e = max(float(np.abs(got[k] - ref[k]).max()) / max(float(np.abs(ref[k]).max()), 1e-300)
                for k in ref)
        errs.append(e)
        exact += all(np.array_equal(got[k], ref[k]) for k in ref)
    ens.close()
    del ens
    torch.cuda.empty_cache()
    return {
        "metric": "ensemble LES grid-point-steps/s (64 members: 32x32^3, 16x48^3, 16x64^3)",
        "value": n_gp / (t_ens / 1e3), "unit": "gp-steps/s", "steps": steps, "warmup": n_warm,
        "ms_per_step": t_ens,
        "sequential": {"value": n_gp / (t_seq / 1e3), "ms_per_step": t_seq,
                       "how": "the same members, one graph step each, one after another"},
        "speedup_vs_sequential": t_seq / t_ens,
        "members_vs_alone": {"max_rel_err": max(errs), "bit_identical": exact,
                             "finite_members": finite, "members": len(errs), "bar": 1e-6,
                             "after_steps": n_warm + steps},
        "dtype": DTYPES[precision],
        "config": {"workload": "neutral ABL members (C1 physics), LASDD-SM, per-member seed, "
                               "u* ~ U[0.3, 0.6] m/s, z0 log-uniform [0.01, 0.5] m, dt scaled "
                               "to the grid",
                   "members": len(members), "grid_points": n_gp, "precision": precision,
                   "timing": "CUDA events on the stream the steps are ordered on"}}


def workloads_measure():
    """The other two configurations of the benchmark matrix, short, beside
    the headline: the convective ABL at 128^3 (mixed and FP64 from the same
    initial fields, 1500 steps of spin-up then 500 steps with the statistics
    accumulated every step; the plane-averaged <u>, <theta>, <w'theta'> and
    <w'w'> profiles of the two compared) and the stable ABL at 256x256x192
    (LAD-SM, 20 graph steps of each precision).  CUDA events on this
    stream."""
    import torch

    from jax_alfa_b200 import cases
    from jax_alfa_b200.api import Simulation, stats_to_dict

    def sim_of(cfg):
        u, v, w, th = cases.initial_fields(cfg, 0)
        sfc = cases.surface_bc_series(cfg) if cfg["optSurfBC"] else None
        return Simulation(cfg, u, v, w, th, surface_series=sfc)

    def timed(sim, n):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        sim.step(n, graph=True)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n

    out = {}
    # convective 128^3
    spin, avg = 1500, 500
    prof, ms = {}, {}
    for p in ("mixed", "fp64"):
        cfg = cases.convective(128, 128, 128, nsteps=spin + avg + 2, precision=p)
        sim = sim_of(cfg)
        sim.step(1)
        if p == "mixed":
            sim.autotune(reps=2)
        ms[p] = timed(sim, spin - 1)
        acc = None
        for _ in range(avg):
            sim.step(1, graph=True)
            acc = sim.stats_sample(acc)
        prof[p] = stats_to_dict(acc, 128, cfg["Ugal"])
        del sim
        torch.cuda.empty_cache()
    n_gp = 128 ** 3
    out["convective_128"] = {
        "workload": "convective ABL 128^3 (CBL_N91 physics), LASDD-SM, 2000 steps",
        "mixed": {"ms_per_step": ms["mixed"], "value": n_gp / (ms["mixed"] / 1e3)},
        "fp64": {"ms_per_step": ms["fp64"], "value": n_gp / (ms["fp64"] / 1e3)},
        "speedup": ms["fp64"] / ms["mixed"],
        "profile_err_vs_fp64": {
            k: float(np.abs(prof["mixed"][k] - prof["fp64"][k]).max()
                     / max(float(np.abs(prof["fp64"][k]).max()), 1e-300))
            for k in ("U", "TH", "wTH", "w2")},
        "profile_definition": "Statistics.py profiles accumulated over steps 1501-2000, max "
                              "|mixed - fp64| / max |fp64|"}
    # stable 256x256x192
    ms, st = {}, {}
    for p in ("mixed", "fp64"):
        cfg = cases.stable(256, 256, 192, nsteps=30, precision=p)
        sim = sim_of(cfg)
        sim.step(1)
        if p == "mixed":
            sim.autotune(reps=2)
        sim.step(3, graph=True)
        ms[p] = timed(sim, 20)
        st[p] = {k: t.cpu().numpy() for k, t in sim.state().items()}
        del sim
        torch.cuda.empty_cache()
    vmax = max(float(np.abs(st["fp64"][k]).max()) for k in ("u", "v", "w"))
    serr = {k: float(np.abs(st["mixed"][k] - st["fp64"][k]).max()) / vmax for k in ("u", "v", "w")}
    for k in ("TH", "p"):
        serr[k] = float(np.abs(st["mixed"][k] - st["fp64"][k]).max()) / max(
            float(np.abs(st["fp64"][k]).max()), 1e-300)
    n_gp = 256 * 256 * 192
    out["stable_256x256x192"] = {
        "workload": "stable ABL 256x256x192 (GABLS1-like), LAD-SM, 20 timed steps",
        "mixed": {"ms_per_step": ms["mixed"], "value": n_gp / (ms["mixed"] / 1e3)},
        "fp64": {"ms_per_step": ms["fp64"], "value": n_gp / (ms["fp64"] / 1e3)},
        "speedup": ms["fp64"] / ms["mixed"],
        "err_vs_fp64": serr,
        "err_definition": "after 24 steps from the same initial fields, as the headline's"}
    return out


def run_ensemble(args):
    """The ensemble form on its own line (`--ensemble`, 500 steps by default)."""
    out = ensemble_measure(args.steps, args.warmup, args.ens_precision)
    out.update({"n_gpus": 1, "higher_is_better": True, "data": "synthetic"})
    print(json.dumps(out), flush=True)
    m = out["members_vs_alone"]
    if not (m["max_rel_err"] <= 1e-6) or m["finite_members"] != m["members"]:
        raise SystemExit(f"ensemble members: max error {m['max_rel_err']:.2e}, "
                         f"{m['finite_members']} of {m['members']} finite")


def run_learned(args):
    """The learned-closure form on the convective ABL at 192x192x128: after
    args.spinup dynamic steps, 2000 more dynamic steps each supply 100
    training samples (200k), the network trains with the hand-written
    kernels, then from one checkpoint args.steps steps run three ways: the
    dynamic procedure every step; the network, judged by the procedure every
    20 steps at a 5 % drift tolerance (windowed, recalibrating the level means
    at each judge step); and the coefficients of the last dynamic step held
    fixed (the reference's static steps, dynamicSGS_call_time never due).
    Reports the step times and the errors of the plane-averaged profiles
    (Statistics.py definitions, accumulated over the run) of the learned and
    the fixed arm against the dynamic one; CUDA events on the current
    stream."""
    import torch

    from jax_alfa_b200 import cases
    from jax_alfa_b200.api import Learned, Simulation, stats_to_dict
    grid = (192, 192, 128)
    cfg = cases.convective(*grid, nsteps=args.spinup + 2000 + args.steps + 10)
    u, v, w, th = cases.initial_fields(cfg, 0)
    sim = Simulation(cfg, u, v, w, th)
    sim.step(1)
    sim.step(args.spinup - 1, graph=True)  # spin-up of the convective layer
    net = Learned(sim, capacity=200_000, seed=1)
    for _ in range(2000):
        sim.step(1)
        net.collect(100)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    loss = net.train(epochs=args.epochs, batch=1024, lr=2e-3)
    ev1.record()
    torch.cuda.synchronize()
    t_train = ev0.elapsed_time(ev1) / 1e3
    ck = sim.checkpoint()
    P, norm = net.params()
    del net, sim
    torch.cuda.empty_cache()

    def run(mode):
        c2 = dict(cfg)
        if mode == "fixed":
            c2["dynamicSGS_call_time"] = 10 ** 9
        s_ = Simulation(c2, u, v, w, th).restore(ck)
        n2 = None
        if mode == "learned":
            n2 = Learned(s_, capacity=1024)
            n2.set_params(P, norm)
        acc, rep = None, None
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            if mode == "learned":
                rep = n2.step(1, judge_every=20, tol=0.05)
            else:
                s_.step(1)
            acc = s_.stats_sample(acc)
        e1.record()
        torch.cuda.synchronize()
        return stats_to_dict(acc, grid[2], cfg["Ugal"]), e0.elapsed_time(e1) / args.steps, rep
    dyn, t_dyn, _ = run("dynamic")
    lrn, t_lrn, rep = run("learned")
    fix, t_fix, _ = run("fixed")
    keys = ("U", "TH", "uw", "vw", "wTH", "txz", "tyz", "qz", "u2", "w2")

    def errs(x):
        return {k: float(np.abs(x[k] - dyn[k]).max() / max(np.abs(dyn[k]).max(), 1e-300))
                for k in keys}
    n_gp = int(np.prod(grid))
    print(json.dumps({
        "metric": "learned-coefficient LES grid-point-steps/s (192x192x128 convective)",
        "value": n_gp / (t_lrn / 1e3), "unit": "gp-steps/s", "n_gpus": 1, "steps": args.steps,
        "higher_is_better": True, "ms_per_step": t_lrn,
        "dynamic": {"value": n_gp / (t_dyn / 1e3), "ms_per_step": t_dyn},
        "fixed": {"value": n_gp / (t_fix / 1e3), "ms_per_step": t_fix,
                  "how": "Cs^2 of the last dynamic step held (static steps)"},
        "speedup_vs_dynamic": t_dyn / t_lrn,
        "profile_errors_vs_dynamic": {"learned": errs(lrn), "fixed": errs(fix),
                                      "definition": "max |x - x_dyn| / max |x_dyn| of the "
                                                    "profiles accumulated over the run"},
        "judge": {"every": 20, "tol": 0.05, "window_judge_steps": 8, "report": rep},
        "training": {"samples": 200000, "from_dynamic_steps": 2000,
                     "after_spinup_steps": args.spinup, "epochs": args.epochs,
                     "batch": 1024, "seconds": t_train, "final_loss_normalised": loss},
        "dtype": "f64 step, f32 network (bf16 weights at inference)", "data": "synthetic",
        "config": {"workload": "convective ABL 192x192x128 (C2 physics), LASDD-SM judge"}}),
        flush=True)


def main():
    args = parse()
    if args.learned:
        run_learned(args)
        return
    if args.ensemble:
        run_ensemble(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if args.impl == "alfa":
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl" if args.impl == "alfa" else "gloo",
                                timeout=datetime.timedelta(seconds=120))
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        else:
            run_alfa(args, rank, world, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
