"""Throughput of the LES step on B200: grid-point-steps per second.

Workload (default): the neutral ABL case at 256^3 (LASDD-SM dynamic SGS,
3/2-rule dealiasing, Thomas pressure solve), FP64 -- the 256^3 LASDD-SM
FP64 configuration of the reference's A100 benchmark table.  Synthetic
seeded initial fields (log-law u with 0.5 % noise below 500 m); every field
(134 MB) is larger than L2 (126 MB), so no L2 flush is needed between steps.

  value  : device-timed whole steps (alfa_step, state resident in HBM),
           CUDA events on the launching stream, max over ranks.
  e2e    : the same steps through the reference-facing per-function API
           (jax_alfa_b200.driver.MainLoop, the Main.py loop on the C-ABI),
           with the initial state copied in from pinned host memory, the
           forcing row going in and the CFL check coming out every step, and
           the final state copied back, all inside the timed region.
  --impl reference : the reference's CPU implementation of the same step
           (the NumPy FP64 port of it, scipy.fft with every host thread) on a
           bounded sample: one step of the same physics on a 128^3 grid.

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

A100_BASELINE = 93.4e6   # gp-steps/s, 256^3 LASDD-SM FP64 on A100 (reference notebook)
METRIC = "LES grid-point-steps/s at 256^3"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="alfa", choices=["alfa", "reference"])
    ap.add_argument("--grid", type=int, nargs=3, default=[256, 256, 256])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--epochs", type=int, default=40,
                    help="training epochs of the learned closure (--learned)")
    ap.add_argument("--no-tune", action="store_true",
                    help="skip the line-pass autotuner (default dispatch)")
    ap.add_argument("--learned", action="store_true",
                    help="the learned SGS coefficient on the 192x192x128 convective case: "
                         "train on the dynamic procedure, then time and compare learned steps")
    ap.add_argument("--ensemble", action="store_true",
                    help="time the 64-member uneven ensemble (32x32^3, 16x48^3, 16x64^3) "
                         "against its members stepped one at a time")
    return ap.parse_args()


def workload_config(grid, nsteps):
    from jax_alfa_b200 import cases
    cfg = cases.neutral(*grid, nsteps=nsteps)
    cfg["case"] = "neutral"
    return cfg


def config_block(grid, world):
    return {"workload": f"neutral ABL {grid[0]}x{grid[1]}x{grid[2]}, LASDD-SM dynamic SGS, "
                        "3/2-rule dealiasing, Thomas pressure, AB2, FP64",
            "grid": list(grid), "sgs": "LASDD-SM (optSgs=1, dynamic every step)",
            "precision": "FP64 plain drop-in", "l2": "every field (8 B x N) exceeds L2; no flush",
            "step": "one CUDA graph replay per step (alfa_step_graph)",
            "parallelism": f"replicas x{world} (no sharding)",
            "baseline": "A100 JAX 256^3 LASDD-SM FP64, 93.4 M gp-steps/s"}


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


def cpu_baseline(threads, grid=(128, 128, 128)):
    """One step of the NumPy FP64 port of the reference on the host."""
    from jax_alfa_b200 import cases
    from oracle import alfa_oracle
    from oracle.alfa_oracle import AlfaOracle, OracleRun
    alfa_oracle.set_fft_workers(threads)
    cfg = workload_config(grid, 2)
    u, v, w, th = cases.initial_fields(cfg, 0)
    o = AlfaOracle(cfg)
    r = OracleRun(cfg, u, v, w, th, adv=o.adv_series(*cases.adv_forcing_series(cfg)))
    t = time.perf_counter()
    with np.errstate(all="ignore"):
        r.step()
    dt = time.perf_counter() - t
    n = grid[0] * grid[1] * grid[2]
    return n / dt, dt


def run_reference(args, rank, world):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    from jax_alfa_b200 import cases
    from oracle import alfa_oracle
    from oracle.alfa_oracle import AlfaOracle, OracleRun
    alfa_oracle.set_fft_workers(threads)
    grid = (128, 128, 128)
    total = args.warmup + args.steps
    cfg = workload_config(grid, total + 1)
    u, v, w, th = cases.initial_fields(cfg, 0)
    o = AlfaOracle(cfg)
    r = OracleRun(cfg, u, v, w, th, adv=o.adv_series(*cases.adv_forcing_series(cfg)))
    with np.errstate(all="ignore"):
        for _ in range(args.warmup):
            r.step()
        t = time.perf_counter()
        for _ in range(args.steps):
            r.step()
        dt = time.perf_counter() - t
    n = grid[0] * grid[1] * grid[2]
    value = n * args.steps / dt
    sample = (f"{args.steps} steps of the same physics on a 128^3 grid (1/8 of the 256^3 "
              f"points), {dt / args.steps:.2f} s/step, NumPy FP64 port of the reference with "
              f"scipy.fft on {threads} threads")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "gp-steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": value / A100_BASELINE, "dtype": "f64", "data": "synthetic",
        "config": config_block(args.grid, world),
        "cpu_baseline": {"value": value, "unit": "gp-steps/s", "cores": threads,
                         "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "gp-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


def run_alfa(args, rank, world, dist):
    import torch
    from jax_alfa_b200 import _lib, cases
    from jax_alfa_b200.api import Simulation
    from jax_alfa_b200.driver import MainLoop

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    grid = tuple(args.grid)
    n_gp = grid[0] * grid[1] * grid[2]
    total = args.warmup + args.steps + 2
    cfg = workload_config(grid, total)
    u, v, w, th = cases.initial_fields(cfg, rank)
    adv = cases.adv_forcing_series(cfg)
    lib = _lib.load()

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---- device-resident whole step -----------------------------------
    sim = Simulation(cfg, u, v, w, th, adv_series=adv)
    # warm-up: the bootstrap step, the line-pass autotuner (fastest variant
    # whose outputs equal the default's), then graph captures of both
    # iteration parities; the timed steps replay them (alfa_step_graph)
    sim.step(1)
    tune = sim.autotune(reps=3) if not args.no_tune else []
    sim.step(max(args.warmup - 1, 2), graph=True)
    stream = torch.cuda.current_stream(dev)
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
    d = sim.diag()
    if not np.isfinite(d["CFL"]):
        raise RuntimeError("non-finite state in the timed run")
    value = n_gp * args.steps * world / (ms / 1e3)

    # ---- dominant kernel, live --------------------------------------------
    import ctypes
    roof = None
    peak, peak_kind = measured_peaks()
    t_ms, t_bytes = ctypes.c_double(), ctypes.c_double()
    a = sim.alfa
    a.lib.alfa_set_stream(a.ctx, ctypes.c_void_p(stream.cuda_stream))
    names = {0: "k_pad3 (y pad pass 256 -> 384, phase-split 3/2 rule)",
             1: "k_pad3 (x pad pass 256 -> 384, phase-split 3/2 rule)",
             2: "k_unpad3 (x unpad pass 384 -> 256)",
             3: "k_unpad3 (y unpad pass 384 -> 256)",
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
    chosen = {c["shape"]: c["variant"] for c in tune if c["chosen"]}
    for which, shape in ((0, "y pad"), (1, "x pad"), (2, "x unpad"), (3, "y unpad"),
                         (4, "x derivative")):
        if which in probes and chosen.get(shape, "default") != "default":
            probes[which]["kernel"] = (f"{shape} line pass, autotuned variant "
                                       f"'{chosen[shape]}'")
    # the split-BF16 tensor-core line pass (FP32 x derivative of a field of
    # this grid): issued tensor flops and bytes per launch
    tc = None
    if a.lib.alfa_time_kernel(a.ctx, 8, 20, ctypes.byref(t_ms), ctypes.byref(t_bytes)) == 0:
        nx_, ny_, nz_ = grid
        flops = 3 * 2.0 * nx_ * nx_ * ny_ * nz_
        tflops = flops / (t_ms.value * 1e-3) / 1e12
        bf16_peak, bf16_kind = measured_bf16_peak()
        gbs = t_bytes.value / (t_ms.value * 1e-3) / 1e9
        tc = {"kernel": "k_line_gemm_bf16x3 (x derivative, FP32 lines, split BF16 on tcgen05)",
              "avg_launch_ms": t_ms.value, "alg_bytes_per_launch": t_bytes.value,
              "achieved_gbs": gbs, "hbm_frac": gbs / peak, "issued_tflops": tflops,
              "tensor_frac": tflops / bf16_peak,
              "tensor_peak": f"{bf16_kind} {bf16_peak:.0f} TFLOP/s bf16 dense (burst)"}
    dom = 1  # the pad passes hold the largest share of the step (profiles/)
    if dom in probes:
        tr = ncu_traffic()
        p1 = probes[dom]
        roof = {"kernel": p1["kernel"], "bound": "hbm", "achieved": p1["achieved_gbs"],
                "peak": peak, "unit": "GB/s", "frac": p1["frac"],
                "peak_source": f"{peak_kind} hbm_gbs (burst copy)",
                "alg_bytes_per_launch": p1["alg_bytes_per_launch"],
                "avg_launch_ms": p1["avg_launch_ms"],
                "traffic": None if tr is None else tr.get("dram_bytes_per_launch"),
                "other_kernels": [probes[k] for k in names if k in probes and k != dom]}
    del sim
    torch.cuda.empty_cache()

    # ---- end to end through the C-ABI with host buffers -----------------
    # e2e: the whole-step entry (alfa_init_state / alfa_step_graph /
    # alfa_get_diag / alfa_get_state) on a context created beforehand: the
    # state comes in from pinned host memory, every step reads its CFL
    # diagnostics back to the host (Main.py:534-540 checks CFL every step),
    # and the final state goes back to pinned host memory, all inside the
    # timed region.  e2e_per_function: the same through the per-function ABI
    # (MainLoop, the loop body of Main.py call for call).
    e2e = e2e_pf = None
    if not args.no_e2e:
        host = [torch.from_numpy(np.ascontiguousarray(x)).pin_memory() for x in (u, v, w, th)]
        outs = [torch.empty(x.shape, dtype=torch.float64).pin_memory() for x in host]
        sim_e = Simulation(cfg, u, v, w, th, adv_series=adv)
        if not args.no_tune:
            sim_e.autotune(reps=3)

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
               "path": "whole-step C-ABI (alfa_init_state, alfa_step_graph, alfa_get_diag "
                       "every step, alfa_get_state): state from and to pinned host memory "
                       "inside the timed region",
               "host_wall_ms": 1e3 * (time.perf_counter() - t0)}
        del sim_e
        torch.cuda.empty_cache()

        ml_warm = MainLoop(cfg, u, v, w, th, adv_series=adv)
        for _ in range(args.warmup):
            ml_warm.step()
        api = ml_warm.a
        if not args.no_tune:
            api.autotune(reps=3)
        del ml_warm
        torch.cuda.synchronize(dev)
        barrier()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        e0.record(stream)
        ml = MainLoop(cfg, *[h.numpy() for h in host], adv_series=adv, api=api)
        for _ in range(args.steps):
            ml.step()
        outs2 = [x.to("cpu", non_blocking=True) for x in (ml.u, ml.v, ml.w, ml.TH)]
        e1.record(stream)
        torch.cuda.synchronize(dev)
        barrier()
        pf_ms = max_over_ranks(e0.elapsed_time(e1))
        e2e_pf = {"value": n_gp * args.steps * world / (pf_ms / 1e3), "unit": "gp-steps/s",
                  "h2d_bytes_per_step": (state_bytes + ml.h2d_bytes) / args.steps,
                  "d2h_bytes_per_step": (state_bytes + ml.d2h_bytes) / args.steps,
                  "path": "MainLoop: Main.py loop body on the per-function C-ABI, state in/out "
                          "from pinned host memory inside the timed region",
                  "host_wall_ms": 1e3 * (time.perf_counter() - t0)}
        del outs2, ml, api

    cpu = None
    if rank == 0 and not args.no_cpu:
        v1, dt1 = cpu_baseline(1)
        cpu = {"value": v1, "unit": "gp-steps/s", "cores": 1, "kind": "port",
               "sample": f"1 step of the same physics on 128^3 (1/8 of the points), "
                         f"{dt1:.1f} s, NumPy FP64 port of the reference, 1 thread"}
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": "gp-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": value / A100_BASELINE,
            "dtype": "f64", "data": "synthetic", "config": config_block(grid, world),
            "clocks": clk, "gpu_launches": int(n1 - n0), "roofline": roof,
            "cpu_baseline": cpu, "e2e": e2e, "e2e_per_function": e2e_pf,
            "tensor_core_line_pass": tc,
            "autotune": [{k: c[k] for k in ("shape", "variant", "ms")} for c in tune
                         if c["chosen"]],
        }), flush=True)


def run_ensemble(args):
    """The ensemble form: 64 independent neutral members of uneven sizes, each
    with its own seed, stepped together (one CUDA graph launch per step)
    against the same members stepped one after another.  Host wall clock
    around synchronised calls (the ensemble's streams are internal)."""
    import time

    import numpy as np
    import torch

    from jax_alfa_b200 import cases
    from jax_alfa_b200.api import Ensemble, Simulation
    grids = [(32, 32, 32)] * 32 + [(48, 48, 48)] * 16 + [(64, 64, 64)] * 16
    total = 2 * (args.warmup + args.steps) + 4
    cfgs = [workload_config(g, total) for g in grids]

    def make(i, c):
        u, v, w, th = cases.initial_fields(c, i)
        return Simulation(c, u, v, w, th, adv_series=cases.adv_forcing_series(c))

    n_gp = int(sum(np.prod(g) for g in grids))
    sims = [make(i, c) for i, c in enumerate(cfgs)]
    for s_ in sims:
        s_.step(args.warmup, graph=True)
    torch.cuda.synchronize()
    t = time.perf_counter()
    for _ in range(args.steps):
        for s_ in sims:
            s_.step(1, graph=True)
    torch.cuda.synchronize()
    t_seq = (time.perf_counter() - t) / args.steps
    del sims
    torch.cuda.empty_cache()
    ens = Ensemble([make(i, c) for i, c in enumerate(cfgs)])
    ens.step(args.warmup).sync()
    t = time.perf_counter()
    ens.step(args.steps).sync()
    t_ens = (time.perf_counter() - t) / args.steps
    ens.close()
    print(json.dumps({
        "metric": "ensemble LES grid-point-steps/s (64 members: 32x32^3, 16x48^3, 16x64^3)",
        "value": n_gp / t_ens, "unit": "gp-steps/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t_ens, "higher_is_better": True,
        "sequential": {"value": n_gp / t_seq, "ms_per_step": 1e3 * t_seq,
                       "how": "the same members, one graph step each, one after another"},
        "speedup_vs_sequential": t_seq / t_ens, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "neutral ABL members (C1 physics), LASDD-SM, FP64",
                   "members": len(grids), "grid_points": n_gp,
                   "timing": "host wall clock around synchronised calls"}}), flush=True)


def run_learned(args):
    """The learned-closure form on the convective ABL at 192x192x128: after
    160 spin-up steps, 40 dynamic steps supply 200k training samples, the network trains with the
    hand-written kernels, then from one checkpoint 20 steps run with the
    dynamic procedure and 20 with the network (judged every 10 steps).
    Reports the step speed-up and the error of the plane-averaged profiles
    (resolved and SGS stresses, w'theta', SGS heat flux) against the dynamic
    run; CUDA events on the current stream."""
    import numpy as np
    import torch

    from jax_alfa_b200 import cases
    from jax_alfa_b200.api import Learned, Simulation, stats_to_dict
    grid = (192, 192, 128)
    cfg = cases.convective(*grid, nsteps=400)
    u, v, w, th = cases.initial_fields(cfg, 0)

    def make():
        return Simulation(cfg, u, v, w, th)
    sim = make()
    sim.step(160)  # spin-up of the convective layer (dynamic procedure)
    net = Learned(sim, capacity=200_000, seed=1)
    for _ in range(40):
        sim.step(1)
        net.collect(5000)
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

    def run(learned):
        s_ = make().restore(ck)
        n2 = None
        if learned:
            n2 = Learned(s_, capacity=1024)
            n2.set_params(P, norm)
        acc, rep = None, None
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            if learned:
                rep = n2.step(1, judge_every=10, tol=0.05, refresh_points=20000,
                              refresh_epochs=3)
            else:
                s_.step(1)
            acc = s_.stats_sample(acc)
        e1.record()
        torch.cuda.synchronize()
        return stats_to_dict(acc, grid[2], cfg["Ugal"]), e0.elapsed_time(e1) / args.steps, rep
    dyn, t_dyn, _ = run(False)
    lrn, t_lrn, rep = run(True)
    errs = {k: float(np.abs(lrn[k] - dyn[k]).max() / max(np.abs(dyn[k]).max(), 1e-300))
            for k in ("uw", "vw", "wTH", "txz", "tyz", "qz", "u2", "w2")}
    n_gp = int(np.prod(grid))
    print(json.dumps({
        "metric": "learned-coefficient LES grid-point-steps/s (192x192x128 convective)",
        "value": n_gp / (t_lrn / 1e3), "unit": "gp-steps/s", "n_gpus": 1, "steps": args.steps,
        "higher_is_better": True, "ms_per_step": t_lrn,
        "dynamic": {"value": n_gp / (t_dyn / 1e3), "ms_per_step": t_dyn},
        "speedup_vs_dynamic": t_dyn / t_lrn,
        "profile_errors_vs_dynamic": errs,
        "judge": {"every": 10, "tol": 0.05, "refresh": "20000 samples, 3 epochs per judge step",
                  "report": rep},
        "training": {"samples": 200000, "after_spinup_steps": 160, "epochs": args.epochs,
                     "batch": 1024, "seconds": t_train,
                     "final_loss_normalised": loss},
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
