"""GPU tests of the learned SGS coefficient (alfa_mlp_*): the training
gradient and the features against the NumPy restatement, an end-to-end run
that trains on the dynamic procedure and steps with the network beside the
dynamic and the fixed-coefficient arms, and the judge's revert."""
import numpy as np
import pytest
import torch

from jax_alfa_b200 import cases

pytestmark = pytest.mark.gpu


def _sim(cfg, seed=0):
    from jax_alfa_b200.api import Simulation
    u, v, w, th = cases.initial_fields(cfg, seed)
    adv = cases.adv_forcing_series(cfg) if cfg["optAdvection"] else None
    sfc = cases.surface_bc_series(cfg) if cfg["optSurfBC"] else None
    return Simulation(cfg, u, v, w, th, surface_series=sfc, adv_series=adv)


def test_training_gradient_matches_oracle():
    from jax_alfa_b200.api import Learned
    from oracle import alfa_mlp_oracle as mo
    sim = _sim(cases.convective(16, 16, 8, nsteps=2))
    net = Learned(sim, capacity=1024, seed=3)
    P, _ = net.params()
    rng = np.random.default_rng(11)
    X = rng.standard_normal((300, 10)).astype(np.float32)
    T = rng.standard_normal((300, 2)).astype(np.float32)
    norm = np.concatenate([rng.standard_normal(12) * 0.1, 0.5 + rng.random(12)]).astype(np.float32)
    loss, g = net.loss_grad(X, T, norm)
    loss_o, g_o = mo.loss_and_grad(P.astype(np.float64), X, T, norm)
    assert abs(loss - loss_o) <= 1e-5 * abs(loss_o)
    err = np.abs(g - g_o).max() / np.abs(g_o).max()
    print(f"gradient: relative error {err:.2e} (FP32 accumulation)")
    assert err <= 1e-4
    net.close()


def test_features_match_oracle():
    from jax_alfa_b200.api import Learned
    from oracle.alfa_oracle import OracleRun
    from oracle import alfa_mlp_oracle as mo
    cfg = cases.convective(24, 24, 16, nsteps=2)
    sim = _sim(cfg).step(1)
    u, v, w, th = cases.initial_fields(cfg, 0)
    r = OracleRun(cfg, u, v, w, th)
    with np.errstate(all="ignore"):
        r.step()
    net = Learned(sim, capacity=1024)
    got = net.features().cpu().numpy().astype(np.float64)
    exp, S, den = mo.features(r.o, r.last["grads"], r.last["dTHdz"], with_scales=True)
    # the ratio features (bounded: |S_ij/|S|| <= 1, Ri/(1+|Ri|) in (-1, 1)) are
    # compared in absolute terms where their denominators are above round-off
    # (|S| and uz^2 + vz^2 vanish at the top level, where both codes divide
    # rounding noise by rounding noise); the others relative to their maximum
    ok_s = S > 1e-6 * S.max()
    ok_r = ok_s & (den > 1e-6 * den.max())
    for f in range(10):
        g, x = got[..., f], exp[..., f]
        if 1 <= f <= 6 or f == 9:
            m = ok_r if f == 9 else ok_s
            e = float(np.abs(g - x)[m].max())
        else:
            e = float(np.abs(g - x).max() / max(np.abs(x).max(), 1e-30))
        print(f"feature {f}: error {e:.2e}")
        assert e <= 1e-5, (f, e)
    net.close()


def test_learned_closure_trains_and_steps(report_line):
    """Train on the dynamic procedure of a spun-up convective layer, then
    from one checkpoint run 200 steps three ways: the dynamic procedure every
    step; the network, judged by the procedure every 10 steps (its windowed
    drift recorded; tol large so every non-judge step stays learned); and the
    coefficients of the last dynamic step held fixed (static steps, the
    method without the network).  The learned steps must be faster than the
    dynamic ones and their windowed drift finite; the profile errors of the
    learned and the fixed arm against the dynamic one are reported."""
    from jax_alfa_b200.api import Learned, stats_to_dict
    spin, ncol, steps = 3000, 200, 200
    cfg = cases.convective(32, 32, 24, nsteps=spin + ncol + steps + 10)
    sim = _sim(cfg)
    sim.step(1)
    sim.step(spin - 1, graph=True)
    net = Learned(sim, capacity=200_000, seed=1)
    for _ in range(ncol):
        sim.step(1)
        net.collect(1000)
    loss = net.train(epochs=60, batch=1024, lr=2e-3)
    ck = sim.checkpoint()
    P, norm = net.params()

    def run(mode):
        c2 = dict(cfg)
        if mode == "fixed":
            c2["dynamicSGS_call_time"] = 10 ** 9
        s = _sim(c2).restore(ck)
        acc, rep = None, None
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if mode == "learned":
            n2 = Learned(s, capacity=1024)
            n2.set_params(P, norm)
        ev0.record()
        for _ in range(steps):
            if mode == "learned":
                rep = n2.step(1, judge_every=10, tol=1e9)
            else:
                s.step(1)
            acc = s.stats_sample(acc)
        ev1.record()
        torch.cuda.synchronize()
        return stats_to_dict(acc, cfg["nz"], cfg["Ugal"]), ev0.elapsed_time(ev1) / steps, rep

    dyn, t_dyn, _ = run("dynamic")
    lrn, t_lrn, rep = run("learned")
    fix, t_fix, _ = run("fixed")
    # the first step of the run and every iteration divisible by 10
    assert steps // 10 <= rep["judged"] <= steps // 10 + 1
    assert rep["learned_steps"] == steps - rep["judged"] and not rep["reverted"]
    assert np.isfinite(rep["max_window_drift"])
    errs = {k: (float(np.abs(lrn[k] - dyn[k]).max() / np.abs(dyn[k]).max()),
                float(np.abs(fix[k] - dyn[k]).max() / np.abs(dyn[k]).max()))
            for k in ("U", "TH", "uw", "wTH", "qz", "w2")}
    report_line(f"learned closure, convective 32x32x24 after {spin} steps, {steps} steps "
                f"(training loss {loss:.2f}): ms/step dynamic {t_dyn:.2f}, learned {t_lrn:.2f}, "
                f"fixed {t_fix:.2f}; judge window drift last {rep['window_drift']:.3f}, max "
                f"{rep['max_window_drift']:.3f}; profile error vs dynamic (learned / fixed): "
                + ", ".join(f"{k} {a:.1e}/{b:.1e}" for k, (a, b) in errs.items()))
    assert t_lrn < t_dyn
    # the same run judged at the 5 % tolerance: either the network is
    # accepted throughout (its windowed drift never above 0.05) or the judge
    # records the revert at the step where it went above
    s5 = _sim(cfg).restore(ck)
    n5 = Learned(s5, capacity=1024)
    n5.set_params(P, norm)
    r5 = n5.step(steps, judge_every=10, tol=0.05)
    if r5["reverted"]:
        assert r5["window_drift"] > 0.05 and r5["reverted_at"] > 0
        assert r5["learned_steps"] + r5["judged"] <= steps  # dynamic steps after the revert
    else:
        assert r5["max_window_drift"] <= 0.05 and r5["learned_steps"] == steps - r5["judged"]
    report_line(f"learned closure at tol 0.05: {'reverted at iteration ' + str(r5['reverted_at']) if r5['reverted'] else 'accepted'}"
                f" (windowed drift last {r5['window_drift']:.3f}, max {r5['max_window_drift']:.3f}, "
                f"{r5['learned_steps']} of {steps} steps learned)")


def test_judge_reverts_to_the_dynamic_procedure():
    """A drift tolerance no network meets (1e-9): the judge reverts once its
    window of ALFA_MLP_JUDGE_WINDOW (8) judge steps is full, and every later
    step runs the dynamic procedure."""
    from jax_alfa_b200.api import Learned
    cfg = cases.convective(16, 16, 8, nsteps=200)
    sim = _sim(cfg)
    sim.step(1)
    net = Learned(sim, capacity=4096, seed=2)
    for _ in range(4):
        sim.step(1)
        net.collect(1024)
    net.train(epochs=2, batch=1024, lr=1e-3)
    rep = net.step(120, judge_every=10, tol=1e-9)
    assert rep["reverted"] == 1 and rep["judged"] >= 8
    first = rep["reverted_at"]
    more = net.step(10, judge_every=10, tol=1e-9)
    assert more["learned_steps"] == rep["learned_steps"]  # no learned step after the revert
    assert first == more["reverted_at"]


def test_tensor_core_inference_matches_cuda_core_inference(report_line):
    """The learned step evaluates the network with its 64 x 64 hidden layer
    on the tensor cores (tcgen05, BF16 activations, FP32 accumulation in
    tensor memory); alfa_mlp_infer evaluates it on the CUDA cores with FP32
    activations.  On the state of a learned step the two Cs^2 fields agree
    to the BF16 rounding of the activations: within 1 % of the field's
    largest value everywhere and 1e-3 on average."""
    from jax_alfa_b200.api import Learned
    cfg = cases.convective(32, 32, 24, nsteps=60)
    sim = _sim(cfg)
    sim.step(1)
    sim.step(29, graph=True)
    net = Learned(sim, capacity=20_000, seed=4)
    for _ in range(5):
        sim.step(1)
        net.collect(4000)
    net.train(epochs=20, batch=1024, lr=2e-3)
    rep = net.step(2, judge_every=1000, tol=1e9)  # the first step judges, the second is learned
    assert rep["learned_steps"] == 1
    n = 32 * 32 * 24
    tc = sim.checkpoint().cpu().numpy()[9 * n:10 * n]  # the step's Cs^2 (checkpoint field 9)
    cuda_core, _ = net.infer()
    cc = cuda_core.cpu().numpy().reshape(-1)
    scale = float(np.abs(cc).max())
    err_max = float(np.abs(tc - cc).max()) / scale
    err_mean = float(np.abs(tc - cc).mean()) / scale
    report_line(f"learned Cs^2, tensor-core vs CUDA-core inference: max {err_max:.1e}, "
                f"mean {err_mean:.1e} of the largest value")
    assert err_max <= 1e-2 and err_mean <= 1e-3
