"""GPU tests of the learned SGS coefficient (alfa_mlp_*): the training
gradient and the features against the NumPy restatement, and an end-to-end
run that trains on the dynamic procedure and steps with the network, judged
by the procedure."""
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


def test_learned_closure_trains_and_steps():
    """Train on 20 dynamic steps, then from the same checkpoint run 20 steps
    three ways: the dynamic procedure, the network (judged every 10 steps),
    and the coefficients of the last dynamic step held fixed (the method
    without the network).  The learned steps must be faster than the dynamic
    ones; the errors of the resolved and SGS flux profiles against the
    dynamic run are reported."""
    from jax_alfa_b200.api import Learned, stats_to_dict
    cfg = cases.convective(32, 32, 24, nsteps=60)
    sim = _sim(cfg)
    net = Learned(sim, capacity=60_000, seed=1)
    for _ in range(20):
        sim.step(1)
        net.collect(3000)
    loss = net.train(epochs=60, batch=512, lr=2e-3)
    print(f"training loss after 60 epochs: {loss:.3e} (normalised units)")
    ck = sim.checkpoint()
    P, norm = net.params()

    def run(mode):
        s = _sim(cfg).restore(ck)
        acc = None
        rep = None
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if mode == "learned":
            n2 = Learned(s, capacity=1024)
            n2.set_params(P, norm)
        ev0.record()
        for _ in range(20):
            if mode == "dynamic":
                s.step(1)
            elif mode == "learned":
                rep = n2.step(1, judge_every=10, tol=1.0)
            acc = s.stats_sample(acc)
        ev1.record()
        torch.cuda.synchronize()
        return stats_to_dict(acc, cfg["nz"], cfg["Ugal"]), ev0.elapsed_time(ev1) / 20, rep

    dyn, t_dyn, _ = run("dynamic")
    lrn, t_lrn, rep = run("learned")
    assert rep["learned_steps"] >= 17 and rep["judged"] >= 2
    print(f"step time: dynamic {t_dyn:.2f} ms, learned {t_lrn:.2f} ms "
          f"(judge drift {rep['max_drift']:.3f})")
    for k in ("wTH", "uw", "txz", "qz"):
        e = np.abs(lrn[k] - dyn[k]).max() / np.abs(dyn[k]).max()
        print(f"{k}: learned vs dynamic relative profile error {e:.3e}")
    assert t_lrn < t_dyn
