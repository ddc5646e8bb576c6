"""Tensor-core MLP of the learned Newton iterate against its numpy oracle
(oracle/mlp_ref.py): forward values, full-batch gradients, training, and the
integrator's use of the learned iterate with the residual fallback.

Tolerances: the device rounds layer inputs to BF16 at the same points as the
oracle, but its FP32 accumulation order differs, so an activation can land
one BF16 ulp away (2^-8 relative); outputs agree to 1e-2 of their range,
gradients to 5e-2 in relative norm per parameter block."""
import numpy as np
import pytest
import torch

import fvmpor_b200 as fb
from oracle import mlp_ref

pytestmark = pytest.mark.gpu


def ctx():
    p = fb.make_problem("richards2d", nx=21, ny=11)
    return p, fb.Physics(p)


def params(seed=1):
    rng = np.random.default_rng(seed)
    mu = rng.normal(0, 1, 8).astype(np.float32)
    sd = (rng.random(8) + 0.5).astype(np.float32)
    return mlp_ref.init_params(seed, mu, sd), mu, sd


def test_forward_matches_oracle(cuda):
    _, ph = ctx()
    pr = fb.Predictor(ph)
    P, mu, sd = params()
    pr.set_params(P)
    assert np.array_equal(pr.get_params(), P)
    rng = np.random.default_rng(0)
    for n in (1000, 128, 77):
        X = (mu + sd * rng.standard_normal((n, 8))).astype(np.float32)
        out = torch.empty(n, dtype=torch.float32, device=cuda)
        assert pr.forward(torch.as_tensor(X, device=cuda), out) == 0
        ref = mlp_ref.forward(P, X)
        err = np.abs(out.cpu().numpy() - ref).max() / max(np.abs(ref).max(), 1e-6)
        assert err < 1e-2, (n, err)


def test_gradient_matches_oracle(cuda):
    _, ph = ctx()
    pr = fb.Predictor(ph)
    P, mu, sd = params(3)
    pr.set_params(P)
    rng = np.random.default_rng(4)
    n = 640
    X = (mu + sd * rng.standard_normal((n, 8))).astype(np.float32)
    Y = rng.standard_normal(n).astype(np.float32)
    g, loss, rc = pr.grad(torch.as_tensor(X, device=cuda), torch.as_tensor(Y, device=cuda))
    assert rc == 0
    g0, loss0 = mlp_ref.grad(P, X, Y)
    assert abs(loss - loss0) < 1e-3 * loss0
    blocks = [(mlp_ref.OFF_W1, mlp_ref.OFF_B1), (mlp_ref.OFF_B1, mlp_ref.OFF_W2), (mlp_ref.OFF_W2, mlp_ref.OFF_B2),
              (mlp_ref.OFF_B2, mlp_ref.OFF_W3), (mlp_ref.OFF_W3, mlp_ref.OFF_B3), (mlp_ref.OFF_B3, mlp_ref.OFF_W4),
              (mlp_ref.OFF_W4, mlp_ref.OFF_B4), (mlp_ref.OFF_B4, mlp_ref.N_TRAIN)]
    for a, b in blocks:
        rel = np.linalg.norm(g[a:b] - g0[a:b]) / max(np.linalg.norm(g0[a:b]), 1e-12)
        assert rel < 5e-2, (a, b, rel)


def test_training_reduces_loss(cuda):
    _, ph = ctx()
    pr = fb.Predictor(ph)
    rng = np.random.default_rng(5)
    n = 30000
    X = rng.standard_normal((n, 8)).astype(np.float32)
    Y = (np.sin(X[:, 0]) + 0.5 * X[:, 1] * X[:, 2] - 0.3 * X[:, 3]).astype(np.float32)
    P = mlp_ref.init_params(6, np.zeros(8, np.float32), np.ones(8, np.float32))
    pr.set_params(P)
    Xt, Yt = torch.as_tensor(X, device=cuda), torch.as_tensor(Y, device=cuda)
    _, l0, _ = pr.grad(Xt, Yt)
    rc, hist = pr.train(Xt, Yt, epochs=30, batch=4096, lr=3e-3)
    assert rc == 0
    _, l1, _ = pr.grad(Xt, Yt)
    assert l1 < 0.2 * l0, (l0, l1, hist)


def test_learned_iterate_in_the_integrator(cuda):
    p, ph = ctx()
    y0 = torch.empty(p.n_nodes, dtype=torch.float64, device=cuda)
    ph.initial_head(y0)
    plain = fb.Integrator(ph, krylov_dim=20)
    cap = 400_000
    X = torch.zeros((cap, 8), dtype=torch.float32, device=cuda)
    Y = torch.zeros(cap, dtype=torch.float32, device=cuda)
    y_plain = torch.empty_like(y0)
    rc, st, cnt = plain.integrate_record(0.0, 7200.0, y0, y_plain, X, Y, stride=1)
    assert rc == 0 and cnt > 1000
    Xn, Yn = X[:cnt].cpu().numpy(), Y[:cnt].cpu().numpy()
    mu, sd = Xn.mean(0), Xn.std(0) + 1e-6
    pr = fb.Predictor(ph)
    pr.set_params(mlp_ref.init_params(7, mu, sd))
    perm = torch.randperm(cnt, device=cuda)
    rc, hist = pr.train(X[:cnt][perm].contiguous(), Y[:cnt][perm].contiguous(), epochs=20, batch=2048, lr=2e-3)
    assert rc == 0 and hist[-1] < hist[0]
    # the learned iterate is tried on retries after a failed corrector; a
    # one-hour first step makes the corrector fail early in the run
    plain_h0 = fb.Integrator(ph, krylov_dim=20, h0=3600.0)
    rc, st = plain_h0.integrate(0.0, 7200.0, y0, y_plain)
    assert rc == 0
    learned = fb.Integrator(ph, krylov_dim=20, use_predictor=1, h0=3600.0)
    y_learn = torch.empty_like(y0)
    ph.profile(True)
    rc, st2 = learned.integrate(0.0, 7200.0, y0, y_learn)
    attempts = ph.profile_read()["learned_attempt"][1]
    ph.profile(False)
    assert rc == 0
    assert st2["ncfn"] > 0
    tr = learned.trace()
    assert len(tr) == st2["nst"] and int(tr["learned"].sum()) == st2["npred"]
    assert int(tr["nli"].sum()) <= st2["nli"]
    # the learned iterate only changes where Newton starts: both runs solve
    # the same BDF problem to the same tolerance
    span = y_plain.abs().max().item()
    assert (y_plain - y_learn).abs().max().item() < 1e-4 * span
    # what the trained network gains over the plain predictor on this
    # problem: how often it was tried and how often the residual test kept
    # its iterate, and the Krylov and Newton work beside the plain run's
    assert attempts > 0   # one per retry after a failed corrector, outside the back-off
    gain = {"attempts": attempts, "accepted_steps": st2["npred"], "steps": st2["nst"],
            "krylov_per_newton_learned": st2["nli"] / st2["nni"], "krylov_per_newton_plain": st["nli"] / st["nni"],
            "newton_per_step_learned": st2["nni"] / st2["nst"], "newton_per_step_plain": st["nni"] / st["nst"]}
    print("learned-iterate gain", gain)
    assert gain["krylov_per_newton_learned"] < 1.5 * gain["krylov_per_newton_plain"]
    # replay A/B: the learned run's accepted steps replayed with the learned
    # start tried on every step and without it, each corrector solved to
    # ||delta|| <= 1e-4; both must reach the same state (the learned start
    # only moves where Newton begins), and the trace must mark the kept starts
    h0 = float(tr["h"][0])
    ys = {}
    work = {}
    for up in (0, 2):
        rep = fb.Integrator(ph, krylov_dim=20, use_predictor=up)
        yr = torch.empty_like(y0)
        rc, st3 = rep.replay(0.0, y0, h0, tr, yr, newton_tol=1e-4)
        assert rc == 0
        rt = rep.trace()
        assert int(rt["learned"].sum()) == st3["npred"]
        if up == 0:
            assert st3["npred"] == 0
        ys[up] = yr
        work[up] = {"krylov": st3["nli"], "newton": st3["nni"], "kept": st3["npred"]}
    print("replay A/B (plain, learned on every step)", work)
    assert (ys[0] - ys[2]).abs().max().item() < 1e-6 * span
