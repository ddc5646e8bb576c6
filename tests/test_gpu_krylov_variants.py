"""The two Gram-Schmidt forms of the fused GMRES cycle (the assembled FP32
Krylov operator): classical Gram-Schmidt with reorthogonalisation (two
reductions per Arnoldi step) and delayed reorthogonalisation (one
reduction; the default).  They span the same Krylov space, so replays of
one step sequence with every corrector solved tightly must reach the same
state, and adaptive runs must take about the same work."""
import ctypes as C

import numpy as np
import pytest
import torch

import fvmpor_b200 as fb

pytestmark = pytest.mark.gpu


def set_variant(ph, v):
    assert fb.lib().fvm_set_krylov_variant(ph._c, v) == 0


def test_variants_replay_to_the_same_state_on_the_box(cuda):
    p = fb.make_problem("richards3d")
    ph = fb.Physics(p)
    y0 = torch.empty(p.n_nodes, dtype=torch.float64, device=cuda)
    ph.initial_head(y0)
    integ = fb.Integrator(ph, krylov_dim=40, max_order=5, max_steps=30, precision=1, krylov_operator=1)
    ye = torch.empty_like(y0)
    rc, st = integ.integrate(0.0, 30 * 86400.0, y0, ye)
    assert rc == 1 and st["nst"] == 30
    tr = integ.trace()
    h0 = float(tr["h"][0])
    out = {}
    for v in (0, 1):
        set_variant(ph, v)
        rep = fb.Integrator(ph, krylov_dim=40, max_order=5, precision=1, krylov_operator=1)
        yr = torch.empty_like(y0)
        rc, st = rep.replay(0.0, y0, h0, tr, yr, newton_tol=1e-5)
        assert rc == 0
        out[v] = (yr.cpu().numpy(), st)
    err = np.abs(out[0][0] - out[1][0]).max() / np.abs(out[0][0]).max()
    assert err < 1e-10, err
    # the same Krylov space: the same iteration counts to within a few
    assert abs(out[0][1]["nli"] - out[1][1]["nli"]) <= 0.05 * out[0][1]["nli"] + 2, (out[0][1], out[1][1])
    set_variant(ph, 1)
    ph.close()


def test_variants_adaptive_plane(cuda):
    p = fb.make_problem("richards2d")
    ph = fb.Physics(p)
    y0 = torch.empty(p.n_nodes, dtype=torch.float64, device=cuda)
    ph.initial_head(y0)
    res = {}
    for v in (0, 1):
        set_variant(ph, v)
        integ = fb.Integrator(ph, krylov_dim=30, max_order=5, precision=1, krylov_operator=1)
        ye = torch.empty_like(y0)
        rc, st = integ.integrate(0.0, 86400.0, y0, ye)
        assert rc == 0
        res[v] = (ye.cpu().numpy(), st)
    span = np.abs(res[0][0]).max()
    assert np.abs(res[0][0] - res[1][0]).max() < 1e-4 * span
    assert abs(res[0][1]["nst"] - res[1][1]["nst"]) <= 0.1 * res[0][1]["nst"]
    set_variant(ph, 1)
    ph.close()
