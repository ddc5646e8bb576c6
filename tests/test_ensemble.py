"""Batched ensemble (independent 2D members in one context): the generator's
member ranges, residual parity of the union against the oracle, and the
union integration against each member integrated on its own."""
import numpy as np
import pytest
import torch

import fvmpor_b200 as fb
from oracle.pyoracle import Oracle


def small_ensemble():
    return fb.Problem("ensemble2d", n_members=4, nmin=300, nmax=900, seed=3)


def test_ensemble_members_are_disjoint():
    p = small_ensemble()
    mp = p.member_ptr
    assert mp[0] == 0 and mp[-1] == p.n_nodes and np.all(np.diff(mp) > 0)
    a = p.arrays()
    owner = np.searchsorted(mp, np.arange(p.n_nodes), side="right") - 1
    eo = owner[a["elem_nodes"]]
    assert np.all(eo == eo[:, :1]), "an element couples two members"
    bo = owner[a["bface_nodes"]]
    assert np.all(bo == bo[:, :1]), "a boundary face couples two members"
    # every member is a complete copy of the 2D problem: both boundary tags
    for m in range(len(mp) - 1):
        tags = set(a["bface_tag"][bo[:, 0] == m].tolist())
        assert tags == {1, 2}, (m, tags)
    # members have their own node counts within the requested range (the
    # grid rounds to whole rows)
    n = np.diff(mp)
    assert n.min() >= 250 and n.max() <= 1000


def test_ensemble_full_size_counts():
    p = fb.Problem("ensemble2d", n_members=256, nmin=2000, nmax=40000, seed=1)
    n = np.diff(p.member_ptr)
    assert len(n) == 256 and n.min() >= 1800 and n.max() <= 41000
    assert 4.0e6 < p.n_nodes < 7.0e6


def state(p, seed):
    a = p.arrays()
    y = p.water_table - a["coords"][:, 1] + 0.05 * np.random.default_rng(seed).standard_normal(p.n_nodes)
    tag = a["node_tag"]
    y[tag == 2] = 0.0
    return y, np.random.default_rng(seed + 1).standard_normal(p.n_nodes) * 1e-6


@pytest.mark.gpu
def test_ensemble_residual_parity(cuda):
    p = small_ensemble()
    ph = fb.Physics(p)
    orc = Oracle(p)
    y, yp = state(p, 2)
    res = torch.empty(p.n_nodes, dtype=torch.float64, device=cuda)
    ph.residual(0.0, torch.as_tensor(y, device=cuda), torch.as_tensor(yp, device=cuda), res)
    ref = orc.residual(0.0, y, yp)
    scale = np.abs(ref) + 1e-3 * np.abs(ref).max() + np.abs(orc.ahh() * yp)
    assert (np.abs(res.cpu().numpy() - ref) / scale).max() < 1e-11


@pytest.mark.gpu
def test_ensemble_matches_members_integrated_alone(cuda):
    p = small_ensemble()
    ph = fb.Physics(p)
    y0 = torch.empty(p.n_nodes, dtype=torch.float64, device=cuda)
    ph.initial_head(y0)
    yu = torch.empty_like(y0)
    integ = fb.Integrator(ph, krylov_dim=30, precision=1)
    rc, st = integ.integrate(0.0, 3600.0, y0, yu)
    assert rc == 0
    yu = yu.cpu().numpy()
    mp = p.member_ptr
    for m in range(len(mp) - 1):
        q = p.member(m)
        phm = fb.Physics(q)
        y0m = torch.empty(q.n_nodes, dtype=torch.float64, device=cuda)
        phm.initial_head(y0m)
        ym = torch.empty_like(y0m)
        rc, _ = fb.Integrator(phm, krylov_dim=30, precision=1).integrate(0.0, 3600.0, y0m, ym)
        assert rc == 0
        ym = ym.cpu().numpy()
        span = np.abs(ym).max()
        err = np.abs(yu[mp[m]:mp[m + 1]] - ym).max() / span
        # both runs meet rtol = atol = 1e-6 per member, with different steps
        assert err < 1e-4, (m, err)


@pytest.mark.gpu
def test_sixteen_members_of_the_configured_sizes(cuda):
    # 16 members drawn from the configured size range (2k-40k nodes each):
    # the union's residual against the oracle, then a one-hour union run
    # (FP32 preconditioner, per-member Newton and error tests, the Krylov
    # tolerance scaled to the smallest member) against every member
    # integrated on its own
    p = fb.Problem("ensemble2d", n_members=16, nmin=2000, nmax=40000, seed=5)
    mp = p.member_ptr
    n = np.diff(mp)
    assert len(n) == 16 and n.min() < 10000 and n.max() > 25000
    ph = fb.Physics(p)
    orc = Oracle(p)
    y, yp = state(p, 4)
    res = torch.empty(p.n_nodes, dtype=torch.float64, device=cuda)
    ph.residual(0.0, torch.as_tensor(y, device=cuda), torch.as_tensor(yp, device=cuda), res)
    ref = orc.residual(0.0, y, yp)
    scale = np.abs(ref) + 1e-3 * np.abs(ref).max() + np.abs(orc.ahh() * yp)
    assert (np.abs(res.cpu().numpy() - ref) / scale).max() < 1e-11
    del orc
    y0 = torch.empty(p.n_nodes, dtype=torch.float64, device=cuda)
    ph.initial_head(y0)
    yu = torch.empty_like(y0)
    rc, st = fb.Integrator(ph, krylov_dim=30, precision=1).integrate(0.0, 3600.0, y0, yu)
    assert rc == 0, st
    yu = yu.cpu().numpy()
    for m in range(len(mp) - 1):
        q = p.member(m)
        phm = fb.Physics(q)
        y0m = torch.empty(q.n_nodes, dtype=torch.float64, device=cuda)
        phm.initial_head(y0m)
        ym = torch.empty_like(y0m)
        rc, _ = fb.Integrator(phm, krylov_dim=30, precision=1).integrate(0.0, 3600.0, y0m, ym)
        assert rc == 0
        ym = ym.cpu().numpy()
        err = np.abs(yu[mp[m]:mp[m + 1]] - ym).max() / np.abs(ym).max()
        assert err < 1e-4, (m, n[m], err)
        phm.close()
    ph.close()
