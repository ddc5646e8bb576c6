"""GPU-vs-oracle parity on the benchmark configurations at their stated
sizes (through the C ABI).

* The 200k-node 3D box (214,221 nodes, 1.2 M tetrahedra): one residual, one
  J*v, one preconditioner set-up (every Jacobian entry) and one
  preconditioner apply on identical matrices, against the FP64 oracle, with
  the tolerances of tests/test_gpu_parity.py.
* The 2D problem as configured (81 x 41 nodes, 1 day, GMRES(30)):
  adaptive runs in FP64 and FP32 against the oracle's adaptive run, then the
  step-sequence replay: the GPU's accepted steps replayed by the GPU (FP64
  and FP32 preconditioner and basis, and the FP32 path whose Krylov operator
  is the assembled Jacobian in one fused launch per GMRES cycle) and by the
  oracle's independent
  Lagrange-form BDF step, every corrector solved to ||delta||_wrms <= 1e-5
  (about 1e-11 m on these heads).  With the step sizes and orders fixed,
  the states must agree to 1e-10 relative, the FP32 path included: it keeps
  the FP64 residual, Newton update and tests, so its precision only slows
  the Krylov solves.
* The 3D box's first steps replayed the same way.
"""
import numpy as np
import pytest
import torch

import fvmpor_b200 as fb
from oracle.pyoracle import Oracle, factor_given

pytestmark = pytest.mark.gpu

REPLAY_TOL = 1e-10   # max |h_gpu - h_oracle| / max |h_oracle| after a replay
# the GPU paths: plain FP64, FP32 factor and basis, and the FP32 path whose
# Krylov operator is the assembled Jacobian (fused cycle)
PATHS = {"fp64": dict(precision=0), "fp32": dict(precision=1),
         "fp32_assembled": dict(precision=1, krylov_operator=1)}


def T(x, dev):
    return torch.as_tensor(np.ascontiguousarray(x, np.float64), device=dev)


@pytest.fixture(scope="module")
def box(cuda):
    p = fb.make_problem("richards3d")
    assert (p.n_nodes, p.n_elements) == (214221, 1200000)
    ph = fb.Physics(p)
    orc = Oracle(p)
    a = p.arrays()
    rng = np.random.default_rng(31)
    y = p.water_table - a["coords"][:, 2] + 0.05 * rng.standard_normal(p.n_nodes)
    fixed = a["node_tag"] != 0
    y[fixed] = (p.water_table - a["coords"][:, 2])[fixed]
    yp = 1e-7 * rng.standard_normal(p.n_nodes)
    yield p, ph, orc, y, yp
    ph.close()


def row_scale(orc, y, yp):
    r = orc.residual(0.0, y, yp)
    return np.abs(r) + 1e-3 * np.abs(r).max() + np.abs(orc.ahh() * yp)


def test_box_residual_and_jv(box, cuda):
    p, ph, orc, y, yp = box
    yt, ypt = T(y, cuda), T(yp, cuda)
    res = torch.empty_like(yt)
    ph.residual(0.0, yt, ypt, res)
    S = row_scale(orc, y, yp)
    ref = orc.residual(0.0, y, yp)
    err = np.abs(res.cpu().numpy() - ref) / S
    assert err.max() < 1e-11, err.max()
    # frozen upwinding, then J*v
    ph.begin_step(0.0, yt, ypt)
    orc.begin_step(0.0, y, yp)
    F0 = orc.residual(0.0, y, yp)
    v = np.random.default_rng(32).standard_normal(p.n_nodes)
    sigma, cj = 1e-5, 3e-3
    out = torch.empty_like(yt)
    ph.jv(0.0, cj, yt, ypt, T(F0, cuda), T(v, cuda), sigma, out)
    ref = orc.jv(0.0, cj, y, yp, F0, v, sigma)
    err = np.abs(out.cpu().numpy() - ref) / (row_scale(orc, y, yp) / sigma)
    assert err.max() < 1e-9, err.max()


@pytest.mark.parametrize("precision", [0, 1])
def test_box_psetup_and_psolve(box, precision, cuda):
    p, ph, orc, y, yp = box
    yt, ypt = T(y, cuda), T(yp, cuda)
    ph.begin_step(0.0, yt, ypt)
    orc.begin_step(0.0, y, yp)
    F0 = orc.residual(0.0, y, yp)
    ewt = 1.0 / (1e-6 * np.abs(y) + 1e-6)
    cj, h = 2e-3, 500.0
    pc = fb.Preconditioner(ph)
    assert pc.setup(0.0, cj, h, yt, ypt, T(F0, cuda), T(ewt, cuda), precision) == 0
    nb = pc.info()["nblocks"]
    assert orc.psetup(0.0, cj, h, y, yp, F0, ewt, nb) == 0
    rp, col, val = pc.jacobian()
    orp, ocol, oval, colour = orc.jacobian()
    assert np.array_equal(rp, orp) and np.array_equal(col, ocol)
    assert pc.info()["ncolours"] == colour.max() + 1
    if precision == 0:
        rows = np.repeat(np.arange(p.n_nodes), np.diff(rp))
        rmax = np.maximum.reduceat(np.abs(oval), rp[:-1])
        d = np.sqrt(np.finfo(float).eps) * np.maximum(np.abs(y), np.maximum(np.abs(h * yp), 1.0 / ewt))
        S = row_scale(orc, y, yp)
        tol = 1e-6 * rmax[rows] + 5e-13 * S[rows] / d[col]
        assert (np.abs(val - oval) / tol).max() < 1.0
    # the apply on the identical matrix (the device's FD values, which the
    # FP32 set-up forms in FP32 slots)
    assert factor_given(orc, val, nb) == 0
    r = np.random.default_rng(33).standard_normal(p.n_nodes)
    z = torch.empty_like(yt)
    pc.apply(T(r, cuda), z)
    ref = orc.psolve(r)
    err = np.abs(z.cpu().numpy() - ref).max() / np.abs(ref).max()
    assert err < (1e-10 if precision == 0 else 2e-4), err


@pytest.fixture(scope="module")
def plane(cuda):
    p = fb.make_problem("richards2d")
    assert p.n_nodes == 81 * 41
    ph = fb.Physics(p)
    orc = Oracle(p)
    y0 = torch.empty(p.n_nodes, dtype=torch.float64, device=cuda)
    ph.initial_head(y0)
    yield p, ph, orc, y0
    ph.close()


def test_plane_one_day_adaptive_and_replay(plane, cuda):
    p, ph, orc, y0 = plane
    day = 86400.0
    ends, traces = {}, {}
    for key, kw in PATHS.items():
        integ = fb.Integrator(ph, krylov_dim=30, max_order=5, **kw)
        ye = torch.empty_like(y0)
        rc, st = integ.integrate(0.0, day, y0, ye)
        assert rc == 0 and abs(st["t"] - day) < 1e-6, (key, st)
        ends[key], traces[key] = ye.cpu().numpy(), integ.trace()
    nb = fb.Preconditioner(ph).info()["nblocks"]   # the partition the runs used
    y0h = y0.cpu().numpy()
    rc, yo, st_o = orc.integrate(fb.default_opts(krylov_dim=30, max_order=5), nb, 0.0, day, y0h)
    assert rc == 0, st_o
    span = np.abs(yo).max()
    # adaptive runs: each meets rtol = atol = 1e-6 on its own step sequence
    for key in PATHS:
        assert np.abs(ends[key] - yo).max() < 1e-4 * span, (key, np.abs(ends[key] - yo).max())
    # replay of the FP64 run's steps with tight correctors
    tr = traces["fp64"]
    h0 = float(tr["h"][0])
    rc, yr, st_r = orc.replay(fb.default_opts(krylov_dim=30, max_order=5), nb, 0.0, y0h, h0, tr, newton_tol=1e-5)
    assert rc == 0
    for key, kw in PATHS.items():
        integ = fb.Integrator(ph, krylov_dim=30, max_order=5, **kw)
        yg = torch.empty_like(y0)
        rc, st = integ.replay(0.0, y0, h0, tr, yg, newton_tol=1e-5)
        assert rc == 0 and st["nst"] == len(tr)
        err = np.abs(yg.cpu().numpy() - yr).max() / np.abs(yr).max()
        assert err <= REPLAY_TOL, (key, err)


def test_box_first_steps_replay(box, cuda):
    p, ph, orc, _, _ = box
    y0 = torch.empty(p.n_nodes, dtype=torch.float64, device=cuda)
    ph.initial_head(y0)
    integ = fb.Integrator(ph, krylov_dim=40, max_order=5, max_steps=8)
    ye = torch.empty_like(y0)
    rc, st = integ.integrate(0.0, 30 * 86400.0, y0, ye)
    assert rc == 1 and st["nst"] == 8
    tr = integ.trace()
    h0 = float(tr["h"][0])
    nb = fb.Preconditioner(ph).info()["nblocks"]
    y0h = y0.cpu().numpy()
    rc, yr, _ = orc.replay(fb.default_opts(krylov_dim=40, max_order=5), nb, 0.0, y0h, h0, tr, newton_tol=1e-5)
    assert rc == 0
    for key, kw in PATHS.items():
        rep = fb.Integrator(ph, krylov_dim=40, max_order=5, **kw)
        yg = torch.empty_like(y0)
        rc, st = rep.replay(0.0, y0, h0, tr, yg, newton_tol=1e-5)
        assert rc == 0
        err = np.abs(yg.cpu().numpy() - yr).max() / np.abs(yr).max()
        assert err <= REPLAY_TOL, (key, err)


@pytest.mark.parametrize("key", ["fp64", "fp32_assembled"])
def test_box_runs_are_bitwise_reproducible(box, key, cuda):
    """Inside the integrator the preconditioner set-up runs on a second
    stream beside the step's first residual evaluation; the fork and the
    join must leave every run's results unchanged.  Two 3-day runs on the
    3D box give the same state, step sequence and counters, bit for bit, and
    the same as a run with the per-category timers on (one stream)."""
    p, ph, _, _, _ = box
    y0 = torch.empty(p.n_nodes, dtype=torch.float64, device=cuda)
    ph.initial_head(y0)
    out = []
    for profiled in (False, False, True):
        integ = fb.Integrator(ph, krylov_dim=40, max_order=5, **PATHS[key])
        ye = torch.empty_like(y0)
        if profiled:
            ph.profile(True)
        rc, st = integ.integrate(0.0, 3 * 86400.0, y0, ye)
        if profiled:
            ph.profile(False)
        assert rc == 0
        tr = integ.trace()
        out.append((ye.cpu().numpy(), np.asarray(tr["h"]), {k: st[k] for k in ("nst", "nni", "nli", "npe", "nre")}))
    for ye, h, st in out[1:]:
        assert np.array_equal(ye, out[0][0])
        assert np.array_equal(h, out[0][1])
        assert st == out[0][2]
