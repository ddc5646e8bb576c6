"""Schur interface coupling of the block ILU(0) on the device (through the C
ABI) against the oracle's restatement of decomp/schur.c:1407-1636.

* The coupled apply on identical matrices: the 2D problem as configured
  (81 x 41 nodes, 3 blocks) in FP64 and FP32, and the 3D box (214,221
  nodes, 148 blocks) in FP32, for 0, 1 and 3 interface sweeps.
* GMRES preconditioned by the coupled apply converges on the box.
* A replayed step sequence of the 2D run with the coupled preconditioner
  reaches the oracle's state to 1e-10: the preconditioner changes the
  Krylov solves, not the converged corrector.
"""
import numpy as np
import pytest
import torch

import fvmpor_b200 as fb
from oracle.pyoracle import Oracle, factor_given

pytestmark = pytest.mark.gpu


def T(x, dev):
    return torch.as_tensor(np.ascontiguousarray(x, np.float64), device=dev)


def state(p, seed):
    a = p.arrays()
    vert = a["coords"][:, 1 if p.mesh.dim == 2 else 2]
    rng = np.random.default_rng(seed)
    y = p.water_table - vert + 0.05 * rng.standard_normal(p.n_nodes)
    fixed = a["node_tag"] != 0
    y[fixed] = (p.water_table - vert)[fixed]
    if p.mesh.dim == 2:
        y[a["node_tag"] == 2] = 0.0
    yp = 1e-7 * rng.standard_normal(p.n_nodes)
    return y, yp


def coupled_apply_vs_oracle(p, precision, iters, cuda, seed):
    ph = fb.Physics(p)
    orc = Oracle(p)
    y, yp = state(p, seed)
    yt, ypt = T(y, cuda), T(yp, cuda)
    ph.begin_step(0.0, yt, ypt)
    F0 = torch.empty_like(yt)
    ph.residual(0.0, yt, ypt, F0)
    ewt = 1.0 / (1e-6 * np.abs(y) + 1e-6)
    pc = fb.Preconditioner(ph)
    pc.set_schur(iters)
    assert pc.setup(0.0, 2e-3, 500.0, yt, ypt, F0, T(ewt, cuda), precision) == 0
    info = pc.schur_info()
    assert info["iters"] == iters and info["interface_rows"] > 0
    assert info["fp32" if precision else "fp64"]
    _, _, val = pc.jacobian()
    nb = pc.info()["nblocks"]
    orc.set_schur(iters)
    orc.psetup(0.0, 2e-3, 500.0, y, yp, F0.cpu().numpy(), ewt, nb)
    assert factor_given(orc, val, nb) == 0
    assert orc.schur_interface_rows() == info["interface_rows"]
    r = np.random.default_rng(seed + 1).standard_normal(p.n_nodes)
    z = torch.empty_like(yt)
    pc.apply(T(r, cuda), z)
    ref = orc.psolve(r)
    ph.close()
    return np.abs(z.cpu().numpy() - ref).max() / np.abs(ref).max()


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("iters", [0, 1, 3])
def test_coupled_apply_plane(precision, iters, cuda):
    p = fb.make_problem("richards2d")
    err = coupled_apply_vs_oracle(p, precision, iters, cuda, 40)
    assert err < (1e-10 if precision == 0 else 2e-4), err


@pytest.mark.parametrize("iters", [0, 2])
def test_coupled_apply_box_fp32(iters, cuda):
    p = fb.make_problem("richards3d")
    err = coupled_apply_vs_oracle(p, 1, iters, cuda, 41)
    assert err < 2e-4, err


def test_coupled_gmres_converges_on_box(cuda):
    p = fb.make_problem("richards3d")
    ph = fb.Physics(p)
    y, yp = state(p, 42)
    yt, ypt = T(y, cuda), T(yp, cuda)
    ph.begin_step(0.0, yt, ypt)
    F0 = torch.empty_like(yt)
    ph.residual(0.0, yt, ypt, F0)
    ewt = T(1.0 / (1e-6 * np.abs(y) + 1e-6), cuda)
    pc = fb.Preconditioner(ph)
    its = {}
    for iters in (-1, 2):
        pc.set_schur(iters)
        assert pc.setup(0.0, 2e-3, 500.0, yt, ypt, F0, ewt, 1) == 0
        x = torch.zeros_like(yt)
        rc, n, rn = pc.gmres(0.0, 2e-3, yt, ypt, F0, ewt, F0, x, m=40, precision=1, tol=1e-6)
        assert rc == 0, (iters, n, rn)
        its[iters] = n
    assert its[2] > 0
    ph.close()


def test_coupled_replay_reaches_the_oracle_state(cuda):
    p = fb.make_problem("richards2d")
    ph = fb.Physics(p)
    orc = Oracle(p)
    y0 = torch.empty(p.n_nodes, dtype=torch.float64, device=cuda)
    ph.initial_head(y0)
    integ = fb.Integrator(ph, krylov_dim=30, max_order=5, max_steps=40)
    ye = torch.empty_like(y0)
    rc, st = integ.integrate(0.0, 86400.0, y0, ye)
    assert rc == 1 and st["nst"] == 40
    tr = integ.trace()
    h0 = float(tr["h"][0])
    nb = fb.Preconditioner(ph).info()["nblocks"]
    y0h = y0.cpu().numpy()
    rc, yr, _ = orc.replay(fb.default_opts(krylov_dim=30, max_order=5), nb, 0.0, y0h, h0, tr, newton_tol=1e-5)
    assert rc == 0
    pc = fb.Preconditioner(ph)
    for precision in (0, 1):
        pc.set_schur(2)
        rep = fb.Integrator(ph, krylov_dim=30, max_order=5, precision=precision)
        yg = torch.empty_like(y0)
        rc, st = rep.replay(0.0, y0, h0, tr, yg, newton_tol=1e-5)
        assert rc == 0
        assert pc.schur_info()["iters"] == 2
        err = np.abs(yg.cpu().numpy() - yr).max() / np.abs(yr).max()
        assert err <= 1e-10, (precision, err)
    pc.set_schur(-1)
    ph.close()
