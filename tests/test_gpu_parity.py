"""Parity of the sm_100a kernels (through the C ABI) with the FP64 CPU oracle.

Tolerances (FP64 throughout): residuals agree to 1e-11 of the per-row flux
scale (the kernels sum the same face fluxes in a different order and with
pre-contracted geometry, so only rounding differs); Jacobian entries, which
are difference quotients with shifts of sqrt(eps)|y|, to 1e-5 of the row
scale; preconditioner applies on identical matrices to 1e-10; integrated
heads to 1e-4 of the head range (both runs converge Newton to 0.33 of the
1e-6 local error tolerance, so they agree to that level, not bitwise).
"""
import numpy as np
import pytest
import torch

import fvmpor_b200 as fb
from oracle.pyoracle import Oracle, factor_given

pytestmark = pytest.mark.gpu


def T(x, dev):
    return torch.as_tensor(np.ascontiguousarray(x, np.float64), device=dev)


def state(p, seed=0, noise=0.05):
    a = p.arrays()
    vert = a["coords"][:, 1 if p.mesh.dim == 2 else 2]
    rng = np.random.default_rng(seed)
    y = p.water_table - vert + noise * rng.standard_normal(p.n_nodes)
    fixed = a["node_tag"] != 0
    y[fixed] = (p.water_table - vert)[fixed]
    if p.mesh.dim == 2:
        y[a["node_tag"] == 2] = 0.0
    yp = 1e-6 * rng.standard_normal(p.n_nodes)
    return y, yp


def row_scale(orc, p, y, yp):
    """per-row magnitude of the flux terms: |F| with all fluxes made positive
    is not available, so use |F| + max|F| * 1e-3 + |ahh y'| as the scale"""
    r = orc.residual(0.0, y, yp)
    return np.abs(r) + 1e-3 * np.abs(r).max() + np.abs(orc.ahh() * yp)


PROBLEMS = {
    "2d_two_zones": lambda: fb.make_problem("richards2d", nx=41, ny=21),
    "2d_lognormal": lambda: fb.Problem("2d", nx=33, ny=17, ln_var=1.0, corr_len=1.0, seed=5),
    "3d_lognormal": lambda: fb.make_problem("richards3d", nx=12, ny=10, nz=6, Lx=12.0, Ly=10.0, Lz=6.0),
}


@pytest.fixture(scope="module", params=list(PROBLEMS))
def case(request):
    return request.param, PROBLEMS[request.param]()


@pytest.mark.parametrize("flags", [fb.FLAG_STORED_GEOMETRY, fb.FLAG_RECOMPUTE_GEOMETRY])
def test_residual_parity(case, flags, cuda):
    name, p = case
    if flags == fb.FLAG_RECOMPUTE_GEOMETRY and p.mesh.dim == 2:
        pytest.skip("geometry recompute is a 3D variant")
    ph = fb.Physics(p, flags)
    orc = Oracle(p)
    for seed in range(3):
        y, yp = state(p, seed)
        res = torch.empty(p.n_nodes, dtype=torch.float64, device=cuda)
        ph.residual(0.0, T(y, cuda), T(yp, cuda), res)
        ref = orc.residual(0.0, y, yp)
        err = np.abs(res.cpu().numpy() - ref) / row_scale(orc, p, y, yp)
        assert err.max() < 1e-11, (name, seed, err.max())


def test_element_pass_chunks_and_autotune(case, cuda):
    """every chunk size and geometry variant gives the oracle's residual;
    each is bitwise reproducible run to run; the autotuner keeps one"""
    name, p = case
    ph = fb.Physics(p)
    orc = Oracle(p)
    y, yp = state(p, 4)
    ref = orc.residual(0.0, y, yp)
    scale = row_scale(orc, p, y, yp)
    res = torch.empty(p.n_nodes, dtype=torch.float64, device=cuda)
    variants = (0, 1) if p.mesh.dim == 3 else (0,)
    for v in variants:
        for ch in (64, 200, 512, 1024):
            ph.set_element_pass(v, ch)
            assert ph.element_pass() == (v, ch)
            ph.residual(0.0, T(y, cuda), T(yp, cuda), res)
            a = res.cpu().numpy()
            ph.residual(0.0, T(y, cuda), T(yp, cuda), res)
            assert np.array_equal(a, res.cpu().numpy()), (name, v, ch)
            err = np.abs(a - ref) / scale
            assert err.max() < 1e-11, (name, v, ch, err.max())
    if p.mesh.dim == 2:
        with pytest.raises(fb.FvmError):
            ph.set_element_pass(1, 256)
    with pytest.raises(fb.FvmError):
        ph.set_element_pass(0, 40000)
    table, best = ph.autotune()
    assert len(table) >= 4 and 0 <= best < len(table)
    assert ph.element_pass() == (table[best][0], table[best][1])
    assert all(t[2] > 0 for t in table)
    ph.residual(0.0, T(y, cuda), T(yp, cuda), res)
    assert (np.abs(res.cpu().numpy() - ref) / scale).max() < 1e-11


def test_initial_head_matches_rules(case, cuda):
    name, p = case
    ph = fb.Physics(p)
    y = torch.zeros(p.n_nodes, dtype=torch.float64, device=cuda)
    ph.initial_head(y)
    a = p.arrays()
    vert = a["coords"][:, 1 if p.mesh.dim == 2 else 2]
    yn = y.cpu().numpy()
    free = a["node_tag"] == 0
    assert np.allclose(yn[free], p.water_table - vert[free], rtol=0, atol=1e-14)


def test_residual_is_bitwise_deterministic(case, cuda):
    name, p = case
    ph = fb.Physics(p)
    y, yp = state(p, 11)
    yt, ypt = T(y, cuda), T(yp, cuda)
    r1 = torch.empty_like(yt)
    r2 = torch.empty_like(yt)
    ph.residual(0.0, yt, ypt, r1)
    for _ in range(3):
        ph.residual(0.0, yt, ypt, r2)
        assert torch.equal(r1, r2)


def test_begin_step_upwinding_parity(case, cuda):
    name, p = case
    ph = fb.Physics(p)
    orc = Oracle(p)
    y, yp = state(p, 2, noise=0.2)
    yt, ypt = T(y, cuda), T(yp, cuda)
    ph.begin_step(0.0, yt, ypt)
    orc.begin_step(0.0, y, yp)
    y2, yp2 = state(p, 3, noise=0.2)
    res = torch.empty_like(yt)
    ph.residual(0.0, T(y2, cuda), T(yp2, cuda), res)
    ref = orc.residual(0.0, y2, yp2)
    err = np.abs(res.cpu().numpy() - ref) / row_scale(orc, p, y2, yp2)
    # edges whose averaged flux is at rounding level may pick either node;
    # such an edge carries a flux of that same size, so the bound holds
    assert np.quantile(err, 0.999) < 1e-11 and err.max() < 1e-8, (name, err.max())


def test_jv_parity(case, cuda):
    name, p = case
    ph = fb.Physics(p)
    orc = Oracle(p)
    y, yp = state(p, 4)
    ph.begin_step(0.0, T(y, cuda), T(yp, cuda))
    orc.begin_step(0.0, y, yp)
    F0 = orc.residual(0.0, y, yp)
    v = np.random.default_rng(9).standard_normal(p.n_nodes)
    sigma, cj = 1e-5, 3e-3
    out = torch.empty(p.n_nodes, dtype=torch.float64, device=cuda)
    ph.jv(0.0, cj, T(y, cuda), T(yp, cuda), T(F0, cuda), T(v, cuda), sigma, out)
    ref = orc.jv(0.0, cj, y, yp, F0, v, sigma)
    # (F(y + s v) - F0) / s amplifies the residual rounding by 1/s; the node
    # pass evaluates van Genuchten through shared logarithms rather than the
    # reference's three pow() calls, a few ulp apart near h = 0
    scale = row_scale(orc, p, y, yp) / sigma
    err = np.abs(out.cpu().numpy() - ref) / scale
    assert err.max() < 1e-9, err.max()


def test_jacobian_parity_and_colouring(case, cuda):
    name, p = case
    ph = fb.Physics(p)
    orc = Oracle(p)
    y, yp = state(p, 5)
    yt, ypt = T(y, cuda), T(yp, cuda)
    ph.begin_step(0.0, yt, ypt)
    orc.begin_step(0.0, y, yp)
    F0 = orc.residual(0.0, y, yp)
    F0g = torch.empty_like(yt)
    ph.residual(0.0, yt, ypt, F0g)
    ewt = 1.0 / (1e-6 * np.abs(y) + 1e-6)
    cj, h = 2e-3, 500.0
    pc = fb.Preconditioner(ph)
    assert pc.setup(0.0, cj, h, yt, ypt, F0g, T(ewt, cuda)) == 0
    assert orc.psetup(0.0, cj, h, y, yp, F0, ewt, 1) == 0
    rp, col, val = pc.jacobian()
    orp, ocol, oval, colour = orc.jacobian()
    assert np.array_equal(rp, orp) and np.array_equal(col, ocol)
    assert pc.info()["ncolours"] == colour.max() + 1
    rows = np.repeat(np.arange(p.n_nodes), np.diff(rp))
    rmax = np.maximum.reduceat(np.abs(oval), rp[:-1])
    # each entry is (F(y + d_j) - F0) / d_j: a rounding-level difference in
    # F (relative 1e-14 of the row's flux scale S_i) becomes S_i 1e-14 / d_j,
    # and d_j = sqrt(eps) max(|y_j|, |h y'_j|, 1/w_j) is as small as 1.5e-14
    # on the h = 0 Dirichlet strip (preconditioner_dss.cpp:322-329)
    d = np.sqrt(np.finfo(float).eps) * np.maximum(np.abs(y), np.maximum(np.abs(h * yp), 1.0 / ewt))
    S = row_scale(orc, p, y, yp)
    tol = 1e-6 * rmax[rows] + 5e-13 * S[rows] / d[col]
    err = np.abs(val - oval) / tol
    assert err.max() < 1.0, (name, err.max())


@pytest.mark.parametrize("precision", [0, 1])
def test_psolve_parity_on_identical_matrix(case, precision, cuda):
    name, p = case
    ph = fb.Physics(p)
    orc = Oracle(p)
    y, yp = state(p, 6)
    yt, ypt = T(y, cuda), T(yp, cuda)
    ph.begin_step(0.0, yt, ypt)
    F0 = torch.empty_like(yt)
    ph.residual(0.0, yt, ypt, F0)
    ewt = 1.0 / (1e-6 * np.abs(y) + 1e-6)
    pc = fb.Preconditioner(ph)
    assert pc.setup(0.0, 1e-2, 100.0, yt, ypt, F0, T(ewt, cuda), precision) == 0
    _, _, val = pc.jacobian()
    nb = pc.info()["nblocks"]
    orc.psetup(0.0, 1e-2, 100.0, y, yp, F0.cpu().numpy(), ewt, nb)
    assert factor_given(orc, val, nb) == 0
    r = np.random.default_rng(7).standard_normal(p.n_nodes)
    z = torch.empty_like(yt)
    pc.apply(T(r, cuda), z)
    ref = orc.psolve(r)
    tol = 1e-10 if precision == 0 else 2e-4
    err = np.abs(z.cpu().numpy() - ref).max() / np.abs(ref).max()
    assert err < tol, (name, precision, err)


@pytest.mark.parametrize("per_sm", [1, 2, 4])
def test_psolve_parity_blocks_per_sm(per_sm, cuda):
    """large-mesh block partitions (a multiple of the SM count, per_sm
    blocks per SM) against the oracle's ILU(0) on the same blocks"""
    p = fb.make_problem("richards3d", nx=36, ny=36, nz=30, Lx=36.0, Ly=36.0, Lz=30.0)
    ph = fb.Physics(p)
    orc = Oracle(p)
    y, yp = state(p, 6)
    yt, ypt = T(y, cuda), T(yp, cuda)
    ph.begin_step(0.0, yt, ypt)
    F0 = torch.empty_like(yt)
    ph.residual(0.0, yt, ypt, F0)
    ewt = 1.0 / (1e-6 * np.abs(y) + 1e-6)
    pc = fb.Preconditioner(ph)
    pc.set_blocks_per_sm(per_sm)
    assert pc.setup(0.0, 1e-2, 100.0, yt, ypt, F0, T(ewt, cuda), 0) == 0
    _, _, val = pc.jacobian()
    nb = pc.info()["nblocks"]
    assert nb == per_sm * torch.cuda.get_device_properties(0).multi_processor_count
    orc.psetup(0.0, 1e-2, 100.0, y, yp, F0.cpu().numpy(), ewt, nb)
    assert factor_given(orc, val, nb) == 0
    r = np.random.default_rng(8).standard_normal(p.n_nodes)
    z = torch.empty_like(yt)
    pc.apply(T(r, cuda), z)
    ref = orc.psolve(r)
    err = np.abs(z.cpu().numpy() - ref).max() / np.abs(ref).max()
    assert err < 1e-10, (per_sm, err)


def test_two_live_contexts_of_different_sizes(cuda):
    """kernel launch limits (dynamic shared memory) belong to the kernel for
    the whole process: a small context created after a large one must not
    lower the limits the large one's preconditioner applies need"""
    big = fb.make_problem("richards3d", nx=36, ny=36, nz=30, Lx=36.0, Ly=36.0, Lz=30.0)
    small = fb.make_problem("richards2d", nx=21, ny=11)
    out = {}
    phs = [fb.Physics(big), fb.Physics(small)]
    pcs = []
    for ph, p in zip(phs, (big, small)):
        y, yp = state(p, 6)
        yt, ypt = T(y, cuda), T(yp, cuda)
        ph.begin_step(0.0, yt, ypt)
        F0 = torch.empty_like(yt)
        ph.residual(0.0, yt, ypt, F0)
        ewt = T(1.0 / (1e-6 * np.abs(y) + 1e-6), cuda)
        pcs.append((fb.Preconditioner(ph), yt, ypt, F0, ewt))
    for prec in (0, 1):
        for k, (pc, yt, ypt, F0, ewt) in enumerate(pcs):   # large set up first, then small
            assert pc.setup(0.0, 1e-2, 100.0, yt, ypt, F0, ewt, prec) == 0
        for k, (pc, yt, ypt, F0, ewt) in enumerate(pcs):
            z = torch.empty_like(yt)
            pc.apply(torch.ones_like(yt), z)   # raised on the large context before
            out[(k, prec)] = z.abs().max().item()
    assert all(np.isfinite(v) and v > 0 for v in out.values()), out
    for ph in phs:
        ph.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_gmres_converges_and_matches_oracle(case, precision, cuda):
    name, p = case
    ph = fb.Physics(p)
    orc = Oracle(p)
    y, yp = state(p, 8)
    yt, ypt = T(y, cuda), T(yp, cuda)
    ph.begin_step(0.0, yt, ypt)
    orc.begin_step(0.0, y, yp)
    F0 = orc.residual(0.0, y, yp)
    ewt = 1.0 / (1e-6 * np.abs(y) + 1e-6)
    cj = 1e-2
    pc = fb.Preconditioner(ph)
    pc.setup(0.0, cj, 100.0, yt, ypt, T(F0, cuda), T(ewt, cuda), precision)
    x = torch.empty_like(yt)
    rc, its, rn = pc.gmres(0.0, cj, yt, ypt, T(F0, cuda), T(ewt, cuda), T(F0, cuda), x, m=30, tol=1e-8,
                           precision=precision)
    assert rc == 0 and rn <= 1e-8, (rc, its, rn)
    orc.psetup(0.0, cj, 100.0, y, yp, F0, ewt, pc.info()["nblocks"])
    orc_rc, xo, its_o, rn_o = orc.gmres(cj, y, yp, F0, ewt, F0, m=30, tol=1e-8)
    assert orc_rc == 0
    # both solve J x = F to 1e-8 in the weighted norm: the solutions agree
    # to about that many weighted units
    d = np.sqrt(np.mean(((x.cpu().numpy() - xo) * ewt) ** 2))
    xn = np.sqrt(np.mean((xo * ewt) ** 2))
    assert d < 1e-3 * max(xn, 1.0), (d, xn)


def test_reductions(cuda):
    p = fb.make_problem("richards2d", nx=41, ny=21)
    ph = fb.Physics(p)
    rng = np.random.default_rng(3)
    x, w = rng.standard_normal(p.n_nodes), rng.random(p.n_nodes) + 0.5
    xt, wt = T(x, cuda), T(w, cuda)
    assert abs(ph.wrms(xt, wt) - np.sqrt(np.mean((x * w) ** 2))) < 1e-14
    assert abs(ph.dot(xt, wt) - x @ w) < 1e-11 * np.abs(x * w).sum()
    assert ph.dot(xt, wt) == ph.dot(xt, wt)


@pytest.mark.parametrize("precision", [0, 1])
def test_integration_matches_oracle(precision, cuda):
    p = fb.make_problem("richards2d", nx=21, ny=11)
    ph = fb.Physics(p)
    orc = Oracle(p)
    y0 = torch.empty(p.n_nodes, dtype=torch.float64, device=cuda)
    ph.initial_head(y0)
    opts = dict(krylov_dim=20, max_order=5, precision=precision)
    integ = fb.Integrator(ph, **opts)
    yend = torch.empty_like(y0)
    rc, st = integ.integrate(0.0, 3600.0, y0, yend)
    assert rc == 0, st
    assert abs(st["t"] - 3600.0) < 1e-6
    pc = fb.Preconditioner(ph)
    nb = pc.info()["nblocks"]
    rc_o, yo, st_o = orc.integrate(fb.default_opts(krylov_dim=20, max_order=5), nb, 0.0, 3600.0,
                                   y0.cpu().numpy())
    assert rc_o == 0, st_o
    yg = yend.cpu().numpy()
    span = np.abs(yo).max()
    assert np.abs(yg - yo).max() < 1e-4 * span, (np.abs(yg - yo).max(), st, st_o)


def test_integrate_host_buffers(cuda):
    p = fb.make_problem("richards2d", nx=21, ny=11)
    ph = fb.Physics(p)
    y0 = torch.empty(p.n_nodes, dtype=torch.float64, device=cuda)
    ph.initial_head(y0)
    integ = fb.Integrator(ph, krylov_dim=20)
    yend = np.zeros(p.n_nodes)
    rc, st = integ.integrate_host(0.0, 600.0, y0.cpu().numpy(), yend)
    assert rc == 0 and np.isfinite(yend).all()
    yd = torch.empty_like(y0)
    rc2, st2 = integ.integrate(0.0, 600.0, y0, yd)
    assert np.array_equal(yd.cpu().numpy(), yend)


def test_dense_output_matches_oracle(cuda):
    """fvm_integrate_outputs (whole steps, heads interpolated at the output
    times, IDAIntegrator::advance(next_time)) against the oracle's
    restatement: same tolerance as the stop-time runs"""
    p = fb.make_problem("richards2d", nx=21, ny=11)
    ph = fb.Physics(p)
    orc = Oracle(p)
    y0 = torch.empty(p.n_nodes, dtype=torch.float64, device=cuda)
    ph.initial_head(y0)
    tout = [600.0, 1800.0, 3600.0]
    integ = fb.Integrator(ph, krylov_dim=20, max_order=5)
    Y = torch.empty(len(tout), p.n_nodes, dtype=torch.float64, device=cuda)
    YP = torch.empty_like(Y)
    rc, st = integ.integrate_outputs(0.0, tout, y0, Y, YP)
    assert rc == 0 and st["t"] >= tout[-1], st
    nb = fb.Preconditioner(ph).info()["nblocks"]
    rc_o, Yo, YPo, st_o = orc.integrate_outputs(fb.default_opts(krylov_dim=20, max_order=5), nb, 0.0,
                                                y0.cpu().numpy(), tout)
    assert rc_o == 0, st_o
    Yg, YPg = Y.cpu().numpy(), YP.cpu().numpy()
    span = np.abs(Yo).max()
    assert np.abs(Yg - Yo).max() < 1e-4 * span, (np.abs(Yg - Yo).max(), st, st_o)
    assert np.abs(YPg - YPo).max() < 1e-2 * np.abs(YPo).max(), np.abs(YPg - YPo).max()
    # a stop-time run to the last output time agrees to the same tolerance
    yend = torch.empty_like(y0)
    rc, _ = integ.integrate(0.0, tout[-1], y0, yend)
    assert rc == 0
    assert np.abs(Yg[-1] - yend.cpu().numpy()).max() < 1e-4 * span


def test_dense_output_at_a_step_time_is_the_state(cuda):
    p = fb.make_problem("richards2d", nx=21, ny=11)
    ph = fb.Physics(p)
    y0 = torch.empty(p.n_nodes, dtype=torch.float64, device=cuda)
    ph.initial_head(y0)
    # a fixed first step makes the step sequence independent of the end time
    yk = torch.empty_like(y0)
    rc, stk = fb.Integrator(ph, krylov_dim=20, h0=1.0, max_steps=12).integrate(0.0, 1e9, y0, yk)
    assert rc == 1 and stk["nst"] == 12
    tk, hk = stk["t"], stk["last_h"]
    integ = fb.Integrator(ph, krylov_dim=20, h0=1.0)
    d = 1e-4 * hk
    tout = [tk - d, tk, 3600.0]
    Y = torch.empty(3, p.n_nodes, dtype=torch.float64, device=cuda)
    YP = torch.empty_like(Y)
    rc, st = integ.integrate_outputs(0.0, tout, y0, Y, YP)
    assert rc == 0
    assert torch.equal(Y[1], yk)
    fd = (Y[1] - Y[0]) / d
    assert (fd - YP[1]).abs().max().item() <= 1e-3 * YP[1].abs().max().item() + 1e-12
    # more output times leave the integration unchanged (yp_out optional)
    Y2 = torch.empty(1, p.n_nodes, dtype=torch.float64, device=cuda)
    rc, st2 = integ.integrate_outputs(0.0, [3600.0], y0, Y2)
    assert rc == 0 and torch.equal(Y2[0], Y[2])
    assert (st2["nst"], st2["nli"]) == (st["nst"], st["nli"])
    with pytest.raises(RuntimeError):
        integ.integrate_outputs(0.0, [3600.0, 3600.0], y0, torch.empty_like(Y[:2]))
