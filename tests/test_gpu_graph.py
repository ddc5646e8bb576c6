"""CUDA-graph batches of the device-driven Arnoldi loop (fvm_opts.graph):
the graph replays the same kernels on the same data in the same order, with
cj and the operator's cj shift read from device memory, so an integration
with it must reproduce the launched-kernel integration bit for bit."""
import numpy as np
import pytest
import torch

import fvmpor_b200 as fb

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("problem,kw,opts", [
    ("richards2d", {}, dict(precision=1)),
    ("richards2d", {}, dict(precision=0)),
    ("richards2d", {}, dict(precision=1, krylov_operator=1, psetup_age=1)),
    ("richards3d", dict(nx=30, ny=30, nz=10, Lx=30.0, Ly=30.0, Lz=10.0), dict(precision=1)),
])
def test_graph_batches_reproduce_launched_batches(problem, kw, opts, cuda):
    p = fb.make_problem(problem, **kw)
    ph = fb.Physics(p)
    y0 = torch.empty(p.n_nodes, dtype=torch.float64, device=cuda)
    ph.initial_head(y0)
    out = {}
    for graph in (0, 1):
        # a tight Krylov tolerance makes every solve run past the first two
        # steps into full 8-step batches, which the graph replays
        integ = fb.Integrator(ph, krylov_dim=30, max_order=5, max_steps=60, graph=graph, eps_lin=1e-8, **opts)
        ye = torch.empty_like(y0)
        rc, st = integ.integrate(0.0, 86400.0, y0, ye)
        assert rc in (0, 1), st
        out[graph] = (ye.cpu().numpy(), st)
    assert np.array_equal(out[0][0], out[1][0])
    for k in ("nst", "nni", "nli", "npe", "nre"):
        assert out[0][1][k] == out[1][1][k], k
    import ctypes as C

    cap, rep = C.c_long(), C.c_long()
    fb.lib().fvm_graph_counters(ph._c, C.byref(cap), C.byref(rep))
    # the 3D problem's solves run into full batches; the graph serves them
    if problem == "richards3d":
        assert cap.value >= 1 and rep.value > cap.value, (cap.value, rep.value)
    ph.close()
