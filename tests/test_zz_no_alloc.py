"""fvm_wrms_noalloc: the allocation-free WRMS norm, for callers that cannot
call cudaMalloc (their device memory comes from their own pool and the norm
runs inside their step loop).  Checked through the C ABI against the
existing fvm_wrms and against an exactly rounded numpy sum, on two calls in
a row, at sizes that fill one block, many blocks and the whole static
scratch, with and without weights; collected last so that a run that stops
at its first failure has already run every other test."""
import ctypes as C
import math

import numpy as np
import pytest
import torch

import fvmpor_b200 as fb

pytestmark = pytest.mark.gpu


def _abi():
    L = fb.lib()
    L.fvm_wrms_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_long, C.c_void_p, C.c_void_p]
    L.fvm_wrms_noalloc.restype = C.c_int
    L.fvm_wrms_noalloc_max_n.restype = C.c_long
    return L


def _exact_wrms(x, w):
    v = x if w is None else x * w
    return math.sqrt(math.fsum((v * v).tolist()) / len(x))


def _call(L, x, w, n, out):
    rc = L.fvm_wrms_noalloc(C.c_void_p(x.data_ptr()), C.c_void_p(w.data_ptr()) if w is not None else None, n,
                            C.c_void_p(out.data_ptr()), None)
    assert rc == 0, L.fvm_last_error()
    torch.cuda.synchronize()
    return out.item()


def test_noalloc_wrms_matches_fvm_wrms_twice(cuda):
    L = _abi()
    p = fb.make_problem("richards2d", nx=41, ny=21)
    ph = fb.Physics(p)
    rng = np.random.default_rng(2)
    out = torch.zeros(1, dtype=torch.float64, device=cuda)
    for call in range(2):
        x = torch.as_tensor(rng.standard_normal(p.n_nodes) * 10.0 ** call, device=cuda)
        w = torch.as_tensor(rng.random(p.n_nodes) + 0.1, device=cuda)
        ref = ph.wrms(x, w)          # existing entry point (context workspace)
        got = _call(L, x, w, p.n_nodes, out)
        # both reduce in FP64 with fixed orders but different block partitions
        assert abs(got - ref) <= 1e-13 * ref, (call, got, ref)
    ph.close()


@pytest.mark.parametrize("n", [3 * 2048 + 5, 5_000_000, "max"])
@pytest.mark.parametrize("weighted", [True, False])
def test_noalloc_wrms_many_blocks_against_exact_sum(n, weighted, cuda):
    """many blocks meet in the last-block reduction; the completion counter
    is re-armed between calls, so two calls in a row both come out right"""
    L = _abi()
    if n == "max":
        n = L.fvm_wrms_noalloc_max_n()
    rng = np.random.default_rng(n % 1000 + weighted)
    out = torch.full((1,), float("nan"), dtype=torch.float64, device=cuda)
    for call in range(2):
        xh = rng.standard_normal(n) * (1.0 + 9.0 * call)
        wh = rng.random(n) + 0.25 if weighted else None
        x = torch.as_tensor(xh, device=cuda)
        w = torch.as_tensor(wh, device=cuda) if weighted else None
        got = _call(L, x, w, n, out)
        ref = _exact_wrms(xh, wh)
        assert abs(got - ref) <= 1e-13 * ref, (n, weighted, call, got, ref)


def test_noalloc_wrms_rejects_oversize(cuda):
    L = _abi()
    nmax = L.fvm_wrms_noalloc_max_n()
    assert nmax == 8_388_608
    x = torch.zeros(1, dtype=torch.float64, device=cuda)
    rc = L.fvm_wrms_noalloc(C.c_void_p(x.data_ptr()), None, nmax + 1, C.c_void_p(x.data_ptr()), None)
    assert rc < 0
    assert b"exceeds the static scratch limit" in L.fvm_last_error()
