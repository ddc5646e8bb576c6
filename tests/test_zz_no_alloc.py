"""fvm_wrms_noalloc: the allocation-free WRMS norm, for callers that cannot
call cudaMalloc (their device memory comes from their own pool and the norm
runs inside their step loop).  Checked through the C ABI against the
existing fvm_wrms on two calls in a row; collected last so that a run that
stops at its first failure has already run every other test."""
import ctypes as C

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
        rc = L.fvm_wrms_noalloc(C.c_void_p(x.data_ptr()), C.c_void_p(w.data_ptr()), p.n_nodes,
                                C.c_void_p(out.data_ptr()), None)
        assert rc == 0, L.fvm_last_error()
        torch.cuda.synchronize()
        got = out.item()
        # both reduce in FP64 with fixed orders but different block partitions
        assert abs(got - ref) <= 1e-13 * ref, (call, got, ref)


def test_noalloc_wrms_rejects_oversize(cuda):
    L = _abi()
    nmax = L.fvm_wrms_noalloc_max_n()
    assert nmax == 8_388_608
    x = torch.zeros(1, dtype=torch.float64, device=cuda)
    rc = L.fvm_wrms_noalloc(C.c_void_p(x.data_ptr()), None, nmax + 1, C.c_void_p(x.data_ptr()), None)
    assert rc < 0
    assert b"exceeds the static scratch limit" in L.fvm_last_error()
