"""ctypes loader for the FP64 CPU oracle (oracle/oracle.cpp).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the FP64 answer results are compared against
(or the timed CPU baseline) — never by the product.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build():
    subprocess.run(["make", "-C", _HERE], check=True, capture_output=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P, D, I = C.c_void_p, C.c_double, C.c_int
        L.orc_create.restype = P
        L.orc_create.argtypes = [P, P, C.c_char_p, I]
        L.orc_destroy.argtypes = [P]
        L.orc_sizes.argtypes = [P, P, P, P, P]
        for name in ("orc_volumes", "orc_cv_normal_sums", "orc_ahh"):
            getattr(L, name).argtypes = [P, P]
        L.orc_residual.argtypes = [P, D, P, P, P]
        L.orc_begin_step.argtypes = [P, D, P, P]
        L.orc_upwind.argtypes = [P, P]
        L.orc_edges.argtypes = [P, P, P]
        L.orc_jv.argtypes = [P, D, D, P, P, P, P, D, P]
        L.orc_psetup.argtypes = [P, D, D, D, P, P, P, P, I]
        L.orc_jacobian_nnz.argtypes = [P]
        L.orc_jacobian.argtypes = [P, P, P, P, P]
        L.orc_psolve.argtypes = [P, P, P]
        L.orc_gmres.argtypes = [P, D, P, P, P, P, P, P, I, I, D, P, P]
        L.orc_integrate.argtypes = [P, P, I, D, D, P, P, P]
        L.orc_integrate_outputs.argtypes = [P, P, I, D, P, I, P, P, P, P]
        L.orc_interp_coefs.argtypes = [P, I, D, P, P]
        L.orc_threads.restype = I
        _lib = L
    return _lib


def _p(a):
    assert a.dtype in (np.float64, np.int32) and a.flags.c_contiguous
    return a.ctypes.data


class Oracle:
    def __init__(self, problem):
        """problem: fvmpor_b200.Problem (only its mesh/physics description is read)."""
        err = C.create_string_buffer(512)
        self._c = lib().orc_create(C.addressof(problem._s.mesh), C.addressof(problem._s.phys), err, 512)
        if not self._c:
            raise RuntimeError("oracle: " + err.value.decode())
        self.N = problem.n_nodes
        self._problem = problem

    def __del__(self):
        if getattr(self, "_c", None):
            lib().orc_destroy(self._c)
            self._c = None

    def sizes(self):
        v = [C.c_int() for _ in range(4)]
        lib().orc_sizes(self._c, *[C.byref(x) for x in v])
        return dict(zip(("E", "Fi", "Fall", "ncolours"), [x.value for x in v]))

    def volumes(self):
        V = np.zeros(self.N)
        lib().orc_volumes(self._c, _p(V))
        return V

    def cv_normal_sums(self):
        S = np.zeros((self.N, 3))
        lib().orc_cv_normal_sums(self._c, _p(S))
        return S

    def ahh(self):
        a = np.zeros(self.N)
        lib().orc_ahh(self._c, _p(a))
        return a

    def residual(self, t, y, yp):
        r = np.zeros(self.N)
        lib().orc_residual(self._c, t, _p(np.ascontiguousarray(y, np.float64)),
                           _p(np.ascontiguousarray(yp, np.float64)), _p(r))
        return r

    def begin_step(self, t, y, yp):
        lib().orc_begin_step(self._c, t, _p(np.ascontiguousarray(y, np.float64)),
                             _p(np.ascontiguousarray(yp, np.float64)))

    def upwind(self):
        E = self.sizes()["E"]
        w = np.zeros(E, np.int32)
        lib().orc_upwind(self._c, _p(w))
        return w

    def jv(self, t, cj, y, yp, F0, v, sigma):
        out = np.zeros(self.N)
        lib().orc_jv(self._c, t, cj, _p(y), _p(yp), _p(F0), _p(v), sigma, _p(out))
        return out

    def psetup(self, t, cj, h, y, yp, F0, ewt, nblocks):
        return lib().orc_psetup(self._c, t, cj, h, _p(y), _p(yp), _p(F0), _p(ewt), nblocks)

    def jacobian(self):
        nnz = lib().orc_jacobian_nnz(self._c)
        rp = np.zeros(self.N + 1, np.int32)
        col = np.zeros(nnz, np.int32)
        val = np.zeros(nnz)
        colour = np.zeros(self.N, np.int32)
        lib().orc_jacobian(self._c, _p(rp), _p(col), _p(val), _p(colour))
        return rp, col, val, colour

    def psolve(self, r):
        z = np.zeros(self.N)
        lib().orc_psolve(self._c, _p(np.ascontiguousarray(r, np.float64)), _p(z))
        return z

    def gmres(self, cj, y, yp, F0, ewt, b, m=30, max_restarts=5, tol=0.0165):
        x = np.zeros(self.N)
        its, rn = C.c_int(), C.c_double()
        r = lib().orc_gmres(self._c, cj, _p(y), _p(yp), _p(F0), _p(ewt), _p(b), _p(x), m, max_restarts, tol,
                            C.byref(its), C.byref(rn))
        return r, x, its.value, rn.value

    def integrate(self, opts, nblocks, t0, t_end, y0):
        from fvmpor_b200 import Stats

        y_end = np.zeros(self.N)
        st = Stats()
        r = lib().orc_integrate(self._c, C.addressof(opts), nblocks, t0, t_end,
                                _p(np.ascontiguousarray(y0, np.float64)), _p(y_end), C.addressof(st))
        return r, y_end, st.as_dict()

    def integrate_outputs(self, opts, nblocks, t0, y0, t_out):
        from fvmpor_b200 import Stats

        tv = np.ascontiguousarray(t_out, np.float64)
        Y = np.zeros((tv.size, self.N))
        YP = np.zeros((tv.size, self.N))
        st = Stats()
        r = lib().orc_integrate_outputs(self._c, C.addressof(opts), nblocks, t0,
                                        _p(np.ascontiguousarray(y0, np.float64)), tv.size, _p(tv), _p(Y),
                                        _p(YP), C.addressof(st))
        return r, Y, YP, st.as_dict()

    @staticmethod
    def threads():
        return lib().orc_threads()


def _declare_extra():
    L = lib()
    P, D, I = C.c_void_p, C.c_double, C.c_int
    L.orc_factor_given.argtypes = [P, P, I]
    L.orc_vg.argtypes = [D, D, D, I, P, P, P, P]
    return L


def vg(alpha, n, S_r, h):
    """Oracle van Genuchten relations (Sw, dSw/dh, krw) at heads h."""
    L = _declare_extra()
    h = np.ascontiguousarray(h, np.float64)
    Sw, dSw, krw = np.zeros_like(h), np.zeros_like(h), np.zeros_like(h)
    L.orc_vg(alpha, n, S_r, len(h), _p(h), _p(Sw), _p(dSw), _p(krw))
    return Sw, dSw, krw


def factor_given(orc: Oracle, values, nblocks):
    L = _declare_extra()
    return L.orc_factor_given(orc._c, _p(np.ascontiguousarray(values, np.float64)), nblocks)
