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
        L.orc_set_schur.argtypes = [P, I]
        L.orc_schur_interface_rows.argtypes = [P]
        L.orc_gmres.argtypes = [P, D, P, P, P, P, P, P, I, I, D, P, P]
        L.orc_integrate.argtypes = [P, P, I, D, D, P, P, P]
        L.orc_integrate_outputs.argtypes = [P, P, I, D, P, I, P, P, P, P]
        L.orc_interp_coefs.argtypes = [P, I, D, P, P]
        L.orc_threads.restype = I
        L.orc_step_trace.restype = C.c_long
        L.orc_step_trace.argtypes = [P, P, C.c_long]
        L.orc_timers.argtypes = [P, P, P, I]
        L.orc_replay.argtypes = [P, P, I, D, P, D, C.c_long, P, D, I, P, P]
        L.orc_replay_controller.argtypes = [P, P, I, D, P, D, C.c_long, P, D, I, P, P]
        L.orc_problem_error.restype = C.c_char_p
        L.orc_initial_head.argtypes = [P, D, P]
        L.fvm_problem_richards2d.argtypes = [I, I, D, D, D, C.c_uint64, D, D, P]
        L.fvm_problem_richards3d.argtypes = [I, I, I, D, D, D, D, C.c_uint64, D, D, D, D, D, P]
        L.fvm_problem_ensemble2d.argtypes = [I, I, I, C.c_uint64, P, P]
        L.fvm_problem_free.argtypes = [P]
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

    def set_schur(self, iters):
        """Schur interface coupling of the block ILU(0): < 0 off, >= 0 the
        interface iterations of every apply (next factorisation on)"""
        lib().orc_set_schur(self._c, int(iters))

    def schur_interface_rows(self):
        return lib().orc_schur_interface_rows(self._c)

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

    def initial_head(self, water_table=None):
        """hydrostatic initial head (the rules of fvm_initial_head)"""
        y = np.zeros(self.N)
        wt = self._problem.water_table if water_table is None else water_table
        lib().orc_initial_head(self._c, wt, _p(y))
        return y

    def trace(self):
        """accepted steps of the last adaptive integration (record array with
        the fields of fvm_step_record)"""
        from fvmpor_b200 import StepRecord

        n = lib().orc_step_trace(self._c, None, 0)
        buf = (StepRecord * max(1, n))()
        lib().orc_step_trace(self._c, buf, n)
        dt = np.dtype([(k, np.float64 if t is C.c_double else np.int32) for k, t in StepRecord._fields_])
        return np.frombuffer(bytes(buf), dtype=dt, count=n).copy() if n > 0 else np.zeros(0, dt)

    TIMER_NAMES = ("newton_residual", "jv", "fd_jacobian", "ilu_factor", "ilu_apply", "krylov_other", "total")
    COUNT_NAMES = ("newton_residuals", "jv", "setups", "applies", "krylov_iterations", "newton_iterations", "steps")

    def timers(self, reset=False):
        """time split (s) and work counters of the integrations and replays
        since creation or the last reset"""
        tm = np.zeros(7)
        cnt = np.zeros(7, np.int64)
        lib().orc_timers(self._c, tm.ctypes.data, cnt.ctypes.data, int(reset))
        return dict(zip(self.TIMER_NAMES, tm.tolist())), dict(zip(self.COUNT_NAMES, cnt.tolist()))

    def replay(self, opts, nblocks, t0, y0, h0, steps, newton_tol=1e-5, max_newton=10, controller=False):
        """replay the accepted steps (records with fields h and order) with
        each corrector solved to ||delta||_wrms <= newton_tol; independent
        Lagrange-form restatement of the BDF step (orc_replay), or, with
        controller=True, the product's controller template on the oracle's
        kernels (orc_replay_controller).  Returns (rc, y_end, stats)."""
        from fvmpor_b200 import Stats, StepRecord

        n = len(steps)
        buf = (StepRecord * n)()
        for i in range(n):
            buf[i].t = float(steps["t"][i])
            buf[i].h = float(steps["h"][i])
            buf[i].order = int(steps["order"][i])
        y_end = np.zeros(self.N)
        st = Stats()
        fn = lib().orc_replay_controller if controller else lib().orc_replay
        r = fn(self._c, C.addressof(opts), nblocks, t0, _p(np.ascontiguousarray(y0, np.float64)), h0, n, buf,
               newton_tol, max_newton, _p(y_end), C.addressof(st))
        if r < 0:
            raise RuntimeError(f"orc_replay failed ({r})")
        return r, y_end, st.as_dict()


class OracleProblem:
    """A benchmark problem generated by the oracle's own copy of the
    generator (no product library in the process).  Offers what Oracle and
    the CPU timing need: the problem struct, sizes, water table, horizon and
    the host arrays."""

    def __init__(self, kind, **kw):
        from fvmpor_b200 import ProblemStruct

        self._s = ProblemStruct()
        L = lib()
        if kind == "2d":
            r = L.fvm_problem_richards2d(kw.get("nx", 81), kw.get("ny", 41), kw.get("Lx", 10.0), kw.get("Ly", 5.0),
                                         kw.get("jitter", 0.2), kw.get("seed", 1), kw.get("ln_var", 0.0),
                                         kw.get("corr_len", 1.0), C.addressof(self._s))
        elif kind == "3d":
            r = L.fvm_problem_richards3d(kw.get("nx", 100), kw.get("ny", 100), kw.get("nz", 20),
                                         kw.get("Lx", 100.0), kw.get("Ly", 100.0), kw.get("Lz", 20.0),
                                         kw.get("jitter", 0.15), kw.get("seed", 1), kw.get("ln_var", 1.0),
                                         kw.get("cx", 10.0), kw.get("cy", 10.0), kw.get("cz", 2.0),
                                         kw.get("Kg", 1e-5), C.addressof(self._s))
        else:
            raise ValueError(kind)
        if r != 0:
            raise RuntimeError("oracle problem generation: " + L.orc_problem_error().decode())
        self.kind = kind

    def __del__(self):
        if getattr(self, "_s", None) is not None and _lib is not None:
            _lib.fvm_problem_free(C.addressof(self._s))
            self._s = None

    mesh = property(lambda self: self._s.mesh)
    phys = property(lambda self: self._s.phys)
    n_nodes = property(lambda self: self._s.mesh.n_nodes)
    n_elements = property(lambda self: self._s.mesh.n_elements)
    water_table = property(lambda self: self._s.water_table)
    t_end = property(lambda self: self._s.t_end)

    def arrays(self):
        m = self._s.mesh
        d = m.dim
        return {
            "coords": np.ctypeslib.as_array(m.coords, (m.n_nodes, 3)).copy(),
            "elem_nodes": np.ctypeslib.as_array(m.elem_nodes, (m.n_elements, d + 1)).copy(),
            "node_tag": np.ctypeslib.as_array(m.node_tag, (m.n_nodes,)).copy(),
        }


# the benchmark configurations, as fvmpor_b200.CONFIGS names them
PROBLEMS = {
    "richards2d": ("2d", dict(nx=81, ny=41, Lx=10.0, Ly=5.0, jitter=0.2, seed=1)),
    "richards3d": ("3d", dict(nx=100, ny=100, nz=20, Lx=100.0, Ly=100.0, Lz=20.0, jitter=0.15, seed=1,
                              ln_var=1.0, cx=10.0, cy=10.0, cz=2.0, Kg=1e-5)),
}


def make_problem(name, **override):
    kind, params = PROBLEMS[name]
    p = dict(params)
    p.update(override)
    return OracleProblem(kind, **p)


def opts(**kw):
    """integrator options with the library's defaults (fvm_opts_default),
    filled without loading the product library"""
    from fvmpor_b200 import Opts

    o = Opts()
    o.rtol, o.atol, o.max_order, o.krylov_dim, o.max_restarts = 1e-6, 1e-6, 5, 30, 5
    o.eps_lin, o.cj_refresh, o.psetup_age = 3e-5, 1.05, 1
    for k, v in kw.items():
        if not hasattr(o, k):
            raise TypeError(f"unknown integrator option {k!r}")
        setattr(o, k, v)
    return o



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
