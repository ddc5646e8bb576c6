"""fvmpor_b200 — B200-native Richards-equation hot path of FVMPor.

Python plumbing over the C ABI in ``include/fvmpor_b200.h`` (the product is
``libfvmpor_b200.so``: sm_100a kernels plus the C++ host controller).  The
classes mirror the reference's call surface for this path:

* :class:`Physics`  — ``residual_evaluation`` / ``preprocess_timestep`` of
  ``VarSatPhysics`` (examples/fvmporMinlin/fvmpor_ODE_impl.cpp:62-141);
* :class:`Preconditioner` — ``setup`` / ``apply``
  (examples/fvmporMinlin/preconditioner_dss.h:27-39);
* :class:`Integrator` — ``IDAIntegrator::advance(t)``
  (include/fvm/integrators/ida_integrator.h:325-340).

Device vectors are ``torch.float64`` CUDA tensors; the library reads and
writes them in place through their data pointers.  There is no CPU
fallback: if the shared library is missing every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfvmpor_b200.so")

_lib = None


class FvmError(RuntimeError):
    pass


def build(force: bool = False) -> str:
    """Compile libfvmpor_b200.so for sm_100a (nvcc, in-tree)."""
    import subprocess

    if force and os.path.exists(LIB_PATH):
        os.remove(LIB_PATH)
    subprocess.run(["make", "-C", _HERE, "-j8"], check=True, capture_output=True)
    return LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FvmError(f"{LIB_PATH} is missing: run fvmpor_b200.build() (no CPU fallback)")
        _lib = C.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


# --------------------------------------------------------------------- structs
class Mesh(C.Structure):
    _fields_ = [
        ("dim", C.c_int), ("n_nodes", C.c_int), ("n_elements", C.c_int), ("n_bfaces", C.c_int),
        ("coords", C.POINTER(C.c_double)), ("elem_nodes", C.POINTER(C.c_int)),
        ("elem_zone", C.POINTER(C.c_int)), ("elem_K", C.POINTER(C.c_double)),
        ("bface_nodes", C.POINTER(C.c_int)), ("bface_elem", C.POINTER(C.c_int)),
        ("bface_tag", C.POINTER(C.c_int)), ("node_tag", C.POINTER(C.c_int)),
    ]


class Zone(C.Structure):
    _fields_ = [("Kxx", C.c_double), ("Kyy", C.c_double), ("Kzz", C.c_double), ("phi", C.c_double),
                ("alphaVG", C.c_double), ("nVG", C.c_double), ("S_r", C.c_double)]


class BC(C.Structure):
    _fields_ = [("tag", C.c_int), ("type", C.c_int), ("value", C.c_double), ("b", C.c_double),
                ("eta", C.c_double)]


class PhysicsDesc(C.Structure):
    _fields_ = [("n_zones", C.c_int), ("zones", C.POINTER(Zone)), ("n_bcs", C.c_int),
                ("bcs", C.POINTER(BC)), ("rho0", C.c_double)]


class ProblemStruct(C.Structure):
    _fields_ = [
        ("mesh", Mesh), ("phys", PhysicsDesc), ("water_table", C.c_double), ("t_end", C.c_double),
        ("coords", C.c_void_p), ("elem_nodes", C.c_void_p), ("elem_zone", C.c_void_p),
        ("elem_K", C.c_void_p), ("bface_nodes", C.c_void_p), ("bface_elem", C.c_void_p),
        ("bface_tag", C.c_void_p), ("node_tag", C.c_void_p), ("zones", C.c_void_p),
        ("bcs", C.c_void_p), ("grid_dims", C.POINTER(C.c_int)),
    ]


class PmeshStruct(C.Structure):
    _fields_ = [("n_dom", C.c_int), ("dom_id", C.c_int), ("dim", C.c_int), ("n_nodes", C.c_int),
                ("n_elements", C.c_int), ("n_bfaces", C.c_int), ("coords", C.POINTER(C.c_double)),
                ("elem_nodes", C.POINTER(C.c_int)), ("elem_tag", C.POINTER(C.c_int)),
                ("bface_nodes", C.POINTER(C.c_int)), ("bface_elem", C.POINTER(C.c_int)),
                ("bface_tag", C.POINTER(C.c_int)), ("node_bc_ptr", C.POINTER(C.c_int)),
                ("node_bc", C.POINTER(C.c_int)), ("perm", C.POINTER(C.c_int)), ("bandwidth_file", C.c_int),
                ("bandwidth", C.c_int)]


class StepRecord(C.Structure):
    _fields_ = [("t", C.c_double), ("h", C.c_double), ("err", C.c_double), ("wall", C.c_double), ("order", C.c_int),
                ("attempts", C.c_int), ("nni", C.c_int), ("nli", C.c_int), ("npe", C.c_int), ("learned", C.c_int)]


class Opts(C.Structure):
    _fields_ = [("rtol", C.c_double), ("atol", C.c_double), ("max_order", C.c_int),
                ("krylov_dim", C.c_int), ("max_restarts", C.c_int), ("precision", C.c_int),
                ("use_predictor", C.c_int), ("h0", C.c_double), ("hmax", C.c_double),
                ("max_steps", C.c_long), ("eps_lin", C.c_double), ("cj_refresh", C.c_double),
                ("psetup_age", C.c_int), ("krylov_operator", C.c_int), ("graph", C.c_int)]


class Stats(C.Structure):
    _fields_ = [("nst", C.c_long), ("nre", C.c_long), ("nni", C.c_long), ("nli", C.c_long),
                ("npe", C.c_long), ("nps", C.c_long), ("ncfn", C.c_long), ("ncfl", C.c_long),
                ("netf", C.c_long), ("npred", C.c_long), ("last_order", C.c_int),
                ("last_h", C.c_double), ("t", C.c_double), ("nsync", C.c_long)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_P = C.c_void_p
_D = C.c_double
_I = C.c_int


class TuneResult(C.Structure):
    _fields_ = [("n", C.c_int), ("best", C.c_int), ("variant", C.c_int * 16), ("chunk", C.c_int * 16),
                ("us", C.c_double * 16)]


def _declare(L):
    L.fvm_create.restype = _P
    L.fvm_create.argtypes = [C.POINTER(Mesh), C.POINTER(PhysicsDesc), _I]
    L.fvm_destroy.argtypes = [_P]
    L.fvm_last_error.restype = C.c_char_p
    L.fvm_n_nodes.argtypes = [_P]
    L.fvm_initial_head.argtypes = [_P, _D, _P]
    L.fvm_residual.argtypes = [_P, _D, _P, _P, _P]
    L.fvm_begin_step.argtypes = [_P, _D, _P, _P]
    L.fvm_jv.argtypes = [_P, _D, _D, _P, _P, _P, _P, _D, _P]
    L.fvm_psetup.argtypes = [_P, _D, _D, _D, _P, _P, _P, _P, _I]
    L.fvm_psolve.argtypes = [_P, _P, _P]
    L.fvm_gmres.argtypes = [_P, _D, _D, _P, _P, _P, _P, _P, _P, _I, _I, _I, _D,
                            C.POINTER(_I), C.POINTER(_D)]
    L.fvm_wrms.restype = _D
    L.fvm_wrms.argtypes = [_P, _P, _P]
    L.fvm_dot.restype = _D
    L.fvm_dot.argtypes = [_P, _P, _P]
    L.fvm_opts_default.argtypes = [C.POINTER(Opts)]
    L.fvm_integrate.argtypes = [_P, C.POINTER(Opts), _D, _D, _P, _P, C.POINTER(Stats)]
    L.fvm_integrate_host.argtypes = [_P, C.POINTER(Opts), _D, _D, _P, _P, C.POINTER(Stats)]
    L.fvm_integrate_outputs.argtypes = [_P, C.POINTER(Opts), _D, _P, C.c_int, _P, _P, _P, C.POINTER(Stats)]
    L.fvm_problem_richards2d.argtypes = [_I, _I, _D, _D, _D, C.c_uint64, _D, _D, C.POINTER(ProblemStruct)]
    L.fvm_problem_richards3d.argtypes = [_I, _I, _I, _D, _D, _D, _D, C.c_uint64, _D, _D, _D, _D, _D,
                                         C.POINTER(ProblemStruct)]
    L.fvm_problem_free.argtypes = [C.POINTER(ProblemStruct)]
    L.fvm_problem_ensemble2d.argtypes = [_I, _I, _I, C.c_uint64, C.POINTER(ProblemStruct), _P]
    L.fvm_set_members.argtypes = [_P, _I, _P]
    L.fvm_integrate_replay.argtypes = [_P, C.POINTER(Opts), _D, _P, _D, C.c_long, C.POINTER(StepRecord), _D,
                                       C.c_int, _P, C.POINTER(Stats)]
    L.fvm_set_krylov_variant.argtypes = [_P, _I]
    L.fvm_graph_counters.argtypes = [_P, C.POINTER(C.c_long), C.POINTER(C.c_long)]
    L.fvm_integrate_batch.argtypes = [_P, _I, C.POINTER(Opts), _D, _D, _P, _P, _P, _P, _I]
    L.fvm_step_trace.restype = C.c_long
    L.fvm_step_trace.argtypes = [_P, C.POINTER(StepRecord), C.c_long]
    L.fvm_pmesh_read.argtypes = [C.c_char_p, _I, C.POINTER(PmeshStruct)]
    L.fvm_pmesh_write.argtypes = [C.c_char_p, C.POINTER(PmeshStruct)]
    L.fvm_pmesh_free.argtypes = [C.POINTER(PmeshStruct)]
    L.fvm_problem_from_pmesh.argtypes = [C.POINTER(PmeshStruct), _I, C.POINTER(Zone), _I, C.POINTER(BC), _D,
                                         C.POINTER(ProblemStruct)]
    L.fvm_write_vtu.argtypes = [C.c_char_p, _I, _I, _I, C.POINTER(Mesh), _P]
    L.fvm_precond_info.argtypes = [_P, C.POINTER(_I), C.POINTER(_I), C.POINTER(_I), C.POINTER(_I)]
    L.fvm_precond_jacobian.argtypes = [_P, _P, _P, _P]
    L.fvm_profile.argtypes = [_P, _I]
    L.fvm_profile_read.argtypes = [_P, _P, _P]
    L.fvm_counters.argtypes = [_P, C.POINTER(C.c_long), C.POINTER(C.c_long)]
    L.fvm_autotune.argtypes = [_P, C.POINTER(TuneResult)]
    L.fvm_set_element_pass.argtypes = [_P, _I, _I]
    L.fvm_element_pass.argtypes = [_P, C.POINTER(_I), C.POINTER(_I)]
    L.fvm_set_precond_blocks.argtypes = [_P, _I]
    L.fvm_set_precond_schur.argtypes = [_P, _I]
    L.fvm_precond_schur_info.argtypes = [_P, C.POINTER(_I), C.POINTER(_I), C.POINTER(_I)]
    L.fvm_mlp_nparams.restype = _I
    L.fvm_mlp_set_params.argtypes = [_P, _P]
    L.fvm_mlp_get_params.argtypes = [_P, _P]
    L.fvm_mlp_forward.argtypes = [_P, _P, _I, _P]
    L.fvm_mlp_grad.argtypes = [_P, _P, _P, _I, _P, C.POINTER(C.c_float)]
    L.fvm_mlp_train.argtypes = [_P, _P, _P, _I, _I, _I, C.c_float, _P]
    L.fvm_integrate_record.argtypes = [_P, C.POINTER(Opts), _D, _D, _P, _P, C.POINTER(Stats), _P, _P, C.c_long,
                                       _I, C.POINTER(C.c_long)]


PROFILE_CATEGORIES = ("node", "element", "gather", "ilu_apply", "gram_schmidt", "ilu_factor", "fd_jacobian",
                      "mlp", "learned_attempt")


def _err(prefix, code=None):
    msg = lib().fvm_last_error().decode()
    return FvmError(f"{prefix}: {msg}" + ("" if code is None else f" (status {code})"))


def _check(code, what):
    if code < 0:
        raise _err(what, code)
    return code


# --------------------------------------------------------------------- problems
class Problem:
    """A synthetic Richards problem generated by the library (host memory)."""

    def __init__(self, kind: str, **kw):
        self._s = ProblemStruct()
        L = lib()
        if kind == "2d":
            r = L.fvm_problem_richards2d(kw.get("nx", 81), kw.get("ny", 41), kw.get("Lx", 10.0),
                                         kw.get("Ly", 5.0), kw.get("jitter", 0.2), kw.get("seed", 1),
                                         kw.get("ln_var", 0.0), kw.get("corr_len", 1.0), C.byref(self._s))
        elif kind == "3d":
            r = L.fvm_problem_richards3d(kw.get("nx", 100), kw.get("ny", 100), kw.get("nz", 20),
                                         kw.get("Lx", 100.0), kw.get("Ly", 100.0), kw.get("Lz", 20.0),
                                         kw.get("jitter", 0.15), kw.get("seed", 1), kw.get("ln_var", 1.0),
                                         kw.get("cx", 10.0), kw.get("cy", 10.0), kw.get("cz", 2.0),
                                         kw.get("Kg", 1e-5), C.byref(self._s))
        elif kind == "ensemble2d":
            nmem = kw.get("n_members", 256)
            mp = (C.c_int * (nmem + 1))()
            r = L.fvm_problem_ensemble2d(nmem, kw.get("nmin", 2000), kw.get("nmax", 40000), kw.get("seed", 1),
                                         C.byref(self._s), mp)
            self.member_ptr = np.array(mp[:], dtype=np.int32)
        else:
            raise ValueError(kind)
        if r != 0:
            raise _err("problem generation", r)
        self.kind = kind
        if kind != "ensemble2d":
            self.member_ptr = None

    def __del__(self):
        try:
            if getattr(self, "_owned", True) and getattr(self, "_s", None) is not None and _lib is not None:
                _lib.fvm_problem_free(C.byref(self._s))
        except Exception:
            pass

    @classmethod
    def from_arrays(cls, dim, coords, elem_nodes, elem_zone, bface_nodes, bface_elem, bface_tag, node_tag,
                    zones, bcs, elem_K=None, water_table=0.0, t_end=86400.0, rho0=1000.0):
        """a problem from host arrays (kept alive by the object)"""
        self = cls.__new__(cls)
        self._owned = False
        self.kind = "arrays"
        self.member_ptr = None
        keep = {
            "coords": np.ascontiguousarray(coords, np.float64).reshape(-1, 3),
            "elem_nodes": np.ascontiguousarray(elem_nodes, np.int32),
            "elem_zone": np.ascontiguousarray(elem_zone, np.int32),
            "bface_nodes": np.ascontiguousarray(bface_nodes, np.int32),
            "bface_elem": np.ascontiguousarray(bface_elem, np.int32),
            "bface_tag": np.ascontiguousarray(bface_tag, np.int32),
            "node_tag": np.ascontiguousarray(node_tag, np.int32),
        }
        if elem_K is not None:
            keep["elem_K"] = np.ascontiguousarray(elem_K, np.float64)
        self._zones = (Zone * len(zones))(*zones)
        self._bcs = (BC * len(bcs))(*bcs)
        self._keep = keep
        s = ProblemStruct()
        m = s.mesh
        m.dim = dim
        m.n_nodes = keep["coords"].shape[0]
        m.n_elements = keep["elem_zone"].shape[0]
        m.n_bfaces = keep["bface_tag"].shape[0]

        def ptr(a, t):
            return a.ctypes.data_as(C.POINTER(t))

        m.coords = ptr(keep["coords"], C.c_double)
        m.elem_nodes = ptr(keep["elem_nodes"], C.c_int)
        m.elem_zone = ptr(keep["elem_zone"], C.c_int)
        m.elem_K = ptr(keep["elem_K"], C.c_double) if "elem_K" in keep else None
        m.bface_nodes = ptr(keep["bface_nodes"], C.c_int)
        m.bface_elem = ptr(keep["bface_elem"], C.c_int)
        m.bface_tag = ptr(keep["bface_tag"], C.c_int)
        m.node_tag = ptr(keep["node_tag"], C.c_int)
        s.phys.n_zones = len(zones)
        s.phys.zones = C.cast(self._zones, C.POINTER(Zone))
        s.phys.n_bcs = len(bcs)
        s.phys.bcs = C.cast(self._bcs, C.POINTER(BC))
        s.phys.rho0 = rho0
        s.water_table = water_table
        s.t_end = t_end
        self._s = s
        return self

    @classmethod
    def from_pmesh(cls, mesh, zones, bcs, rho0=1000.0, t_end=0.0, rcm=True):
        """a problem on a .pmesh mesh (a path or a Pmesh): zones indexed by
        the element's physical tag - 100, Dirichlet node tags from the
        boundary conditions (fvm_problem_from_pmesh)"""
        pm = mesh if isinstance(mesh, Pmesh) else read_pmesh(mesh, rcm=rcm)
        self = cls.__new__(cls)
        self._s = ProblemStruct()
        zs = (Zone * len(zones))(*zones)
        bs = (BC * max(1, len(bcs)))(*bcs)
        r = lib().fvm_problem_from_pmesh(C.byref(pm._s), len(zones), zs, len(bcs), bs, rho0, C.byref(self._s))
        if r != 0:
            self._s = None
            raise _err("fvm_problem_from_pmesh", r)
        self._s.t_end = t_end
        self.kind = "pmesh"
        self.member_ptr = None
        self.pmesh = pm
        return self

    def write_vtu(self, stem, step, head, rank=0, n_ranks=1):
        """VTK XML output of a head field (<stem>_dom<rank>_<step>.vtu and,
        on rank 0, <stem>_head_<step>.pvtu)"""
        h = np.ascontiguousarray(np.asarray(head, dtype=np.float64))
        if h.shape != (self.n_nodes,):
            raise ValueError(f"head must have {self.n_nodes} values")
        _check(lib().fvm_write_vtu(str(stem).encode(), step, rank, n_ranks, C.byref(self._s.mesh),
                                   h.ctypes.data), "fvm_write_vtu")

    def member(self, m):
        """member m of an ensemble problem as a standalone problem"""
        a, b = int(self.member_ptr[m]), int(self.member_ptr[m + 1])
        if getattr(self, "_member_index", None) is None:
            # once per problem: the arrays and, per member, its elements and
            # boundary faces (members never share either)
            arr = self.arrays()
            nm = len(self.member_ptr) - 1
            eown = np.searchsorted(self.member_ptr, arr["elem_nodes"][:, 0], side="right") - 1
            bown = np.searchsorted(self.member_ptr, arr["bface_nodes"][:, 0], side="right") - 1
            eord = np.argsort(eown, kind="stable")
            bord = np.argsort(bown, kind="stable")
            eptr = np.searchsorted(eown[eord], np.arange(nm + 1))
            bptr = np.searchsorted(bown[bord], np.arange(nm + 1))
            self._member_index = (arr, eord, eptr, bord, bptr)
        arr, eord, eptr, bord, bptr = self._member_index
        d = self.mesh.dim
        en = arr["elem_nodes"]
        eidx = eord[eptr[m]:eptr[m + 1]]
        sel = eidx
        bf = arr["bface_nodes"]
        bsel = bord[bptr[m]:bptr[m + 1]]
        be = np.ctypeslib.as_array(self.mesh.bface_elem, (self.mesh.n_bfaces,))[bsel]
        emap = np.full(self.n_elements, -1, np.int64)
        emap[eidx] = np.arange(len(eidx))
        zones = [self.phys.zones[i] for i in range(self.phys.n_zones)]
        bcs = [self.phys.bcs[i] for i in range(self.phys.n_bcs)]
        return Problem.from_arrays(d, arr["coords"][a:b], en[sel] - a, arr["elem_zone"][sel], bf[bsel] - a,
                                   emap[be], arr["bface_tag"][bsel], arr["node_tag"][a:b], zones, bcs,
                                   elem_K=arr["elem_K"][sel] if "elem_K" in arr else None,
                                   water_table=self.water_table, t_end=self.t_end, rho0=self.phys.rho0)

    @property
    def mesh(self) -> Mesh:
        return self._s.mesh

    @property
    def phys(self) -> PhysicsDesc:
        return self._s.phys

    @property
    def n_nodes(self):
        return self._s.mesh.n_nodes

    @property
    def n_elements(self):
        return self._s.mesh.n_elements

    @property
    def water_table(self):
        return self._s.water_table

    @property
    def t_end(self):
        return self._s.t_end

    def arrays(self):
        m = self._s.mesh
        d = m.dim
        out = {
            "coords": np.ctypeslib.as_array(m.coords, (m.n_nodes, 3)).copy(),
            "elem_nodes": np.ctypeslib.as_array(m.elem_nodes, (m.n_elements, d + 1)).copy(),
            "elem_zone": np.ctypeslib.as_array(m.elem_zone, (m.n_elements,)).copy(),
            "bface_nodes": np.ctypeslib.as_array(m.bface_nodes, (m.n_bfaces, d)).copy(),
            "bface_tag": np.ctypeslib.as_array(m.bface_tag, (m.n_bfaces,)).copy(),
            "node_tag": np.ctypeslib.as_array(m.node_tag, (m.n_nodes,)).copy(),
        }
        if m.elem_K:
            out["elem_K"] = np.ctypeslib.as_array(m.elem_K, (m.n_elements,)).copy()
        return out


def _ptr(t):
    """device pointer of a contiguous float64 CUDA tensor"""
    import torch

    if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.float64 or not t.is_contiguous():
        raise TypeError("expected a contiguous torch.float64 CUDA tensor")
    return C.c_void_p(t.data_ptr())


FLAG_RECOMPUTE_GEOMETRY = 1   # element pass rebuilds the face geometry (3D default)
FLAG_AUTOTUNE = 2             # pick the element-pass variant and chunk size at creation
FLAG_STORED_GEOMETRY = 4      # element pass streams stored face coefficients


class Physics:
    """Device-resident Richards physics for one mesh (fvm_ctx)."""

    def __init__(self, problem: Problem, flags: int = 0):
        self.problem = problem
        self._c = lib().fvm_create(C.byref(problem._s.mesh), C.byref(problem._s.phys), flags)
        if self._c and getattr(problem, "member_ptr", None) is not None:
            mp = np.ascontiguousarray(problem.member_ptr, np.int32)
            _check(lib().fvm_set_members(self._c, len(mp) - 1, mp.ctypes.data), "fvm_set_members")
        if not self._c:
            raise _err("fvm_create")
        self.N = problem.n_nodes

    def close(self):
        if getattr(self, "_c", None):
            lib().fvm_destroy(self._c)
            self._c = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # reference: set_initial_conditions (vs.h:8-32)
    def initial_head(self, y, water_table=None):
        wt = self.problem.water_table if water_table is None else water_table
        _check(lib().fvm_initial_head(self._c, wt, _ptr(y)), "fvm_initial_head")

    # reference: preprocess_evaluation + residual_evaluation
    def residual(self, t, y, yp, res):
        _check(lib().fvm_residual(self._c, t, _ptr(y), _ptr(yp), _ptr(res)), "fvm_residual")

    # reference: preprocess_timestep
    def begin_step(self, t, y, yp):
        _check(lib().fvm_begin_step(self._c, t, _ptr(y), _ptr(yp)), "fvm_begin_step")

    def jv(self, t, cj, y, yp, F0, v, sigma, out):
        _check(lib().fvm_jv(self._c, t, cj, _ptr(y), _ptr(yp), _ptr(F0), _ptr(v), sigma, _ptr(out)), "fvm_jv")

    def wrms(self, x, ewt=None):
        return lib().fvm_wrms(self._c, _ptr(x), _ptr(ewt) if ewt is not None else None)

    def dot(self, x, y):
        return lib().fvm_dot(self._c, _ptr(x), _ptr(y))

    def profile(self, enable: bool):
        _check(lib().fvm_profile(self._c, 1 if enable else 0), "fvm_profile")

    def autotune(self):
        """time every element-pass candidate on this mesh, keep the fastest;
        returns [(variant, chunk, us)] and the index kept"""
        r = TuneResult()
        _check(lib().fvm_autotune(self._c, C.byref(r)), "fvm_autotune")
        return [(r.variant[i], r.chunk[i], r.us[i]) for i in range(r.n)], r.best

    def set_element_pass(self, variant, chunk):
        _check(lib().fvm_set_element_pass(self._c, variant, chunk), "fvm_set_element_pass")

    def element_pass(self):
        v, ch = _I(), _I()
        _check(lib().fvm_element_pass(self._c, C.byref(v), C.byref(ch)), "fvm_element_pass")
        return v.value, ch.value

    def counters(self):
        a, b = C.c_long(), C.c_long()
        _check(lib().fvm_counters(self._c, C.byref(a), C.byref(b)), "fvm_counters")
        return {"launches": a.value, "residuals": b.value}

    def profile_read(self):
        ms = np.zeros(len(PROFILE_CATEGORIES))
        cnt = np.zeros(len(PROFILE_CATEGORIES), np.int64)
        _check(lib().fvm_profile_read(self._c, ms.ctypes.data, cnt.ctypes.data), "fvm_profile_read")
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(PROFILE_CATEGORIES)}


class Preconditioner:
    """Coloured-FD Jacobian + block-ILU(0) (Preconditioner::setup/apply)."""

    def __init__(self, physics: Physics):
        self.ph = physics

    def setup(self, t, cj, h, y, yp, F0, ewt, precision=0):
        return _check(lib().fvm_psetup(self.ph._c, t, cj, h, _ptr(y), _ptr(yp), _ptr(F0), _ptr(ewt), precision),
                      "fvm_psetup")

    def apply(self, r, z):
        _check(lib().fvm_psolve(self.ph._c, _ptr(r), _ptr(z)), "fvm_psolve")

    def set_blocks_per_sm(self, per_sm):
        """block-ILU blocks per SM on large meshes (drops the current factor)"""
        _check(lib().fvm_set_precond_blocks(self.ph._c, per_sm), "fvm_set_precond_blocks")

    def set_schur(self, iters):
        """Schur interface coupling of the block ILU(0): iters < 0 off, else
        the interface sweeps of every apply (drops the current factor)"""
        _check(lib().fvm_set_precond_schur(self.ph._c, int(iters)), "fvm_set_precond_schur")

    def schur_info(self):
        a, b, c = _I(), _I(), _I()
        _check(lib().fvm_precond_schur_info(self.ph._c, C.byref(a), C.byref(b), C.byref(c)),
               "fvm_precond_schur_info")
        return {"iters": a.value, "interface_rows": b.value, "fp64": bool(c.value & 1), "fp32": bool(c.value & 2)}

    def info(self):
        a, b, c, d = _I(), _I(), _I(), _I()
        _check(lib().fvm_precond_info(self.ph._c, C.byref(a), C.byref(b), C.byref(c), C.byref(d)),
               "fvm_precond_info")
        return {"nnz": a.value, "ncolours": b.value, "nblocks": c.value, "max_levels": d.value}

    def jacobian(self):
        inf = self.info()
        rp = np.zeros(self.ph.N + 1, np.int32)
        col = np.zeros(inf["nnz"], np.int32)
        val = np.zeros(inf["nnz"], np.float64)
        _check(lib().fvm_precond_jacobian(self.ph._c, rp.ctypes.data, col.ctypes.data, val.ctypes.data),
               "fvm_precond_jacobian")
        return rp, col, val

    def gmres(self, t, cj, y, yp, F0, ewt, b, x, m=30, max_restarts=5, precision=0, tol=0.0165):
        its, rn = _I(), _D()
        r = lib().fvm_gmres(self.ph._c, t, cj, _ptr(y), _ptr(yp), _ptr(F0), _ptr(ewt), _ptr(b), _ptr(x), m,
                            max_restarts, precision, tol, C.byref(its), C.byref(rn))
        _check(r, "fvm_gmres")
        return r, its.value, rn.value


def integrate_batch(physics_list, t0, t_end, y0_list, y_end_list, n_threads=8, **opts):
    """independent problems, one Physics context each, integrated
    concurrently with their own step sequences (fvm_integrate_batch);
    returns (rc, per-member status codes, per-member stats dicts)"""
    n = len(physics_list)
    o = default_opts(**opts)
    ctxs = (C.c_void_p * n)(*[ph._c for ph in physics_list])
    y0s = (C.c_void_p * n)(*[_ptr(v) for v in y0_list])
    yes = (C.c_void_p * n)(*[_ptr(v) for v in y_end_list])
    st = (Stats * n)()
    status = (C.c_int * n)()
    rc = lib().fvm_integrate_batch(ctxs, n, C.byref(o), t0, t_end, y0s, yes, st, status, n_threads)
    if rc < 0:
        raise _err("fvm_integrate_batch", rc)
    return rc, [int(x) for x in status], [s_.as_dict() for s_ in st]


def default_opts(**kw) -> Opts:
    o = Opts()
    lib().fvm_opts_default(C.byref(o))
    names = {f for f, _ in Opts._fields_}
    for k, v in kw.items():
        if k not in names:
            raise TypeError(f"unknown integrator option {k!r}")
        setattr(o, k, v)
    return o


class Integrator:
    """Variable-order BDF + Newton-GMRES on the device (IDAIntegrator)."""

    def __init__(self, physics: Physics, **opts):
        self.ph = physics
        self.opts = default_opts(**opts)

    def integrate(self, t0, t_end, y0, y_end):
        st = Stats()
        r = lib().fvm_integrate(self.ph._c, C.byref(self.opts), t0, t_end, _ptr(y0), _ptr(y_end), C.byref(st))
        if r < 0:
            raise _err("fvm_integrate", r)
        return r, st.as_dict()

    def trace(self):
        """the accepted steps of the last integration on this context, as a
        numpy record array (t, h, err, wall, order, attempts, nni, nli, npe,
        learned)"""
        L = lib()
        n = L.fvm_step_trace(self.ph._c, None, 0)
        buf = (StepRecord * max(1, n))()
        L.fvm_step_trace(self.ph._c, buf, n)
        dt = np.dtype([(k, np.float64 if t is C.c_double else np.int32) for k, t in StepRecord._fields_])
        return np.frombuffer(bytes(buf), dtype=dt, count=n).copy() if n > 0 else np.zeros(0, dt)

    def replay(self, t0, y0, h0, steps, y_end, newton_tol=1e-5, max_newton=10):
        """replay the accepted steps ``steps`` (a trace record array, or any
        array with fields h and order) from (t0, y0) with every corrector
        solved to ||delta||_wrms <= newton_tol (fvm_integrate_replay);
        returns (rc, stats), rc 1 when some corrector stopped at max_newton"""
        n = len(steps)
        buf = (StepRecord * n)()
        for i in range(n):
            buf[i].h = float(steps["h"][i])
            buf[i].order = int(steps["order"][i])
        st = Stats()
        r = lib().fvm_integrate_replay(self.ph._c, C.byref(self.opts), t0, _ptr(y0), h0, n, buf, newton_tol,
                                       max_newton, _ptr(y_end), C.byref(st))
        if r < 0:
            raise _err("fvm_integrate_replay", r)
        return r, st.as_dict()

    def integrate_outputs(self, t0, t_out, y0, y_out, yp_out=None):
        """integrate from (t0, y0) through the ascending output times t_out
        without shortening steps to meet them (IDAIntegrator::advance); the
        heads at t_out[i] go to y_out[i] and their time derivatives to
        yp_out[i] (float64 CUDA tensors [len(t_out), N]; yp_out optional),
        interpolated from the step that reached each time"""
        tv = np.ascontiguousarray(t_out, np.float64)
        n = tv.size
        if y_out.shape != (n, self.ph.problem.n_nodes) or (yp_out is not None and yp_out.shape != y_out.shape):
            raise ValueError("y_out / yp_out must have shape (len(t_out), n_nodes)")
        st = Stats()
        r = lib().fvm_integrate_outputs(self.ph._c, C.byref(self.opts), t0, _ptr(y0), n, tv.ctypes.data,
                                        _ptr(y_out), _ptr(yp_out) if yp_out is not None else None,
                                        C.byref(st))
        if r < 0:
            raise _err("fvm_integrate_outputs", r)
        return r, st.as_dict()

    def integrate_host(self, t0, t_end, y0: np.ndarray, y_end: np.ndarray):
        st = Stats()
        y0 = np.ascontiguousarray(y0, np.float64)
        assert y_end.dtype == np.float64 and y_end.flags.c_contiguous
        r = lib().fvm_integrate_host(self.ph._c, C.byref(self.opts), t0, t_end, y0.ctypes.data,
                                     y_end.ctypes.data, C.byref(st))
        if r < 0:
            raise _err("fvm_integrate_host", r)
        return r, st.as_dict()

    def integrate_record(self, t0, t_end, y0, y_end, X, Y, stride=64):
        """integrate while recording (features, target) pairs of every
        stride-th node per accepted step into the float32 CUDA tensors X
        [cap, 8] and Y [cap]; returns (rc, stats, count)"""
        import torch

        assert X.is_cuda and X.dtype == torch.float32 and Y.is_cuda and Y.dtype == torch.float32
        st = Stats()
        cnt = C.c_long()
        r = lib().fvm_integrate_record(self.ph._c, C.byref(self.opts), t0, t_end, _ptr(y0), _ptr(y_end),
                                       C.byref(st), C.c_void_p(X.data_ptr()), C.c_void_p(Y.data_ptr()),
                                       Y.numel(), stride, C.byref(cnt))
        if r < 0:
            raise _err("fvm_integrate_record", r)
        return r, st.as_dict(), cnt.value


class Predictor:
    """Per-node MLP that proposes the Newton initial iterate (BF16 weights,
    FP32 accumulation on the tcgen05 tensor cores; fvm_mlp_*)."""

    # parameter vector layout (fvm_mlp_set_params): W1[64x8] b1[64]
    # W2[64x64] b2[64] W3[64x64] b3[64] w4[64] b4 | feature mean[8], std[8]
    IN, H = 8, 64

    def __init__(self, physics: Physics):
        self.ph = physics
        self.n = lib().fvm_mlp_nparams()

    def init(self, X, seed=0):
        """the untrained network: normal(0, 1/fan_in) weights, zero biases,
        and feature scalers from the mean / std of the columns of X (a CUDA
        float32 tensor [n, 8] of recorded features)"""
        IN, H = self.IN, self.H
        mu = X.mean(0).double().cpu().numpy()
        sd = X.std(0).double().cpu().numpy() + 1e-6
        rng = np.random.default_rng(seed)
        parts = [rng.normal(0, 1 / np.sqrt(IN), H * IN), np.zeros(H),
                 rng.normal(0, 1 / np.sqrt(H), H * H), np.zeros(H),
                 rng.normal(0, 1 / np.sqrt(H), H * H), np.zeros(H),
                 rng.normal(0, 1 / np.sqrt(H), H), np.zeros(1), mu, sd]
        P = np.concatenate(parts).astype(np.float32)
        assert P.size == self.n
        self.set_params(P)

    def set_params(self, P):
        P = np.ascontiguousarray(P, np.float32)
        assert P.size == self.n
        _check(lib().fvm_mlp_set_params(self.ph._c, P.ctypes.data), "fvm_mlp_set_params")

    def get_params(self):
        P = np.zeros(self.n, np.float32)
        _check(lib().fvm_mlp_get_params(self.ph._c, P.ctypes.data), "fvm_mlp_get_params")
        return P

    def forward(self, X, out):
        r = lib().fvm_mlp_forward(self.ph._c, C.c_void_p(X.data_ptr()), X.shape[0], C.c_void_p(out.data_ptr()))
        _check(r, "fvm_mlp_forward")
        return r

    def grad(self, X, Y):
        """full-batch gradient of mean((mlp(X) - Y)^2) and the loss"""
        g = np.zeros(self.n - 16, np.float32)   # trainable part (feature scalers excluded)
        loss = C.c_float()
        r = lib().fvm_mlp_grad(self.ph._c, C.c_void_p(X.data_ptr()), C.c_void_p(Y.data_ptr()), Y.numel(),
                               g.ctypes.data, C.byref(loss))
        _check(r, "fvm_mlp_grad")
        return g, loss.value, r

    def train(self, X, Y, epochs=5, batch=0, lr=1e-3):
        hist = np.zeros(epochs, np.float32)
        r = lib().fvm_mlp_train(self.ph._c, C.c_void_p(X.data_ptr()), C.c_void_p(Y.data_ptr()), Y.numel(), epochs,
                                batch, lr, hist.ctypes.data)
        _check(r, "fvm_mlp_train")
        return r, hist


@dataclass
class Config:
    """Benchmark problems (seeded synthetic inputs of the named shapes)."""

    name: str
    kind: str
    params: dict


class Pmesh:
    """A .pmesh mesh read by the library (fvm_pmesh_read); the arrays are
    numpy views of library-owned memory, released with the object."""

    def __init__(self, s: PmeshStruct):
        self._s = s
        d = s.dim
        n, ne, nb = s.n_nodes, s.n_elements, s.n_bfaces

        def view(p, shape):
            return np.ctypeslib.as_array(p, shape) if int(np.prod(shape)) > 0 else np.zeros(shape, np.int32)

        self.dim, self.n_nodes, self.n_elements, self.n_bfaces = d, n, ne, nb
        self.coords = view(s.coords, (n, 3))
        self.elem_nodes = view(s.elem_nodes, (ne, d + 1))
        self.elem_tag = view(s.elem_tag, (ne,))
        self.bface_nodes = view(s.bface_nodes, (nb, d))
        self.bface_elem = view(s.bface_elem, (nb,))
        self.bface_tag = view(s.bface_tag, (nb,))
        self.node_bc_ptr = view(s.node_bc_ptr, (n + 1,))
        self.node_bc = view(s.node_bc, (int(self.node_bc_ptr[-1]),))
        self.perm = view(s.perm, (n,))
        self.bandwidth_file, self.bandwidth = s.bandwidth_file, s.bandwidth

    @classmethod
    def from_problem(cls, problem: "Problem"):
        """the mesh of a problem as a Pmesh (physical tag = zone, node
        boundary tags = the Dirichlet node tags), e.g. to write it as a
        .pmesh file; the arrays belong to the object"""
        a = problem.arrays()
        m = problem.mesh
        nt = np.ascontiguousarray(a["node_tag"], np.int32)
        keep = {
            "coords": np.ascontiguousarray(a["coords"], np.float64),
            "elem_nodes": np.ascontiguousarray(a["elem_nodes"], np.int32),
            "elem_tag": np.ascontiguousarray(a["elem_zone"], np.int32),
            "bface_nodes": np.ascontiguousarray(a["bface_nodes"], np.int32),
            "bface_elem": np.ascontiguousarray(np.ctypeslib.as_array(m.bface_elem, (m.n_bfaces,)), np.int32),
            "bface_tag": np.ascontiguousarray(a["bface_tag"], np.int32),
            "node_bc_ptr": np.concatenate([[0], np.cumsum(nt != 0)]).astype(np.int32),
            "node_bc": np.ascontiguousarray(nt[nt != 0], np.int32),
            "perm": np.arange(m.n_nodes, dtype=np.int32),
        }
        s = PmeshStruct()
        s.n_dom, s.dom_id, s.dim = 1, 0, m.dim
        s.n_nodes, s.n_elements, s.n_bfaces = m.n_nodes, m.n_elements, m.n_bfaces
        for k, v in keep.items():
            setattr(s, k, v.ctypes.data_as(C.POINTER(C.c_double if v.dtype == np.float64 else C.c_int)))
        self = cls(s)
        self._owned_arrays = keep
        return self

    def write(self, path):
        _check(lib().fvm_pmesh_write(str(path).encode(), C.byref(self._s)), "fvm_pmesh_write")

    def __del__(self):
        try:
            if getattr(self, "_owned_arrays", None) is not None:
                return
            if _lib is not None and getattr(self, "_s", None) is not None:
                _lib.fvm_pmesh_free(C.byref(self._s))
                self._s = None
        except Exception:
            pass


def read_pmesh(path, rcm=True) -> Pmesh:
    """reads a one-domain .pmesh of triangles or tetrahedra; rcm renumbers
    the nodes by reverse Cuthill-McKee as the reference's Mesh does"""
    s = PmeshStruct()
    r = lib().fvm_pmesh_read(str(path).encode(), FVM_PMESH_RCM if rcm else 0, C.byref(s))
    if r != 0:
        raise _err(f"fvm_pmesh_read({path})", r)
    return Pmesh(s)


FVM_PMESH_RCM = 1


def cassion_physics():
    """zones and boundary conditions of the reference's caisson
    infiltration problem (examples/fvmporMinlin/cassion.h:36-116; the EEM
    example uses the same file): four van Genuchten zones with K =
    rho0 g / mu * k, no-flow tag 1, inflow of 2.3148e-7 m/s on tag 2
    (prescribed flux, positive outwards), uniform initial head -7.34 m"""
    factor = 1000.0 * 9.80665 / 1e-3
    rows = [(9.33e-12, 0.368, 3.34, 1.982, 0.2771), (5.55e-12, 0.3510, 3.63, 1.632, 0.2806),
            (4.898e-12, 0.3250, 3.45, 1.573, 0.2643), (4.898e-11, 0.3250, 3.45, 1.573, 0.2643)]
    zones = [Zone(factor * k, factor * k, factor * k, phi, a, n, sr) for k, phi, a, n, sr in rows]
    bcs = [BC(1, 3, 0.0, 0.0, 0.0), BC(2, 3, -2.3148e-7, 0.0, 0.0)]
    return zones, bcs, -7.34


CONFIGS = {
    "richards2d": Config("richards2d: 81x41 jittered Delaunay, 2 layers, 1 day", "2d",
                         dict(nx=81, ny=41, Lx=10.0, Ly=5.0, jitter=0.2, seed=1)),
    "ensemble2d": Config("ensemble2d: 256 independent 2D meshes, 2k-40k nodes each, own lognormal Ks, 1 day",
                         "ensemble2d", dict(n_members=256, nmin=2000, nmax=40000, seed=1)),
    "richards3d": Config("richards3d: 100x100x20 hex -> 6 tets (214,221 nodes), lognormal Ks, 30 days", "3d",
                         dict(nx=100, ny=100, nz=20, Lx=100.0, Ly=100.0, Lz=20.0, jitter=0.15, seed=1,
                              ln_var=1.0, cx=10.0, cy=10.0, cz=2.0, Kg=1e-5)),
    "richards3d_1m": Config("richards3d_1m: 200x200x25 hex -> 6 tets (1,050,426 nodes), the 3D statistics", "3d",
                            dict(nx=200, ny=200, nz=25, Lx=200.0, Ly=200.0, Lz=25.0, jitter=0.15, seed=1,
                                 ln_var=1.0, cx=10.0, cy=10.0, cz=2.0, Kg=1e-5)),
}


def make_problem(name: str, **override) -> Problem:
    cfg = CONFIGS[name]
    p = dict(cfg.params)
    p.update(override)
    return Problem(cfg.kind, **p)
