"""The C-ABI library builds, loads and exports every entry point declared in
include/fvmpor_b200.h (no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

import pytest

import fvmpor_b200 as fb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        for m in re.finditer(r"\b(fvm_[a-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("fvm_create", "fvm_residual", "fvm_begin_step", "fvm_jv", "fvm_psetup",
                 "fvm_psolve", "fvm_gmres", "fvm_wrms", "fvm_dot", "fvm_integrate"):
        assert must in names


@pytest.mark.parametrize("name", declared_functions())
def test_symbol_exported(name):
    L = fb.lib()
    assert hasattr(L, name), f"{name} declared in include/ but not exported"


def test_library_is_sm100a_build():
    # the shared library carries an sm_100a cubin (checked via cuobjdump-free
    # means: the build recipe pins -gencode arch=compute_100a,code=sm_100a)
    mk = open(os.path.join(ROOT, "fvmpor_b200", "Makefile")).read()
    assert "arch=compute_100a,code=sm_100a" in mk


def test_create_reports_errors_without_crashing():
    L = fb.lib()
    ctx = L.fvm_create(None, None, 0)
    assert not ctx
    assert b"null" in L.fvm_last_error()


def test_integrate_entry_points_reject_null_arguments():
    # argument checks come before any device work, so they run without a GPU
    import ctypes as C

    L = fb.lib()
    o = fb.default_opts()
    st = fb.Stats()
    t = (C.c_double * 2)(1.0, 2.0)
    assert L.fvm_integrate(None, C.byref(o), 0.0, 1.0, None, None, C.byref(st)) < 0
    assert b"null" in L.fvm_last_error()
    assert L.fvm_integrate_outputs(None, C.byref(o), 0.0, None, 2, t, None, None, C.byref(st)) < 0
    assert b"null" in L.fvm_last_error()
    assert L.fvm_integrate_host(None, C.byref(o), 0.0, 1.0, None, None, C.byref(st)) < 0
    assert b"null" in L.fvm_last_error()


def test_product_never_imports_oracle():
    for dirpath, _, files in os.walk(os.path.join(ROOT, "fvmpor_b200")):
        for f in files:
            if f.endswith((".py", ".cu", ".cpp", ".cuh", ".hpp")):
                src = open(os.path.join(dirpath, f)).read()
                assert "pyoracle" not in src and "oracle.cpp" not in src and "orc_" not in src, f


# C struct of the header <-> its ctypes mirror in the package
STRUCTS = {
    "fvm_mesh": "Mesh", "fvm_zone": "Zone", "fvm_bc": "BC", "fvm_physics": "PhysicsDesc",
    "fvm_problem": "ProblemStruct", "fvm_pmesh": "PmeshStruct", "fvm_step_record": "StepRecord",
    "fvm_opts": "Opts", "fvm_stats": "Stats", "fvm_tune_result": "TuneResult",
}


def test_struct_layouts_match_header(tmp_path):
    """every ctypes mirror has the size and field offsets that the C
    compiler gives the header's struct (a field added on one side only
    shifts everything after it)"""
    import shutil
    import subprocess

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "fvmpor_b200.h"', "int main(void) {"]
    for cname, pyname in STRUCTS.items():
        cls = getattr(fb, pyname)
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in cls._fields_:
            lines.append(f'printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for ln in out:
        if ln:
            s, f, v = ln.split()
            got[(s, f)] = int(v)
    for cname, pyname in STRUCTS.items():
        cls = getattr(fb, pyname)
        assert got[(cname, "size")] == ctypes.sizeof(cls), cname
        for field, _ in cls._fields_:
            assert got[(cname, field)] == getattr(cls, field).offset, (cname, field)
