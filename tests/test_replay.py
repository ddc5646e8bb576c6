"""Step-sequence replay on the CPU (no GPU).

The oracle restates the fixed-leading-coefficient BDF step independently of
the product's controller: a replayed step's predictor is the polynomial
through the newest solution values in Lagrange form (orc_replay).  The same
sequence replayed through the controller template
(fvmb::bdf_replay_step, modified divided differences) on the same oracle
kernels must give the same state to the corrector tolerance, which pins the
controller's predictor and corrector formulas.  Also checked here: the
oracle's own copy of the benchmark generator reproduces the product's
meshes exactly, and a process that times the CPU oracle never loads the
product library.
"""
import os
import subprocess
import sys

import numpy as np

from oracle.pyoracle import Oracle, make_problem, opts

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_replay_lagrange_form_matches_controller():
    p = make_problem("richards2d", nx=21, ny=11)
    o = Oracle(p)
    y0 = o.initial_head()
    op = opts(krylov_dim=30)
    rc, ya, st = o.integrate(op, 1, 0.0, 6 * 3600.0, y0)
    assert rc == 0
    tr = o.trace()
    assert len(tr) == st["nst"] and tr["order"].max() >= 3
    h0 = float(tr["h"][0])
    r1, y1, s1 = o.replay(op, 1, 0.0, y0, h0, tr, newton_tol=1e-6)
    r2, y2, s2 = o.replay(op, 1, 0.0, y0, h0, tr, newton_tol=1e-6, controller=True)
    assert r1 == 0 and r2 == 0
    assert s1["nst"] == s2["nst"] == len(tr)
    assert abs(s1["t"] - s2["t"]) <= 1e-12 * s1["t"]
    scale = np.abs(y1).max()
    # tight correctors: the two forms agree far below the 1e-10 target
    assert np.abs(y1 - y2).max() <= 1e-11 * scale
    # and the replay stays within the adaptive run's own Newton tolerance
    assert np.abs(y1 - ya).max() <= 1e-5 * scale


def test_replay_rejects_bad_sequences():
    p = make_problem("richards2d", nx=11, ny=6)
    o = Oracle(p)
    y0 = o.initial_head()
    rec = np.zeros(2, dtype=[("t", "f8"), ("h", "f8"), ("order", "i4")])
    rec["h"] = [1.0, 1.0]
    rec["order"] = [1, 3]   # the history holds 3 points after one step
    import pytest

    with pytest.raises(RuntimeError):
        o.replay(opts(), 1, 0.0, y0, 1.0, rec)


def test_oracle_generator_matches_product_generator():
    import fvmpor_b200 as fb

    for name, kw in (("richards2d", {}), ("richards3d", dict(nx=12, ny=10, nz=6, Lx=12.0, Ly=10.0, Lz=6.0))):
        a = fb.make_problem(name, **kw).arrays()
        b = make_problem(name, **kw).arrays()
        for k in b:
            assert np.array_equal(a[k], b[k]), (name, k)


def test_cpu_reference_process_does_not_load_the_product_library():
    code = (
        "import sys; sys.path.insert(0, %r)\n"
        "import numpy as np\n"
        "from oracle.pyoracle import Oracle, make_problem\n"
        "p = make_problem('richards2d', nx=11, ny=6)\n"
        "o = Oracle(p)\n"
        "y = o.initial_head()\n"
        "r = o.residual(0.0, y, np.zeros_like(y))\n"
        "maps = open('/proc/self/maps').read()\n"
        "assert 'libfvmpor_b200' not in maps, 'product library mapped'\n"
        "print('ok', float(np.abs(r).max()))\n" % ROOT)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert out.stdout.startswith("ok")
