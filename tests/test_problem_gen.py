"""Synthetic benchmark problems: sizes, Delaunay property, orientation,
boundary tags and the lognormal conductivity field."""
import numpy as np
import pytest

import fvmpor_b200 as fb


def test_richards2d_sizes_and_delaunay():
    from scipy.spatial import Delaunay

    p = fb.make_problem("richards2d")
    a = p.arrays()
    assert p.n_nodes == 81 * 41 == 3321
    assert p.n_elements == 6400
    d = Delaunay(a["coords"][:, :2])
    assert set(map(tuple, np.sort(d.simplices, 1))) == set(map(tuple, np.sort(a["elem_nodes"], 1)))
    X = a["coords"]
    e = a["elem_nodes"]
    area = 0.5 * ((X[e[:, 1], 0] - X[e[:, 0], 0]) * (X[e[:, 2], 1] - X[e[:, 0], 1])
                  - (X[e[:, 1], 1] - X[e[:, 0], 1]) * (X[e[:, 2], 0] - X[e[:, 0], 0]))
    assert (area > 0).all()
    assert abs(area.sum() - 50.0) < 1e-10
    assert len(a["bface_tag"]) == 2 * 80 + 2 * 40
    top = a["node_tag"] == 2
    assert top.sum() > 0 and np.all(np.abs(X[top, 1] - 5.0) < 1e-12)
    assert np.all((X[top, 0] >= 4.0 - 1e-9) & (X[top, 0] <= 6.0 + 1e-9))
    # zones split at y = 2.5
    yc = X[e, 1].mean(1)
    assert np.all(a["elem_zone"] == (yc >= 2.5))


def test_richards2d_reproducible_by_seed():
    a = fb.make_problem("richards2d", seed=7).arrays()
    b = fb.make_problem("richards2d", seed=7).arrays()
    c = fb.make_problem("richards2d", seed=8).arrays()
    assert np.array_equal(a["coords"], b["coords"])
    assert not np.array_equal(a["coords"], c["coords"])


def test_richards3d_small_box():
    p = fb.make_problem("richards3d", nx=10, ny=8, nz=5, Lx=10.0, Ly=8.0, Lz=5.0)
    a = p.arrays()
    assert p.n_nodes == 11 * 9 * 6
    assert p.n_elements == 6 * 10 * 8 * 5
    X, e = a["coords"], a["elem_nodes"]
    u = X[e[:, 1]] - X[e[:, 0]]
    v = X[e[:, 2]] - X[e[:, 0]]
    w = X[e[:, 3]] - X[e[:, 0]]
    vol = np.einsum("ij,ij->i", u, np.cross(v, w)) / 6.0
    assert (vol > 0).all()
    assert abs(vol.sum() - 400.0) < 1e-9
    # every boundary cell face is split into two triangles
    assert len(a["bface_tag"]) == 2 * 2 * (10 * 8 + 10 * 5 + 8 * 5)
    assert np.all(a["node_tag"][np.abs(X[:, 0]) < 1e-12] == 3)


def test_benchmark_box_sizes():
    p = fb.make_problem("richards3d")
    assert p.n_nodes == 101 * 101 * 21 == 214221
    assert p.n_elements == 1_200_000
    lk = np.log(p.arrays()["elem_K"])
    # ln-variance 1.0 (within sampling error of a 10 m correlated field)
    assert 0.6 < lk.var() < 1.4


def test_lognormal_field_statistics_2d():
    # many independent small fields: pooled ln-variance matches the target
    v = []
    for s in range(12):
        p = fb.Problem("2d", nx=41, ny=21, ln_var=1.5, corr_len=0.5, seed=100 + s)
        a = p.arrays()
        lk = np.log(a["elem_K"] / np.where(a["elem_zone"] == 0, 1e-5, 1e-6))
        v.append(lk.var())
    assert 1.1 < np.mean(v) < 1.9
