"""The .pmesh reader, the VTK writer and the caisson run.

The reference's only stored results are the EEM example's caisson run
(examples/EEM/CASS_dom0_<k>.vtu, on meshing/meshes/cassion_1_0.pmesh),
kept as fixtures under tests/golden/ by make_cassion.py.  They pin:

* the reader and its reverse Cuthill-McKee renumbering against the node
  order the reference wrote (connectivity bit-identical, points equal to
  the files' 6 significant digits);
* the discretisation and the BDF integration, loosely: the reference ran
  an exponential integrator at rtol = atol = 5e-4, so its heads carry its
  own time error; ours (rtol = atol = 1e-6) must agree to 0.06 m in max
  norm (under 1% of the 6.9 m head range) and 5e-3 m rms at every stored
  time.
"""
import gzip
import os
import xml.etree.ElementTree as ET

import numpy as np
import pytest

import fvmpor_b200 as fb

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
MAX_DIFF_M = 0.06
RMS_DIFF_M = 5e-3


@pytest.fixture(scope="module")
def cass_path(tmp_path_factory):
    d = tmp_path_factory.mktemp("cass")
    p = d / "cassion_1_0.pmesh"
    p.write_bytes(gzip.open(os.path.join(GOLD, "cassion_1_0.pmesh.gz")).read())
    return p


@pytest.fixture(scope="module")
def eem():
    return np.load(os.path.join(GOLD, "cassion_eem.npz"))


def test_reader_counts_and_tags(cass_path):
    pm = fb.read_pmesh(cass_path, rcm=False)
    assert (pm.dim, pm.n_nodes, pm.n_elements) == (2, 1599, 3064)
    assert np.bincount(pm.elem_tag).tolist() == [232, 266, 2320, 246]
    tags, counts = np.unique(pm.bface_tag, return_counts=True)
    assert tags.tolist() == [1, 2] and counts.tolist() == [116, 16]
    assert np.array_equal(pm.perm, np.arange(1599))
    # every boundary face is a face of its element
    for b in range(pm.n_bfaces):
        assert set(pm.bface_nodes[b]) <= set(pm.elem_nodes[pm.bface_elem[b]])
    assert np.all(pm.coords[:, 2] == 0.0)


def test_rcm_reproduces_reference_node_order(cass_path, eem):
    pm = fb.read_pmesh(cass_path)
    assert pm.bandwidth < pm.bandwidth_file  # 1466 -> 63
    assert sorted(pm.perm.tolist()) == list(range(pm.n_nodes))
    assert np.array_equal(pm.elem_nodes, eem["connectivity"])
    rel = np.abs(pm.coords - eem["points"]) / np.maximum(1.0, np.abs(eem["points"]))
    assert rel.max() <= 5e-6  # 6-significant-digit text
    raw = fb.read_pmesh(cass_path, rcm=False)
    assert np.array_equal(raw.coords[pm.perm], pm.coords)


def test_rcm_on_shuffled_grid_reduces_bandwidth(tmp_path):
    p = fb.make_problem("richards2d", nx=31, ny=17)
    a0 = p.arrays()
    rng = np.random.default_rng(3)
    sh = rng.permutation(p.n_nodes).astype(np.int32)  # new -> old
    inv = np.empty_like(sh)
    inv[sh] = np.arange(p.n_nodes, dtype=np.int32)
    be = np.ctypeslib.as_array(p.mesh.bface_elem, (p.mesh.n_bfaces,)).copy()
    zones = [p.phys.zones[i] for i in range(p.phys.n_zones)]
    bcs = [p.phys.bcs[i] for i in range(p.phys.n_bcs)]
    ps = fb.Problem.from_arrays(2, a0["coords"][sh], inv[a0["elem_nodes"]], a0["elem_zone"], inv[a0["bface_nodes"]],
                                be, a0["bface_tag"], a0["node_tag"][sh], zones, bcs)
    pm = fb.Pmesh.from_problem(ps)
    pm.write(tmp_path / "shuffled.pmesh")
    a = fb.read_pmesh(tmp_path / "shuffled.pmesh", rcm=False)
    b = fb.read_pmesh(tmp_path / "shuffled.pmesh")
    assert b.bandwidth < a.bandwidth / 5
    assert np.array_equal(a.coords[b.perm], b.coords)
    # same elements, renumbered
    q = np.empty(p.n_nodes, np.int64)
    q[b.perm] = np.arange(p.n_nodes)
    assert np.array_equal(q[a.elem_nodes], b.elem_nodes)


@pytest.mark.parametrize("kind", ["2d", "3d"])
def test_write_read_roundtrip(tmp_path, kind):
    p = fb.make_problem("richards2d", nx=13, ny=7) if kind == "2d" else fb.make_problem(
        "richards3d", nx=5, ny=4, nz=3, Lx=5.0, Ly=4.0, Lz=3.0)
    pm = fb.Pmesh.from_problem(p)
    pm.write(tmp_path / "m.pmesh")
    r = fb.read_pmesh(tmp_path / "m.pmesh", rcm=False)
    assert (r.dim, r.n_nodes, r.n_elements) == (pm.dim, pm.n_nodes, pm.n_elements)
    assert np.array_equal(r.coords, pm.coords)  # %.17g round-trips
    assert np.array_equal(r.elem_nodes, pm.elem_nodes)
    assert np.array_equal(r.elem_tag, pm.elem_tag)
    key = lambda n, e, t: sorted((tuple(sorted(x)), int(y), int(z)) for x, y, z in zip(n, e, t))
    assert key(r.bface_nodes, r.bface_elem, r.bface_tag) == key(pm.bface_nodes, pm.bface_elem, pm.bface_tag)
    assert np.array_equal(r.node_bc_ptr, pm.node_bc_ptr) and np.array_equal(r.node_bc, pm.node_bc)


BAD = {
    "truncated": ("1 0\n0 3\n3 3 0 0 1 0\n0 0 0 0\n1 0 0 0\n", -2, "end of file"),
    "quad": ("1 0\n0 4\n4 4 0 0 1 0\n0 0 0 0\n1 0 0 0\n1 1 0 0\n0 1 0 0\n3 100 0 1 2 3 0 0 0 0\n", -4,
             "quadrilateral"),
    "halo": ("2 0\n0 3 6\n6 3 0 1 1 0\n5\n", -3, "halo"),
    "node_range": ("1 0\n0 3\n3 3 0 0 1 0\n0 0 0 0\n1 0 0 0\n0 1 0 0\n2 100 0 1 7 0 0 0\n", -2, "out of range"),
    "not_a_number": ("1 0\n0 3\n3 3 0 0 1 0\n0 0 zero 0\n", -2, "expected a number"),
}


@pytest.mark.parametrize("case", sorted(BAD))
def test_reader_errors(tmp_path, case):
    text, code, words = BAD[case]
    f = tmp_path / f"{case}.pmesh"
    f.write_text(text)
    with pytest.raises(fb.FvmError) as ei:
        fb.read_pmesh(f)
    assert f"status {code}" in str(ei.value) and words in str(ei.value)


def test_reader_missing_file(tmp_path):
    with pytest.raises(fb.FvmError, match="cannot open"):
        fb.read_pmesh(tmp_path / "nope.pmesh")


def test_problem_from_pmesh_tags(cass_path):
    zones, bcs, _ = fb.cassion_physics()
    pm = fb.read_pmesh(cass_path)
    p = fb.Problem.from_pmesh(pm, zones, bcs)
    a = p.arrays()
    assert np.all(a["node_tag"] == 0)  # no Dirichlet condition in the caisson problem
    assert np.array_equal(a["elem_zone"], pm.elem_tag)
    # a Dirichlet condition on tag 1 marks exactly the nodes that carry tag 1
    dbc = [fb.BC(1, 1, -1.0, 0.0, 0.0), bcs[1]]
    p2 = fb.Problem.from_pmesh(pm, zones, dbc)
    has1 = np.array([1 in pm.node_bc[pm.node_bc_ptr[i]:pm.node_bc_ptr[i + 1]] for i in range(pm.n_nodes)])
    assert np.array_equal(p2.arrays()["node_tag"] == 1, has1)
    with pytest.raises(fb.FvmError, match="no boundary condition"):
        fb.Problem.from_pmesh(pm, zones, bcs[:1])
    with pytest.raises(fb.FvmError, match="outside the 3 zones"):
        fb.Problem.from_pmesh(pm, zones[:3], bcs)


def _vtu_arrays(path):
    root = ET.parse(path).getroot()
    out = {}
    for da in root.iter("DataArray"):
        out[da.get("Name") or "Points"] = (da.get("type"), np.array(da.text.split(), dtype=np.float64))
    return root, out


def test_vtu_writer(tmp_path, cass_path, eem):
    zones, bcs, h0 = fb.cassion_physics()
    p = fb.Problem.from_pmesh(cass_path, zones, bcs)
    head = eem["head"][5] + 1e-7 * np.arange(p.n_nodes)
    p.write_vtu(tmp_path / "CASS", 5, head)
    root, arr = _vtu_arrays(tmp_path / "CASS_dom0_5.vtu")
    piece = root.find("UnstructuredGrid/Piece")
    assert piece.get("NumberOfPoints") == "1599" and piece.get("NumberOfCells") == "3064"
    assert arr["pressure_head"][0] == "Float32"
    # 9 digits identify the Float32 value exactly
    assert np.array_equal(arr["pressure_head"][1].astype(np.float32), head.astype(np.float32))
    assert np.array_equal(arr["connectivity"][1].reshape(-1, 3), eem["connectivity"])
    assert np.array_equal(arr["offsets"][1], 3 * np.arange(1, 3065))
    assert np.all(arr["types"][1] == 5) and np.all(arr["dom"][1] == 0)
    assert np.abs(arr["Points"][1].reshape(-1, 3) - eem["points"]).max() < 1e-4
    hdr = ET.parse(tmp_path / "CASS_head_5.pvtu").getroot()
    assert [pc.get("Source") for pc in hdr.iter("Piece")] == ["CASS_dom0_5.vtu"]
    with pytest.raises(ValueError):
        p.write_vtu(tmp_path / "x", 0, head[:-1])


def _compare(y, ref):
    d = y - ref
    return float(np.abs(d).max()), float(np.sqrt(np.mean(d * d)))


def test_cassion_oracle_matches_reference_run(cass_path, eem):
    from oracle.pyoracle import Oracle

    zones, bcs, h0 = fb.cassion_physics()
    p = fb.Problem.from_pmesh(cass_path, zones, bcs)
    assert np.all(eem["head"][0] == h0)
    o = Oracle(p)
    opts = fb.default_opts(krylov_dim=30, max_order=5, rtol=1e-6, atol=1e-6)
    y, t = np.full(p.n_nodes, h0), 0.0
    for k in range(1, 12):
        rc, y, st = o.integrate(opts, 1, t, eem["t"][k], y)
        t = eem["t"][k]
        assert rc == 0 and abs(st["t"] - t) < 1e-6 * t
        mx, rms = _compare(y, eem["head"][k])
        assert mx < MAX_DIFF_M and rms < RMS_DIFF_M, (k, mx, rms)


def test_cassion_oracle_dense_output_matches_reference_run(cass_path, eem):
    """one continuous run through the stored output times, heads interpolated
    at each as the reference's advance(next_time) does (no restart at the
    output times: 739 steps against 969 with restarts)"""
    from oracle.pyoracle import Oracle

    zones, bcs, h0 = fb.cassion_physics()
    p = fb.Problem.from_pmesh(cass_path, zones, bcs)
    o = Oracle(p)
    opts = fb.default_opts(krylov_dim=30, max_order=5, rtol=1e-6, atol=1e-6)
    rc, Y, YP, st = o.integrate_outputs(opts, 1, 0.0, np.full(p.n_nodes, h0), eem["t"][1:12])
    assert rc == 0 and st["t"] >= eem["t"][11]
    for k in range(1, 12):
        mx, rms = _compare(Y[k - 1], eem["head"][k])
        assert mx < MAX_DIFF_M and rms < RMS_DIFF_M, (k, mx, rms)


@pytest.mark.gpu
def test_cassion_device_dense_output_matches_reference_run_and_oracle(cass_path, eem):
    import torch

    from oracle.pyoracle import Oracle

    zones, bcs, h0 = fb.cassion_physics()
    p = fb.Problem.from_pmesh(cass_path, zones, bcs)
    ph = fb.Physics(p)
    tout = eem["t"][1:12]
    y0 = torch.full((p.n_nodes,), h0, dtype=torch.float64, device="cuda")
    Y = torch.empty(len(tout), p.n_nodes, dtype=torch.float64, device="cuda")
    rc, st = fb.Integrator(ph, krylov_dim=30, max_order=5).integrate_outputs(0.0, tout, y0, Y)
    assert rc == 0
    opts = fb.default_opts(krylov_dim=30, max_order=5)
    rc, Yo, _, _ = Oracle(p).integrate_outputs(opts, 1, 0.0, np.full(p.n_nodes, h0), tout)
    assert rc == 0
    Yg = Y.cpu().numpy()
    for k in range(1, 12):
        mx, rms = _compare(Yg[k - 1], eem["head"][k])
        assert mx < MAX_DIFF_M and rms < RMS_DIFF_M, (k, mx, rms)
        assert np.abs(Yg[k - 1] - Yo[k - 1]).max() < 2e-3, (k, np.abs(Yg[k - 1] - Yo[k - 1]).max())


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_cassion_device_matches_reference_run_and_oracle(cass_path, eem, precision):
    from oracle.pyoracle import Oracle

    zones, bcs, h0 = fb.cassion_physics()
    p = fb.Problem.from_pmesh(cass_path, zones, bcs)
    ph = fb.Physics(p)
    integ = fb.Integrator(ph, krylov_dim=30, max_order=5, rtol=1e-6, atol=1e-6, precision=precision)
    o = Oracle(p)
    opts = fb.default_opts(krylov_dim=30, max_order=5, rtol=1e-6, atol=1e-6)
    y = np.full(p.n_nodes, h0)
    yo = y.copy()
    t = 0.0
    for k in range(1, 12):
        ye = np.zeros(p.n_nodes)
        rc, st = integ.integrate_host(t, eem["t"][k], y, ye)
        assert rc == 0
        rc, yo, _ = o.integrate(opts, 1, t, eem["t"][k], yo)
        assert rc == 0
        y, t = ye, eem["t"][k]
        mx, rms = _compare(y, eem["head"][k])
        assert mx < MAX_DIFF_M and rms < RMS_DIFF_M, (k, mx, rms)
        # device and oracle: both solve to 1e-6, different Krylov and
        # preconditioner arithmetic
        assert np.abs(y - yo).max() < 2e-3, (k, np.abs(y - yo).max())
