"""Builds the caisson fixtures from a checkout of the reference.

The reference ships one stored run: the EEM example's caisson infiltration
problem (examples/EEM/fvmpor_ODE.cpp, physics examples/EEM/cassion.h), run
on meshing/meshes/cassion_1_0.pmesh to t = 2.5e6 s with rtol = atol = 5e-4,
written as VTK XML at t_k = k * 2.5e6 / 11, k = 0..11
(examples/EEM/CASS_dom0_<k>.vtu; times in examples/EEM/output/
MPI_solution_1_0.log).  This script stores

  cassion_1_0.pmesh.gz   the mesh file, unchanged (gzip)
  cassion_eem.npz        from the .vtu files: points [1599, 3] and
                         connectivity [3064, 3] (the reference's node order
                         after its reverse Cuthill-McKee renumbering),
                         pressure head [12, 1599] at the times t [12]

Values in the .vtu files are 6-significant-digit ASCII; they are stored as
float64 exactly as parsed.

usage: python tests/golden/make_cassion.py /path/to/reference
"""
import gzip
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def arrays(path):
    txt = open(path).read()
    out = {}
    for hdr, body in re.findall(r"<DataArray([^>]*)>(.*?)</DataArray>", txt, re.S):
        name = re.search(r'Name="([^"]*)"', hdr)
        out[name.group(1) if name else "Points"] = np.array(body.split(), dtype=np.float64)
    return out


def main(ref):
    mesh = os.path.join(ref, "meshing", "meshes", "cassion_1_0.pmesh")
    with open(mesh, "rb") as f, gzip.open(os.path.join(HERE, "cassion_1_0.pmesh.gz"), "wb", 9) as g:
        g.write(f.read())
    heads = []
    pts = conn = None
    for k in range(12):
        a = arrays(os.path.join(ref, "examples", "EEM", f"CASS_dom0_{k}.vtu"))
        heads.append(a["pressure_head"])
        if pts is None:
            pts = a["Points"].reshape(-1, 3)
            conn = a["connectivity"].astype(np.int32).reshape(-1, 3)
        else:
            assert np.array_equal(pts, a["Points"].reshape(-1, 3))
    t = np.arange(12) * 2.5e6 / 11
    np.savez_compressed(os.path.join(HERE, "cassion_eem.npz"), points=pts, connectivity=conn,
                        head=np.array(heads), t=t)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_cassion.py /path/to/reference")
    main(sys.argv[1])
