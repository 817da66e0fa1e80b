"""Generate the committed golden fixtures from the reference tree.

Run once in a container that has the reference checkout (read-only):

    python tests/golden/make_fixtures.py /path/to/fesom-c

It writes tests/golden/le_medium.npz with the LE_medium lock-exchange test
case of the reference (test_cases/LE_medium):

  nod_xy, nod_index   MESH/nod2d.out  (lon/lat in degrees, node flag)
  elem_nodes          MESH/elem2d.out (4 nodes per row, 1-based)
  edges, edge_tri     MESH/edges.out, MESH/edge_tri.out (edge list written by
                      the reference's mesh tooling; internal edges first)
  edgenum             MESH/edgenum.out (total, internal)
  energy              postproc/energy_tocheck.dat, first ENERGY_ROWS rows of
                      (model days, domain energy per unit area), printed by
                      the reference with format 4e16.7 every IREP=100 steps
                      (src/fv_main.F90:619)

The GPU box has no reference checkout, so the tests read only this file.
"""
import os
import sys

import numpy as np

ENERGY_ROWS = 2000


def _ints(path):
    with open(path) as f:
        return [list(map(int, line.split())) for line in f if line.strip()]


def main(ref_root):
    case = os.path.join(ref_root, "test_cases", "LE_medium")
    mesh = os.path.join(case, "MESH")
    with open(os.path.join(mesh, "nod2d.out")) as f:
        n = int(f.readline())
        rows = [f.readline().split() for _ in range(n)]
    nod_id = np.array([int(r[0]) for r in rows], dtype=np.int32)
    assert np.array_equal(nod_id, np.arange(1, n + 1))
    nod_xy = np.array([[float(r[1]), float(r[2])] for r in rows], dtype=np.float64)
    nod_index = np.array([int(r[3]) for r in rows], dtype=np.int32)
    with open(os.path.join(mesh, "elem2d.out")) as f:
        e = int(f.readline())
        vals = np.array(f.read().split(), dtype=np.int32)
    elem_nodes = vals[: 4 * e].reshape(e, 4)
    edges = np.array(_ints(os.path.join(mesh, "edges.out")), dtype=np.int32)
    edge_tri = np.array(_ints(os.path.join(mesh, "edge_tri.out")), dtype=np.int32)
    edgenum = np.array([r[0] for r in _ints(os.path.join(mesh, "edgenum.out"))], dtype=np.int32)
    energy = np.loadtxt(os.path.join(case, "postproc", "energy_tocheck.dat"), max_rows=ENERGY_ROWS)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "le_medium.npz")
    np.savez_compressed(out, nod_xy=nod_xy, nod_index=nod_index, elem_nodes=elem_nodes,
                        edges=edges, edge_tri=edge_tri, edgenum=edgenum, energy=energy)
    print("wrote", out, "nodes", n, "elements", e, "edges", len(edges), "energy rows", len(energy))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_fixtures.py <path to the fesom-c checkout>")
    main(sys.argv[1])
