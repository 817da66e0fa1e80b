"""Host mesh builder: pinned against the reference's own mesh files and
checked for the invariants the time step relies on."""
import numpy as np
import pytest

from conftest import ROOT
import os


@pytest.fixture(scope="module")
def le(built):
    from fesomc import cases
    return cases.le_medium(), np.load(os.path.join(ROOT, "tests", "golden", "le_medium.npz"))


def test_le_edges_match_reference_files(le):
    case, g = le
    m = case.mesh
    assert (m.Ed, m.Ed_in) == tuple(g["edgenum"])
    np.testing.assert_array_equal(m.edge_nodes, g["edges"])
    np.testing.assert_array_equal(m.edge_tri, g["edge_tri"])


def test_le_geometry_invariants(le):
    case, _ = le
    m = case.mesh
    np.testing.assert_allclose(m.w_cv.sum(axis=1), 1.0, rtol=0, atol=1e-14)
    assert abs(m.area.sum() / m.elem_area.sum() - 1.0) < 1e-13
    # every internal edge lists two elements that are neighbours of each other
    et = m.edge_tri[: m.Ed_in] - 1
    nb = m.elem_neighbors - 1
    for a, b in et[:500]:
        assert b in nb[a] and a in nb[b]
    # boundary edges carry -999 as second element
    assert np.all(m.edge_tri[m.Ed_in:, 1] == -999)
    # gradient of a linear function is exact on every element
    x = m.coord_nod2D[:, 0]
    en = m.elem2D_nodes - 1
    gx = (m.gradient_sca[:, :4] * x[en]).sum(axis=1)
    gy = (m.gradient_sca[:, 4:] * x[en]).sum(axis=1)
    assert np.all(np.abs(gy) < 1e-20 + 1e-9 * np.abs(gx).max())


def test_estuary_counts(built):
    from fesomc import cases
    xy, idx, el, dep, (nxn, nyn) = cases.estuary_geometry(40, 16, 300.0)
    ntri = int((el[:, 0] == el[:, 3]).sum())
    assert len(xy) == 41 * 17
    assert len(el) - ntri // 2 == 40 * 16            # each split quad -> two triangles
    assert 0.2 < (ntri // 2) / (40 * 16) < 0.4        # ~30 % split
    m = cases.HostMesh(xy, idx, el, dep, cartesian=True, nsigma=11)
    # Euler: E + N - Ed = 1 for a simply connected planar mesh
    assert m.E + m.N - m.Ed == 1
    assert m.Ed - m.Ed_in == 2 * (40 + 16)
    np.testing.assert_allclose(m.w_cv.sum(axis=1), 1.0, atol=1e-14)
    assert abs(m.area.sum() - 40 * 16 * 300.0 * 300.0) < 1e-6 * m.area.sum()
    ud = m.edge_up_dn_tri
    assert (ud > 0).all(axis=1).mean() > 0.8


def _sponge_restatement(m, radius, cartesian):
    """ac_create / Dist2in1 (src/fv_utilit.F90:53-88,184-220) in numpy."""
    p = m.coord_nod2D
    ob = p[m.index_nod2D == 2]
    r_earth = 6400000.0                                   # r_earth, src/fv_var.F90
    if cartesian:
        d = ((ob[None, :, 0] - p[:, None, 0]) ** 2 + (ob[None, :, 1] - p[:, None, 1]) ** 2).min(axis=1)
        dist = np.sqrt(d) * r_earth
    else:
        a = (np.sin((ob[None, :, 1] - p[:, None, 1]) * 0.5) ** 2
             + np.cos(p[:, None, 1]) * np.cos(ob[None, :, 1]) * np.sin((ob[None, :, 0] - p[:, None, 0]) * 0.5) ** 2)
        dist = 2.0 * r_earth * np.arcsin(np.minimum(1.0, np.sqrt(a.min(axis=1))))
    return np.where(dist < radius, dist / radius, 1.0)


@pytest.mark.parametrize("cartesian", [True, False])
def test_sponge_layer(built, cartesian):
    from fesomc import cases
    xy, idx, el, dep, (nxn, nyn) = cases.estuary_geometry(40, 16, 300.0)
    if not cartesian:
        xy = xy / 300.0 * 0.01 + np.array([5.0, 50.0])   # degrees, 0.01 degree spacing
    radius = 2000.0
    m = cases.HostMesh(xy, idx, el, dep, cartesian=cartesian, nsigma=5, with_up_dn_tri=False,
                       sponge_radius=radius)
    ac = m.ac
    ob = m.index_nod2D == 2
    assert ob.sum() == nyn
    np.testing.assert_array_equal(ac[ob], 0.0)
    assert ac.max() == 1.0 and 0.0 < ac[~ob].min() < 1.0
    np.testing.assert_allclose(ac, _sponge_restatement(m, radius, cartesian), rtol=1e-13, atol=1e-15)
    # without a sponge radius every node keeps the full terms
    m0 = cases.HostMesh(xy, idx, el, dep, cartesian=cartesian, nsigma=5, with_up_dn_tri=False)
    np.testing.assert_array_equal(m0.ac, 1.0)


def test_sponge_rejects_bad_radius(built):
    from fesomc import cases
    xy, idx, el, dep, _ = cases.estuary_geometry(8, 4, 300.0)
    with pytest.raises(RuntimeError, match="EINVAL"):
        cases.HostMesh(xy, idx, el, dep, cartesian=True, nsigma=5, with_up_dn_tri=False, sponge_radius=-1.0)


def test_orientation_fixed_and_bad_quad_rejected(built):
    from fesomc import cases
    xy = np.array([[0, 0], [1, 0], [1, 1], [0, 1], [2, 0], [2, 1]], float) * 100.0
    idx = np.ones(6, np.int32)
    # counter-clockwise quads are reordered to clockwise by test_elem
    el = np.array([[1, 2, 3, 4], [2, 5, 6, 3]], np.int32)
    m = cases.HostMesh(xy, idx, el, np.full(6, 10.0), cartesian=True, nsigma=5, with_up_dn_tri=False)
    e = m.elem2D_nodes
    p = m.coord_nod2D
    for q in e - 1:
        b = p[q[1]] - p[q[0]]
        c = p[q[2]] - p[q[0]]
        assert b[0] * c[1] - b[1] * c[0] < 0
    # a self-intersecting (bow-tie) quad is the reference's "Node list problem"
    bad = np.array([[1, 3, 2, 4], [2, 5, 6, 3]], np.int32)
    with pytest.raises(RuntimeError, match="EMESH"):
        cases.HostMesh(xy, idx, bad, np.full(6, 10.0), cartesian=True, nsigma=5, with_up_dn_tri=False)
