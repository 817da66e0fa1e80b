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


MESH_ARRAYS = ["index_nod2D", "elem2D_nodes", "edge_nodes", "edge_tri", "elem_edges", "elem_neighbors",
               "nod_in_elem2D_num", "nod_in_elem2D", "edge_up_dn_tri", "coord_nod2D", "depth", "area", "elem_area",
               "elem_cos", "coriolis", "w_cv", "gradient_sca", "gradient_vec", "edge_dxdy", "edge_cross_dxdy",
               "sigma", "a_tp", "ac", "in_obn", "nod_rivers"]


def _same_mesh(a, b):
    assert (a.N, a.E, a.Ed, a.Ed_in, a.NS) == (b.N, b.E, b.Ed, b.Ed_in, b.NS)
    assert a.c.nod_in_elem2D_max == b.c.nod_in_elem2D_max
    assert a.scale_area == b.scale_area
    bad = [k for k in MESH_ARRAYS if not np.array_equal(getattr(a, k), getattr(b, k))]
    assert bad == []


@pytest.mark.parametrize("name", ["small", "cfg0"])
def test_oracle_mesh_equals_product_mesh_estuary(built, name):
    """The oracle's own restatement of the mesh set-up (oracle/oracle_mesh.c,
    written from the Fortran alone) and the product's host builder give the
    same arrays bit for bit on the estuary, whose 30 % triangles no reference
    file pins; this makes the oracle's inputs independent of the product."""
    import pyoracle
    from fesomc import abi, cases
    ol = pyoracle.MeshLib(abi)
    p = cases.estuary(name)
    o = cases.estuary(name, lib=ol)
    _same_mesh(p.mesh, o.mesh)
    assert p.params.density_0 == o.params.density_0
    for k in p.state0:
        assert np.array_equal(p.state0[k], o.state0[k]), k


def test_oracle_mesh_equals_product_mesh_le_and_tidal_potential(built):
    """LE (spherical coordinates, all quads), the a_tp weights of the tidal
    potential, and on a spherical estuary the ind_sigma = 2 (tanh) levels,
    rivers and the haversine sponge."""
    import pyoracle
    from fesomc import abi, cases
    ol = pyoracle.MeshLib(abi)
    _same_mesh(cases.le_medium().mesh, cases.le_medium(lib=ol).mesh)
    _same_mesh(cases.estuary("small", T_potential=1).mesh, cases.estuary("small", T_potential=1, lib=ol).mesh)
    xy, idx, el, dep, _ = cases.estuary_geometry(40, 16, 300.0)
    xy = xy / 300.0 * 0.01 + np.array([5.0, 50.0])
    kw = dict(cartesian=False, nsigma=21, ind_sigma=2, lev_bot=1.5, lev_sur=0.8, coriolis_on=True,
              sponge_radius=2000.0, rivers=[1, 42])
    _same_mesh(cases.HostMesh(xy, idx, el, dep, **kw), cases.HostMesh(xy, idx, el, dep, lib=ol, **kw))


def test_estuary_triangle_gradients_exact_for_linear_fields(built):
    """gradient_sca of a linear field is exact on every element of the
    estuary, triangles and quads alike (mesh_arrays2, fv_mesh_array.F90:
    1261-1302), and gradient_vec reproduces a linear velocity field exactly on
    interior elements (least squares over the neighbour centres); for the
    product's mesh builder and the oracle's."""
    import pyoracle
    from fesomc import abi, cases
    for lib in (None, pyoracle.MeshLib(abi)):
        m = cases.estuary("small", lib=lib).mesh
        en = m.elem2D_nodes - 1
        tri = en[:, 0] == en[:, 3]
        assert tri.sum() > 100
        p = m.coord_nod2D * cases.R_EARTH                  # metres (cartesian)
        f = 3.0 * p[:, 0] - 2.0 * p[:, 1]
        gx = (m.gradient_sca[:, :4] * f[en]).sum(axis=1)
        gy = (m.gradient_sca[:, 4:] * f[en]).sum(axis=1)
        # triangles carry a zero fourth weight, so the repeated node adds nothing
        np.testing.assert_array_equal(m.gradient_sca[tri][:, [3, 7]], 0.0)
        np.testing.assert_allclose(gx, 3.0, rtol=0, atol=1e-9)
        np.testing.assert_allclose(gy, -2.0, rtol=0, atol=1e-9)
        # element centres as the reference computes them (elem_center)
        xs, ys = p[:, 0], p[:, 1]
        s1 = np.abs((xs[en[:, 2]] - xs[en[:, 3]]) * (ys[en[:, 0]] - ys[en[:, 3]])
                    - (ys[en[:, 2]] - ys[en[:, 3]]) * (xs[en[:, 0]] - xs[en[:, 3]]))
        s2 = np.abs((xs[en[:, 2]] - xs[en[:, 1]]) * (ys[en[:, 0]] - ys[en[:, 1]])
                    - (ys[en[:, 2]] - ys[en[:, 1]]) * (xs[en[:, 0]] - xs[en[:, 1]]))
        qx = ((xs[en[:, 0]] + xs[en[:, 2]] + xs[en[:, 3]]) * s1 + (xs[en[:, 0]] + xs[en[:, 1]] + xs[en[:, 2]]) * s2) \
            / 3.0 / (s1 + s2)
        qy = ((ys[en[:, 0]] + ys[en[:, 2]] + ys[en[:, 3]]) * s1 + (ys[en[:, 0]] + ys[en[:, 1]] + ys[en[:, 2]]) * s2) \
            / 3.0 / (s1 + s2)
        cx = np.where(tri, p[en[:, :3], 0].mean(axis=1), qx)
        cy = np.where(tri, p[en[:, :3], 1].mean(axis=1), qy)
        u = 0.5 * cx + 0.25 * cy
        nb = m.elem_neighbors
        interior = (nb > 0).all(axis=1)
        for e in np.nonzero(interior)[0][::7]:
            q = 3 if tri[e] else 4
            du = u[nb[e, :q] - 1] - u[e]
            gux = (m.gradient_vec[e, :q] * du).sum()
            guy = (m.gradient_vec[e, 4:4 + q] * du).sum()
            assert abs(gux - 0.5) < 1e-9 and abs(guy - 0.25) < 1e-9, e
