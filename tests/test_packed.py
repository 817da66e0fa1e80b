"""Packed members on the host: the packed mesh maps back to every member's
own arrays, the state and forcing split and concatenate member by member,
and fesomc_gpu_init_packed refuses member tables that do not describe
disjoint members (before any CUDA call, so this runs without a GPU)."""
import ctypes as C

import numpy as np
import pytest

NODES = (1200, 3000)


def _members(n=3, nsigma=None):
    from fesomc import cases
    out, i = [], 0
    while len(out) < n:
        c = cases.ensemble_member(i, nodes_range=NODES)
        i += 1
        if nsigma is None:
            nsigma = c.mesh.NS
        if c.mesh.NS == nsigma:
            out.append(c)
    return out


@pytest.fixture(scope="module")
def pack(built):
    from fesomc import packed
    members = _members()
    return members, packed.PackedCase(members)


def test_packed_mesh_maps_back_to_members(pack):
    members, pc = pack
    pm = pc.mesh
    assert pm.N == sum(m.mesh.N for m in members) and pm.E == sum(m.mesh.E for m in members)
    assert pm.Ed_in == sum(m.mesh.Ed_in for m in members)
    # every internal edge before every boundary edge
    et = pm.edge_tri
    assert np.all(et[:pm.Ed_in, 1] > 0) and np.all(et[pm.Ed_in:, 1] <= 0)
    for k, m in enumerate(members):
        no, eo, rows = pm.node_off[k], pm.elem_off[k], pm.edge_rows[k]
        # each member's edges keep their relative order (internal, boundary)
        assert np.all(np.diff(rows[:m.mesh.Ed_in]) == 1) and np.all(np.diff(rows[m.mesh.Ed_in:]) == 1)
        assert np.array_equal(pm.edge_nodes[rows], m.mesh.edge_nodes + no)
        tri = m.mesh.edge_tri
        assert np.array_equal(pm.edge_tri[rows], np.where(tri > 0, tri + eo, tri))
        assert np.array_equal(pm.elem2D_nodes[eo:pm.elem_off[k + 1]], m.mesh.elem2D_nodes + no)
        ee = m.mesh.elem_edges
        assert np.array_equal(pm.elem_edges[eo:pm.elem_off[k + 1]], np.where(ee > 0, rows[np.maximum(ee, 1) - 1] + 1, ee))
        nb = m.mesh.elem_neighbors
        assert np.array_equal(pm.elem_neighbors[eo:pm.elem_off[k + 1]], np.where(nb > 0, nb + eo, nb))
        for f in ("w_cv", "gradient_sca", "elem_area", "coriolis"):
            assert np.array_equal(getattr(pm, f)[eo:pm.elem_off[k + 1]], getattr(m.mesh, f))
        for f in ("edge_dxdy", "edge_cross_dxdy", "edge_up_dn_tri"):
            got, ref = getattr(pm, f)[rows], getattr(m.mesh, f)
            if f == "edge_up_dn_tri":
                ref = np.where(ref > 0, ref + eo, ref)
            assert np.array_equal(got, ref), f
        assert np.array_equal(pm.a_tp[:, no:pm.node_off[k + 1]], m.mesh.a_tp)
        num = m.mesh.nod_in_elem2D_num
        nie = pm.nod_in_elem2D[no:pm.node_off[k + 1]]
        for i in range(m.mesh.N):
            assert np.array_equal(nie[i, :num[i]], m.mesh.nod_in_elem2D[i, :num[i]] + eo)
    assert np.array_equal(pm.scale_area, [m.mesh.scale_area for m in members])


def test_state_and_forcing_split_by_member(pack):
    members, pc = pack
    parts = pc.split_state(pc.state0)
    for k, m in enumerate(members):
        for name, v in m.state0.items():
            assert np.array_equal(parts[k][name], v), name
    t = pc.params.time_jd0 + 0.25
    f = pc.forcing_fn(3, t)
    refs = [m.forcing_fn(3, t) for m in members]
    assert np.array_equal(f["taux"], np.concatenate([r["taux"] for r in refs]))
    assert np.array_equal(f["amp_factor"], refs[0]["amp_factor"])
    # (nobn, 12) column-major: 12 columns, each the members' OB nodes in turn
    got = f["ampt"].reshape(12, -1)
    off = 0
    for r, m in zip(refs, members):
        nb = m.mesh.c.nobn
        assert np.array_equal(got[:, off:off + nb], r["ampt"].reshape(12, nb))
        off += nb


def test_packing_refuses_mixed_level_counts(built):
    from fesomc import cases, packed
    a = _members(1)[0]
    other = 21 if a.mesh.NS == 11 else 11
    b = _members(1, nsigma=other)[0]
    with pytest.raises(ValueError):
        packed.PackedCase([a, b])


def _init_packed(lib, pc, node_off, elem_off, scale_area):
    from fesomc import abi
    arrays = pc.new_state_arrays()
    st = pc.state_struct(arrays, pc.params.time_jd0)
    no = np.ascontiguousarray(node_off, dtype=np.int32)
    eo = np.ascontiguousarray(elem_off, dtype=np.int32)
    sa = np.ascontiguousarray(scale_area, dtype=np.float64)
    mb = abi.Members()
    mb.n, mb.node_off, mb.elem_off, mb.scale_area = len(sa), abi.iptr(no), abi.iptr(eo), abi.dptr(sa)
    h = C.c_void_p()
    rc = lib.fesomc_gpu_init_packed(C.byref(pc.mesh.c), C.byref(pc.params), C.byref(st), C.byref(mb), C.byref(h))
    if h.value:
        lib.fesomc_gpu_finalize(h)
    return rc


def test_init_packed_refuses_bad_member_tables(pack):
    from fesomc import abi
    lib = abi.load()
    members, pc = pack
    no, eo, sa = pc.mesh.node_off.copy(), pc.mesh.elem_off.copy(), pc.mesh.scale_area.copy()
    EINVAL = 1
    bad = []
    x = no.copy(); x[-1] -= 1; bad.append((x, eo, sa))            # does not end at nod2D
    x = eo.copy(); x[0] = 1; bad.append((no, x, sa))              # does not start at 0
    x = no.copy(); x[1] = x[2]; bad.append((x, eo, sa))           # empty member
    x = no.copy(); x[1] += 1; bad.append((x, eo, sa))             # an element reaches the next member
    x = eo.copy(); x[1] -= 1; bad.append((no, x, sa))             # an element with another member's nodes
    y = sa.copy(); y[1] = 0.0; bad.append((no, eo, y))            # scale_area not positive
    for case in bad:
        assert _init_packed(lib, pc, *case) == EINVAL
    # the true table passes validation (no GPU here: a CUDA error, not EINVAL)
    assert _init_packed(lib, pc, no, eo, sa) != EINVAL
