"""Mesh decomposition, host side (no GPU): the Hilbert partition, the
sub-meshes and their edge order, and the halo exchange between two
processes over torch.distributed (gloo), checked against the owners'
values."""
import os

import numpy as np
import pytest


@pytest.fixture(scope="module")
def case(built):
    from fesomc import cases
    return cases.estuary_case("decomp", 60, 24, 300.0, 11, 2.0, 25.0, stress=(0.0, 0.05))


def test_partition_is_balanced_and_compact(case):
    from fesomc import decomp
    mesh = case.mesh
    for nr in (1, 2, 3, 4):
        own = decomp.partition(mesh, nr)
        counts = np.bincount(own, minlength=nr)
        assert counts.sum() == mesh.N and counts.max() - counts.min() <= 1
    # a Hilbert range is compact: the 2-way cut crosses few elements
    own = decomp.partition(mesh, 2)
    en = mesh.elem2D_nodes - 1
    cut = (own[en].min(axis=1) != own[en].max(axis=1)).sum()
    assert cut < 0.1 * mesh.E


def test_hilbert_keys_visit_neighbours_in_turn():
    from fesomc import decomp
    n = 16
    g = np.stack(np.meshgrid(np.arange(n), np.arange(n), indexing="ij"), -1).reshape(-1, 2).astype(float)
    k = decomp.hilbert_keys(g, order=4)
    assert sorted(k.tolist()) == list(range(n * n))
    path = g[np.argsort(k)]
    assert np.all(np.abs(np.diff(path, axis=0)).sum(axis=1) == 1)   # unit steps


@pytest.mark.parametrize("halo", [0, 3])
def test_sub_meshes_keep_the_global_order(case, halo):
    from fesomc import decomp
    mesh = case.mesh
    d = decomp.Decomposition(case, 2, halo)
    for p in d.parts:
        s = p.mesh
        assert np.all(np.diff(p.nodes) > 0) and np.all(np.diff(p.elems) > 0)
        ein = s.edges[:s.Ed_in]
        ebd = s.edges[s.Ed_in:s.Ed - s.n_rim_edges]
        assert np.all(np.diff(ein) > 0) and np.all(ein < mesh.Ed_in)
        assert np.all(np.diff(ebd) > 0) and np.all(ebd >= mesh.Ed_in)
        # the sub-mesh's elements are the global ones, renumbered
        en = s.elem2D_nodes - 1
        assert np.array_equal(p.nodes[en] + 1, mesh.elem2D_nodes[p.elems])
        # edges of an owned node whose elements are all in the sub-mesh: the
        # same edges, in the same order, as in the whole mesh
        gen = mesh.edge_nodes - 1
        sen = s.edge_nodes - 1
        for li in np.nonzero(p.own_nodes)[0][:50]:
            g = p.nodes[li]
            ge = np.nonzero((gen == g).any(axis=1))[0]
            se = s.edges[np.nonzero((sen == li).any(axis=1))[0]]
            if np.isin(mesh.edge_tri[ge][mesh.edge_tri[ge] > 0] - 1, p.elems).all():
                assert np.array_equal(np.sort(se), ge)
        assert s.c.nobn == len(s.in_obn) and s.c.n_rivers == len(s.nod_rivers)


def test_state_and_forcing_follow_the_sub_mesh(case):
    from fesomc import decomp
    d = decomp.Decomposition(case, 2, 2)
    L = case.mesh.L
    for p in d.parts:
        st = p.case.state0
        assert np.array_equal(st["TF"].reshape(-1, L), case.state0["TF"].reshape(-1, L)[p.nodes])
        assert np.array_equal(st["U_n_2D"].reshape(-1, 2), case.state0["U_n_2D"].reshape(-1, 2)[p.elems])
        f = p.case.forcing_fn(1, case.params.time_jd0 + 1.0)
        g = case.forcing_fn(1, case.params.time_jd0 + 1.0)
        assert np.array_equal(f["taux"], g["taux"][p.elems])
        assert len(f["runoff_rivers"]) == p.mesh.c.n_rivers
        assert np.array_equal(f["runoff_rivers"], g["runoff_rivers"][p.mesh.river_sel])
        nob = case.mesh.c.nobn
        assert np.array_equal(f["ampt"].reshape(12, -1), g["ampt"].reshape(12, nob)[:, p.mesh.obn_sel])
    assert abs(sum(p.mesh.c.n_rivers for p in d.parts) - case.mesh.c.n_rivers) <= case.mesh.c.n_rivers


def _labelled(d, r):
    """Rank r's state with every owned value set from its global index and
    every halo value NaN."""
    mesh, p = d.case.mesh, d.parts[r]
    L, NS = mesh.L, mesh.NS
    out = {}
    from fesomc.decomp import STATE_KIND
    for f, (k, (ent, w)) in enumerate(STATE_KIND.items()):
        w = {"L": L, "NS": NS}.get(w, w)
        ids = p.nodes if ent == "n" else p.elems
        own = p.own_nodes if ent == "n" else p.own_elems
        a = (ids[:, None] * 1000.0 + np.arange(w)[None, :] + f * 1e7).astype(np.float64)
        a[~own] = np.nan
        out[k] = np.ascontiguousarray(a.reshape(-1))
    return out


def test_host_exchange_fills_every_halo(case):
    from fesomc import decomp
    d = decomp.Decomposition(case, 3, 2)
    states = [_labelled(d, r) for r in range(3)]
    bufs = {(r, q): d.pack(r, q, states[r]) for r in range(3) for q in range(3) if q != r}
    for r in range(3):
        for q in range(3):
            if q != r:
                d.unpack(r, q, states[r], bufs[(q, r)])
    for r in range(3):
        p = d.parts[r]
        for k, v in states[r].items():
            assert not np.isnan(v).any(), (r, k)
        ent_ids = p.nodes
        L = case.mesh.L
        t = states[r]["TF"].reshape(-1, L)
        f_tf = list(decomp.STATE_KIND).index("TF")
        assert np.array_equal(t[:, 0], ent_ids * 1000.0 + f_tf * 1e7)


def _dist_rank(rank, world, port, path):
    import torch.distributed as dist
    from fesomc import cases, decomp
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        c = cases.estuary_case("decomp", 60, 24, 300.0, 11, 2.0, 25.0, stress=(0.0, 0.05))
        d = decomp.Decomposition(c, world, 2)
        st = _labelled(d, rank)
        decomp.exchange_dist(d, rank, st, dist)
        rng = decomp.range_dist(d, rank, {"TF": np.nan_to_num(st["TF"]), "SF": np.nan_to_num(st["SF"])}, dist)
        np.savez(os.path.join(path, "r%d.npz" % rank), rng=rng, **st)
    finally:
        dist.destroy_process_group()


def test_exchange_over_gloo_matches_the_host_exchange(case, tmp_path):
    import socket
    import torch.multiprocessing as mp
    from fesomc import decomp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    mp.start_processes(_dist_rank, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    d = decomp.Decomposition(case, 2, 2)
    states = [_labelled(d, r) for r in range(2)]
    for r in range(2):
        d.unpack(r, 1 - r, states[r], d.pack(1 - r, r, states[1 - r]))
    ranges = []
    for r in range(2):
        got = np.load(tmp_path / ("r%d.npz" % r))
        for k, v in states[r].items():
            assert np.array_equal(got[k], v), (r, k)
        ranges.append(got["rng"])
    assert np.array_equal(ranges[0], ranges[1])
    own = [d.own_range(r, states[r]) for r in range(2)]
    assert np.array_equal(ranges[0], decomp.combine_ranges(own))
