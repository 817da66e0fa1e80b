"""One mesh over several GPUs: partition, sub-meshes with a deep halo, and
the halo exchange (the reference's domain decomposition: the METIS
partition of src/metis_wrapper.c and the halo exchange of
src/gen_halo_exchange_c.F90:130-165,663-793).

Partition.  The nodes are ordered along a Hilbert curve through their
coordinates and cut into nranks contiguous ranges of equal size; a node
belongs to the rank of its range, an element to the rank of its first node.

Sub-meshes.  A rank holds the elements within `halo` rings of what it owns
(ring 0: the elements that touch one of its nodes or are its own), their
nodes, and every edge of those elements, and runs the ordinary one-GPU
step on that sub-mesh.  Near the sub-mesh's rim the stencils are cut, so
values there are wrong, and the error moves inward by the step's
dependency radius in every internal step; with a halo deeper than that
radius the rank's own nodes and elements come out of the step exactly as
in the undecomposed run.  Copying the halo's state from its owners after
every internal step then restores the rim.  The reference exchanges after
each routine whose output a neighbour reads (exchange_nod / exchange_elem);
this form trades that for redundant work in the halo and one exchange per
internal step.

The sub-mesh arrays keep the global relative order of nodes, elements and
edges (internal edges, then the mesh's boundary edges, then the rim edges:
internal edges whose second element is outside the sub-mesh), so every
per-node sum over edges runs in the reference's edge order.

Reductions.  The tracer min / max of solve_tracers (src/fv_tracer.F90:18-27)
is taken over every rank's own nodes and given to each rank's model before
its step (fesomc_gpu_set_tracer_range); the energy diagnostic is summed
over the ranks' own nodes and elements on the host.

Transports.  `LocalRanks` runs all ranks in one process (one model each)
and exchanges the whole state through host arrays; `DeviceRanks` does the
same with the halos packed and unpacked on the device
(fesomc_gpu_halo_pack / _unpack); `DistRank` is one rank per process over
torch.distributed (the tracer range all-reduced, the packed halos sent
with isend / irecv: device buffers with NCCL, staged through host tensors
with gloo); `exchange_dist` is the host-array exchange over
torch.distributed.
"""
import ctypes as C

import numpy as np

from . import abi, cases, model

# state fields by entity and values per entity: n nodes, e elements,
# L levels, NS interfaces
STATE_KIND = {
    "eta_n": ("n", 1), "eta_n_1": ("n", 1), "eta_n_2": ("n", 1), "etaAB": ("n", 1), "ssh_gp": ("n", 1),
    "mask_wd_node": ("n", 1), "U_filt_2D": ("e", 1), "V_filt_2D": ("e", 1), "mask_wd": ("e", 1),
    "U_n_2D": ("e", 2), "U_n_1": ("e", 2), "U_n_2": ("e", 2), "Bar_pr_2D": ("e", 2),
    "U_n": ("e", "L"), "V_n": ("e", "L"), "U_rhsAB": ("e", "L"), "V_rhsAB": ("e", "L"),
    "U_n_filt": ("e", "L"), "V_n_filt": ("e", "L"),
    "TF": ("n", "L"), "SF": ("n", "L"), "T_old": ("n", "L"), "S_old": ("n", "L"), "Tclim": ("n", "L"),
    "Sclim": ("n", "L"), "rho_c": ("n", "L"),
    "bt": ("n", "NS"), "snu": ("n", "NS"), "Kv": ("n", "NS"), "Ri": ("n", "NS"), "tke_dissip": ("n", "NS"),
    "Wvel": ("n", "NS"), "hpressure": ("n", "NS"), "Av": ("e", "NS"),
}
# forcing arrays by what they are given per
FORCING_KIND = {
    "taux": ("e", 1), "tauy": ("e", 1), "windx": ("n", 1), "windy": ("n", 1), "mslp": ("n", 1),
    "emp": ("n", 1), "qsr": ("n", 1), "qns": ("n", 1), "Rj": ("n", 1), "aj": ("n", 1), "bj": ("n", 1),
    "Tclim": ("n", "L"), "Sclim": ("n", "L"), "runoff_rivers": ("river", 1), "ampt": ("obn", 12),
    "fazt": ("obn", 12), "amp_factor": ("all", 1), "phy_factor": ("all", 1),
}
BOUNDARY = -999   # edge_tri / elem_neighbors marker of a missing element
# halo rings: one internal step of the estuary configuration (10 sub-steps,
# MUSCL tracers, filter viscosity, wetting / drying) needs 12 for the owned
# entities to come out exact, 8 is not enough; the default keeps a margin
# for the options with wider stencils (biharmonic, filter-2x viscosities)
DEFAULT_HALO = 16


def _width(w, L, NS):
    return {"L": L, "NS": NS}.get(w, w)


def hilbert_keys(xy, order=16):
    """Position of every point along a Hilbert curve over the bounding square
    of xy (the classic xy -> d mapping: per level, the quadrant's offset
    along the curve, then the rotation / reflection into the quadrant)."""
    xy = np.asarray(xy, dtype=np.float64)
    lo = xy.min(axis=0)
    span = float((xy.max(axis=0) - lo).max()) or 1.0
    n = 1 << order
    q = np.minimum(((xy - lo) / span * (n - 1)).round().astype(np.int64), n - 1)
    x, y = q[:, 0].copy(), q[:, 1].copy()
    d = np.zeros(len(xy), dtype=np.int64)
    s = n >> 1
    while s > 0:
        rx = (x & s) > 0
        ry = (y & s) > 0
        d += s * s * ((3 * rx.astype(np.int64)) ^ ry.astype(np.int64))
        flip = ~ry & rx
        x = np.where(flip, n - 1 - x, x)
        y = np.where(flip, n - 1 - y, y)
        swap = ~ry
        x, y = np.where(swap, y, x), np.where(swap, x, y)
        s >>= 1
    return d


def partition(mesh, nranks):
    """Owner rank of every node (0-based array): equal contiguous ranges of
    the nodes' Hilbert order."""
    if nranks < 1 or nranks > mesh.N:
        raise ValueError("nranks must be in 1..%d" % mesh.N)
    order = np.argsort(hilbert_keys(mesh.coord_nod2D), kind="stable")
    owner = np.empty(mesh.N, dtype=np.int32)
    for r, chunk in enumerate(np.array_split(order, nranks)):
        owner[chunk] = r
    return owner


def _map(n, ids):
    m = np.full(n, -1, dtype=np.int64)
    m[ids] = np.arange(len(ids))
    return m


class SubMesh:
    """The fesomc_mesh of the nodes `nodes` and elements `elems` (global,
    0-based, ascending) of `mesh`, with every edge of those elements (see
    the module docstring for the edge order)."""

    def __init__(self, mesh, nodes, elems):
        self.nodes, self.elems = np.asarray(nodes), np.asarray(elems)
        nmap, emap = _map(mesh.N, self.nodes), _map(mesh.E, self.elems)
        self.NS, self.L = mesh.NS, mesh.L
        self.N, self.E = len(self.nodes), len(self.elems)
        en = mesh.elem2D_nodes[self.elems] - 1
        if (nmap[en] < 0).any():
            raise ValueError("an element's node is outside the sub-mesh")
        ee = mesh.elem_edges[self.elems]
        edges = np.unique(ee[ee > 0] - 1)
        et = mesh.edge_tri[edges]
        t0 = emap[et[:, 0] - 1]
        t1 = np.where(et[:, 1] > 0, emap[np.maximum(et[:, 1], 1) - 1], -1)
        glob_in = edges < mesh.Ed_in
        internal = glob_in & (t0 >= 0) & (t1 >= 0)
        rim = glob_in & ~internal
        order = np.concatenate([edges[internal], edges[~glob_in], edges[rim]])
        self.edges = order
        self.Ed, self.Ed_in = len(order), int(internal.sum())
        self.n_rim_edges = int(rim.sum())
        edmap = _map(mesh.Ed, order)

        def emap1(v):   # 1-based global elements -> 1-based local, missing -> marker
            v = np.asarray(v, dtype=np.int64)
            loc = np.where(v > 0, emap[np.maximum(v, 1) - 1], -1)
            return loc

        a = {}
        a["index_nod2D"] = mesh.index_nod2D[self.nodes]
        a["elem2D_nodes"] = (nmap[en] + 1).astype(np.int32)
        a["edge_nodes"] = (nmap[mesh.edge_nodes[order] - 1] + 1).astype(np.int32)
        tri = emap1(mesh.edge_tri[order])
        cross = mesh.edge_cross_dxdy[order].copy()
        # rim edges: the element inside the sub-mesh first, the other marked
        swap = (tri[:, 0] < 0) & (tri[:, 1] >= 0)
        tri[swap] = tri[swap][:, ::-1]
        cross[swap] = cross[swap][:, [2, 3, 0, 1]]
        a["edge_tri"] = np.where(tri >= 0, tri + 1, BOUNDARY).astype(np.int32)
        a["edge_cross_dxdy"] = cross
        a["edge_dxdy"] = mesh.edge_dxdy[order]
        a["elem_edges"] = (edmap[ee - 1] + 1).astype(np.int32)
        nb = emap1(mesh.elem_neighbors[self.elems])
        a["elem_neighbors"] = np.where(nb >= 0, nb + 1, BOUNDARY).astype(np.int32)
        # elements of each node, in the global order, those of the sub-mesh
        nie_g = mesh.nod_in_elem2D[self.nodes]
        loc = emap1(nie_g)
        wmax = nie_g.shape[1]
        keep = loc >= 0
        first = np.argsort(~keep, axis=1, kind="stable")      # kept entries first, in order
        nie = np.where(np.take_along_axis(keep, first, 1), np.take_along_axis(loc, first, 1) + 1, 0)
        a["nod_in_elem2D"] = nie.astype(np.int32)
        a["nod_in_elem2D_num"] = keep.sum(axis=1).astype(np.int32)
        self.wmax = wmax
        self.with_updn = bool(mesh.c.edge_up_dn_tri)
        if self.with_updn:
            ud = emap1(mesh.edge_up_dn_tri[order])
            a["edge_up_dn_tri"] = np.where(ud >= 0, ud + 1, 0).astype(np.int32)
        for name in ("coord_nod2D", "depth", "area", "ac"):
            a[name] = getattr(mesh, name)[self.nodes]
        for name in ("elem_area", "elem_cos", "coriolis", "w_cv", "gradient_sca", "gradient_vec"):
            a[name] = getattr(mesh, name)[self.elems]
        a["sigma"] = mesh.sigma
        a["a_tp"] = mesh.a_tp[:, self.nodes]
        obn = mesh.in_obn - 1 if mesh.c.nobn > 0 else np.zeros(0, dtype=np.int64)
        self.obn_sel = np.nonzero(nmap[obn] >= 0)[0]
        a["in_obn"] = (nmap[obn[self.obn_sel]] + 1).astype(np.int32)
        riv = mesh.nod_rivers - 1 if mesh.c.n_rivers > 0 else np.zeros(0, dtype=np.int64)
        self.river_sel = np.nonzero(nmap[riv] >= 0)[0]
        a["nod_rivers"] = (nmap[riv[self.river_sel]] + 1).astype(np.int32)
        self.nobn_global = int(mesh.c.nobn)
        self.scale_area = mesh.scale_area
        self._a = {k: np.ascontiguousarray(v) for k, v in a.items()}
        c = abi.Mesh()
        c.nod2D, c.elem2D, c.edge2D, c.edge2D_in, c.nsigma = self.N, self.E, self.Ed, self.Ed_in, self.NS
        c.nod_in_elem2D_max = wmax
        for name, _ in abi.Mesh._fields_:
            if name in self._a:
                v = self._a[name]
                setattr(c, name, abi.iptr(v) if v.dtype == np.int32 else abi.dptr(v))
        c.nobn, c.n_rivers = len(self._a["in_obn"]), len(self._a["nod_rivers"])
        if not self.with_updn:
            c.edge_up_dn_tri = None
        self.c = c

    def __getattr__(self, k):
        a = self.__dict__.get("_a")
        if a is not None and k in a:
            return a[k].copy()
        raise AttributeError(k)


def _take(arr, idx, width):
    return np.ascontiguousarray(np.asarray(arr).reshape(-1, width)[idx].reshape(-1))


class RankPart:
    """Rank r's share of a case: its sub-mesh and case, what it owns, and its
    halo (the entities it receives after every step, with their owners)."""

    def __init__(self, case, owner, rank, halo):
        mesh = case.mesh
        self.rank, self.halo = rank, halo
        en = mesh.elem2D_nodes - 1
        owner_e = owner[en[:, 0]]
        own_n = owner == rank
        local_e = own_n[en].any(axis=1) | (owner_e == rank)
        for _ in range(halo):
            nmask = np.zeros(mesh.N, dtype=bool)
            nmask[en[local_e]] = True
            local_e = nmask[en].any(axis=1)
        elems = np.nonzero(local_e)[0]
        nodes = np.unique(en[elems])
        self.mesh = SubMesh(mesh, nodes, elems)
        L, NS = mesh.L, mesh.NS
        self.own_nodes = owner[nodes] == rank            # local masks
        self.own_elems = owner_e[elems] == rank
        if not self.own_nodes.any() or not np.array_equal(np.nonzero(own_n)[0], nodes[self.own_nodes]):
            raise ValueError("rank %d: owned nodes outside its sub-mesh" % rank)
        self.node_owner, self.elem_owner = owner[nodes], owner_e[elems]
        p = type(case.params)()
        C.memmove(C.byref(p), C.byref(case.params), C.sizeof(p))
        p.scale_area = case.params.scale_area            # the whole mesh's
        sub = self.mesh
        state = {k: _take(v, nodes if STATE_KIND[k][0] == "n" else elems, _width(STATE_KIND[k][1], L, NS))
                 for k, v in case.state0.items()}

        def forcing(step, time_jd, _f=case.forcing_fn):
            g = _f(step, time_jd)
            out = {}
            for k, v in g.items():
                kind, w = FORCING_KIND[k]
                v = np.asarray(v, dtype=np.float64)
                if kind == "n":
                    out[k] = _take(v, nodes, _width(w, L, NS))
                elif kind == "e":
                    out[k] = _take(v, elems, _width(w, L, NS))
                elif kind == "river":
                    out[k] = np.ascontiguousarray(v[sub.river_sel])
                elif kind == "obn":       # 12 columns of nobn (Fortran (nobn, 12))
                    out[k] = np.ascontiguousarray(v.reshape(12, sub.nobn_global)[:, sub.obn_sel].reshape(-1))
                else:
                    out[k] = v
            return out

        self.case = cases.Case("%s.rank%d" % (case.name, rank), sub, p, state, forcing, meta=dict(case.meta))
        self.nodes, self.elems = nodes, elems


class Decomposition:
    """The partition of `case` over nranks with the given halo depth, the
    ranks' parts, and the exchange lists between every pair of ranks: for
    rank r and peer q, recv[r][q] = (local nodes, local elements) of r owned
    by q, and send[q][r] = the same entities as local indices of q (both in
    ascending global order)."""

    def __init__(self, case, nranks, halo=DEFAULT_HALO):
        self.case, self.nranks, self.halo = case, nranks, halo
        self.owner = partition(case.mesh, nranks)
        self.parts = [RankPart(case, self.owner, r, halo) for r in range(nranks)]
        mesh = case.mesh
        nmaps = [_map(mesh.N, p.nodes) for p in self.parts]
        emaps = [_map(mesh.E, p.elems) for p in self.parts]
        self.recv = [[None] * nranks for _ in range(nranks)]
        self.send = [[None] * nranks for _ in range(nranks)]
        for r, p in enumerate(self.parts):
            for q in range(nranks):
                if q == r:
                    continue
                rn = np.nonzero(p.node_owner == q)[0]
                re = np.nonzero(p.elem_owner == q)[0]
                gn, ge = p.nodes[rn], p.elems[re]
                sn, se = nmaps[q][gn], emaps[q][ge]
                if (sn < 0).any() or (se < 0).any():
                    raise ValueError("rank %d holds entities its owner %d lacks" % (r, q))
                self.recv[r][q] = (rn, re)
                self.send[q][r] = (sn, se)

    def halo_sizes(self):
        return [(int((~p.own_nodes).sum()), int((~p.own_elems).sum())) for p in self.parts]

    def count(self, r, q, fields):
        """Values rank r sends to peer q for `fields`."""
        sn, se = self.send[r][q]
        L, NS = self.case.mesh.L, self.case.mesh.NS
        return sum(len(sn if STATE_KIND[k][0] == "n" else se) * _width(STATE_KIND[k][1], L, NS)
                   for k in STATE_KIND if k in fields)

    def pack(self, r, q, state):
        """Rank r's values for peer q, one flat array (fields in STATE_KIND
        order)."""
        sn, se = self.send[r][q]
        L, NS = self.case.mesh.L, self.case.mesh.NS
        out = []
        for k, (ent, w) in STATE_KIND.items():
            if k in state:
                out.append(_take(state[k], sn if ent == "n" else se, _width(w, L, NS)))
        return np.concatenate(out) if out else np.zeros(0)

    def unpack(self, r, q, state, buf):
        """Write peer q's values (pack(q, r, ...)) into rank r's halo."""
        rn, re = self.recv[r][q]
        L, NS = self.case.mesh.L, self.case.mesh.NS
        off = 0
        for k, (ent, w) in STATE_KIND.items():
            if k not in state:
                continue
            w = _width(w, L, NS)
            idx = rn if ent == "n" else re
            n = len(idx) * w
            state[k].reshape(-1, w)[idx] = buf[off:off + n].reshape(-1, w)
            off += n
        if off != len(buf):
            raise ValueError("exchange buffer of %d values, expected %d" % (len(buf), off))

    def own_range(self, r, state):
        """(Tmin, Tmax, Smin, Smax) over rank r's own nodes."""
        p = self.parts[r]
        L = self.case.mesh.L
        t = state["TF"].reshape(-1, L)[p.own_nodes]
        s = state["SF"].reshape(-1, L)[p.own_nodes]
        return np.array([t.min(), t.max(), s.min(), s.max()])

    def assemble(self, states):
        """The whole mesh's state from the ranks' own entities."""
        mesh = self.case.mesh
        L, NS = mesh.L, mesh.NS
        out = {}
        for k, (ent, w) in STATE_KIND.items():
            if k not in states[0]:
                continue
            w = _width(w, L, NS)
            n = mesh.N if ent == "n" else mesh.E
            a = np.full((n, w), np.nan)
            for p, st in zip(self.parts, states):
                own = p.own_nodes if ent == "n" else p.own_elems
                ids = p.nodes if ent == "n" else p.elems
                a[ids[own]] = st[k].reshape(-1, w)[own]
            out[k] = a.reshape(-1)
        return out


def combine_ranges(ranges):
    r = np.asarray(ranges)
    return np.array([r[:, 0].min(), r[:, 1].max(), r[:, 2].min(), r[:, 3].max()])


class LocalRanks:
    """All ranks of a decomposition in this process, one model each (on the
    current device, or on devices[r]), stepped together: before every step
    the tracer range over all ranks' own nodes goes to every model, after it
    the halos are refreshed from their owners through host arrays."""

    def __init__(self, decomp, devices=None):
        self.dec = decomp
        self.models = []
        lib = abi.load()
        for r, p in enumerate(decomp.parts):
            if devices is not None:
                abi.check(lib.fesomc_gpu_set_device(int(devices[r])), "fesomc_gpu_set_device")
            self.models.append(model.GpuModel(p.case))
        self.states = [g.state() for g in self.models]

    def step(self, nsteps=1):
        dec = self.dec
        for _ in range(nsteps):
            rng = combine_ranges([dec.own_range(r, st) for r, st in enumerate(self.states)])
            arr = np.ascontiguousarray(rng, dtype=np.float64)
            for g in self.models:
                abi.check(g.lib.fesomc_gpu_set_tracer_range(g.h, abi.dptr(arr)), "fesomc_gpu_set_tracer_range")
                g.step(1)
            self.states = [g.state() for g in self.models]
            bufs = {(r, q): dec.pack(r, q, self.states[r]) for r in range(dec.nranks)
                    for q in range(dec.nranks) if q != r}
            for r in range(dec.nranks):
                for q in range(dec.nranks):
                    if q != r:
                        dec.unpack(r, q, self.states[r], bufs[(q, r)])
            for g, st in zip(self.models, self.states):
                arrays = {k: v for k, v in st.items() if k != "_time_jd"}
                s = g.case.state_struct(arrays, g.time_jd, lfirst=0)
                abi.check(g.lib.fesomc_gpu_sync_from_host(g.h, abi.F_ALL, C.byref(s)), "fesomc_gpu_sync_from_host")

    def assemble(self):
        return self.dec.assemble(self.states)

    def close(self):
        for g in self.models:
            g.close()
        self.models = []


def _plan(g, nodes, elems):
    n = np.ascontiguousarray(nodes, dtype=np.int32)
    e = np.ascontiguousarray(elems, dtype=np.int32)
    h = C.c_void_p()
    abi.check(g.lib.fesomc_gpu_halo_plan(g.h, len(n), abi.iptr(n), len(e), abi.iptr(e), C.byref(h)),
              "fesomc_gpu_halo_plan")
    c = C.c_int64()
    abi.check(g.lib.fesomc_gpu_halo_size(h, C.byref(c)), "fesomc_gpu_halo_size")
    return h, int(c.value)


class RankPlans:
    """Device halo plans of rank r's model g: for every peer q the entities
    it sends (send[q]) and receives (recv[q]), as (plan, doubles), and its
    own nodes (own), whose tracer range it contributes."""

    def __init__(self, dec, r, g):
        self.g, self.send, self.recv = g, {}, {}
        for q in range(dec.nranks):
            if q != r:
                self.send[q] = _plan(g, *dec.send[r][q])
                self.recv[q] = _plan(g, *dec.recv[r][q])
        self.own = _plan(g, np.nonzero(dec.parts[r].own_nodes)[0], np.zeros(0, dtype=np.int32))

    def range(self):
        out = np.zeros(4)
        abi.check(self.g.lib.fesomc_gpu_halo_range(self.g.h, self.own[0], abi.dptr(out)), "fesomc_gpu_halo_range")
        return out

    def pack(self, q, ptr):
        abi.check(self.g.lib.fesomc_gpu_halo_pack(self.g.h, self.send[q][0], C.c_void_p(ptr)), "fesomc_gpu_halo_pack")

    def unpack(self, q, ptr):
        abi.check(self.g.lib.fesomc_gpu_halo_unpack(self.g.h, self.recv[q][0], C.c_void_p(ptr)),
                  "fesomc_gpu_halo_unpack")

    def close(self):
        for h, _ in list(self.send.values()) + list(self.recv.values()) + [self.own]:
            self.g.lib.fesomc_gpu_halo_free(h)
        self.send, self.recv = {}, {}


def _set_range(g, rng):
    arr = np.ascontiguousarray(rng, dtype=np.float64)
    abi.check(g.lib.fesomc_gpu_set_tracer_range(g.h, abi.dptr(arr)), "fesomc_gpu_set_tracer_range")


class DeviceRanks:
    """All ranks in this process on the current GPU, the halos packed and
    unpacked on the device (fesomc_gpu_halo_*) through device buffers, the
    tracer range combined from the ranks' own nodes."""

    def __init__(self, decomp):
        import torch
        self.dec = decomp
        self.models = [model.GpuModel(p.case) for p in decomp.parts]
        self.plans = [RankPlans(decomp, r, g) for r, g in enumerate(self.models)]
        n = max([c for pl in self.plans for _, c in pl.send.values()] + [1])
        self.buf = torch.empty(n, dtype=torch.float64, device="cuda")

    def step(self, nsteps=1):
        dec = self.dec
        for _ in range(nsteps):
            rng = combine_ranges([pl.range() for pl in self.plans])
            for g in self.models:
                _set_range(g, rng)
                g.step(1)
            for r in range(dec.nranks):
                for q in range(dec.nranks):
                    if q != r:
                        self.plans[r].pack(q, self.buf.data_ptr())
                        self.plans[q].unpack(r, self.buf.data_ptr())

    def assemble(self):
        return self.dec.assemble([g.state() for g in self.models])

    def close(self):
        for pl in self.plans:
            pl.close()
        for g in self.models:
            g.close()
        self.models, self.plans = [], []


class DistRank:
    """This process's rank of a decomposition over torch.distributed (`dist`,
    initialised; world size = ranks): its model on the current GPU, the
    tracer range all-reduced, the packed halos exchanged with isend / irecv
    after every step (device buffers with NCCL; staged through host tensors
    with gloo).  Every rank builds the same decomposition."""

    def __init__(self, case, dist, halo=DEFAULT_HALO):
        import torch
        self.dist = dist
        self.rank, world = dist.get_rank(), dist.get_world_size()
        self.dec = Decomposition(case, world, halo)
        self.g = model.GpuModel(self.dec.parts[self.rank].case)
        self.plans = RankPlans(self.dec, self.rank, self.g)
        self.nccl = dist.get_backend() == "nccl"
        dev = "cuda" if self.nccl else "cpu"
        self.sbuf = {q: torch.empty(c, dtype=torch.float64, device="cuda") for q, (_, c) in self.plans.send.items()}
        self.rbuf = {q: torch.empty(c, dtype=torch.float64, device="cuda") for q, (_, c) in self.plans.recv.items()}
        self.shost = {q: torch.empty(c, dtype=torch.float64, device=dev) for q, (_, c) in self.plans.send.items()}
        self.rhost = {q: torch.empty(c, dtype=torch.float64, device=dev) for q, (_, c) in self.plans.recv.items()}

    def step(self, nsteps=1):
        import torch
        dist = self.dist
        dev = "cuda" if self.nccl else "cpu"
        for _ in range(nsteps):
            r = self.plans.range()
            lo = torch.tensor([r[0], r[2]], dtype=torch.float64, device=dev)
            hi = torch.tensor([r[1], r[3]], dtype=torch.float64, device=dev)
            dist.all_reduce(lo, op=dist.ReduceOp.MIN)
            dist.all_reduce(hi, op=dist.ReduceOp.MAX)
            _set_range(self.g, [lo[0].item(), hi[0].item(), lo[1].item(), hi[1].item()])
            self.g.step(1)
            for q in self.sbuf:
                self.plans.pack(q, self.sbuf[q].data_ptr())
                if not self.nccl:
                    self.shost[q].copy_(self.sbuf[q])
            src = self.sbuf if self.nccl else self.shost
            dst = self.rbuf if self.nccl else self.rhost
            if self.nccl:   # one group: the sends and receives of every peer together
                ops = [dist.P2POp(dist.isend, src[q], q) for q in sorted(src)]
                ops += [dist.P2POp(dist.irecv, dst[q], q) for q in sorted(dst)]
                reqs = dist.batch_isend_irecv(ops) if ops else []
            else:
                reqs = [dist.isend(src[q], q) for q in sorted(src)] + [dist.irecv(dst[q], q) for q in sorted(dst)]
            for rq in reqs:
                rq.wait()
            if self.nccl:
                torch.cuda.synchronize()
            for q in self.rbuf:
                if not self.nccl:
                    self.rbuf[q].copy_(self.rhost[q])
                    torch.cuda.synchronize()
                self.plans.unpack(q, self.rbuf[q].data_ptr())

    def own_state(self):
        """This rank's state (its sub-mesh) for assembling on one rank."""
        return self.g.state()

    def close(self):
        self.plans.close()
        self.g.close()


def exchange_dist(decomp, rank, state, dist):
    """The halo exchange of rank `rank` with every peer over
    torch.distributed (`dist`, initialised, world size = nranks): sends
    what each peer holds of this rank's entities, receives its own halo.
    Every rank posts all its sends and receives, then waits for them."""
    import torch
    reqs, recv = [], {}
    for q in range(decomp.nranks):
        if q == rank:
            continue
        out = torch.from_numpy(decomp.pack(rank, q, state))
        inp = torch.empty(decomp.count(q, rank, state), dtype=torch.float64)
        recv[q] = inp
        reqs.append(dist.isend(out, q))
        reqs.append(dist.irecv(inp, q))
    for rq in reqs:
        rq.wait()
    for q, buf in recv.items():
        decomp.unpack(rank, q, state, buf.numpy())


def range_dist(decomp, rank, state, dist):
    """The tracer range over all ranks' own nodes (all-reduce of min / max)."""
    import torch
    r = decomp.own_range(rank, state)
    lo = torch.tensor([r[0], r[2]], dtype=torch.float64)
    hi = torch.tensor([r[1], r[3]], dtype=torch.float64)
    dist.all_reduce(lo, op=dist.ReduceOp.MIN)
    dist.all_reduce(hi, op=dist.ReduceOp.MAX)
    return np.array([lo[0].item(), hi[0].item(), lo[1].item(), hi[1].item()])
