"""Packed members: several meshes of the same level count advanced as one
model (fesomc_gpu_init_packed), so that every kernel of a step covers all
members in one launch and one captured graph drives them all.

PackedMesh concatenates the members' fesomc_mesh arrays with their indices
offset: nodes and elements member after member, all members' internal edges
first and then all boundary edges (the kernels tell the two apart by edge
index), each member's edges keeping their own order, so every per-node sum
still runs in the member's own edge order.  PackedCase does the same for the
initial state and the forcing and splits results back per member.  Each
member advances bit for bit as it does alone; the library takes the tracer
means and scale_area per member.

The reference runs one mesh per executable; there is no counterpart.
"""
import ctypes as C

import numpy as np

from . import abi, cases

# fesomc_params fields that may differ between packed members (given per
# member in fesomc_members instead)
PER_MEMBER_PARAMS = ("scale_area",)
# forcing arrays shared by all members (the tidal nodal factors of the time)
GLOBAL_FORCING = ("amp_factor", "phy_factor")
# forcing arrays laid out (nobn, 12) in Fortran order: 12 columns of nobn
OB_FORCING = ("ampt", "fazt")


def _offset_pos(a, off):
    """a + off where a > 0 (1-based indices; boundary markers <= 0 kept)."""
    a = np.asarray(a, dtype=np.int32)
    return np.where(a > 0, a + off, a).astype(np.int32)


class PackedMesh:
    """The members' meshes as one fesomc_mesh (see the module docstring)."""

    def __init__(self, meshes):
        if not meshes:
            raise ValueError("no members")
        ns = {m.NS for m in meshes}
        if len(ns) != 1:
            raise ValueError("packed members need one level count, got %s" % sorted(ns))
        sig0 = meshes[0].sigma
        for m in meshes[1:]:
            if not np.array_equal(m.sigma, sig0):
                raise ValueError("packed members need the same sigma levels")
        self.members = list(meshes)
        n = len(meshes)
        self.NS = meshes[0].NS
        self.L = self.NS - 1
        Ns = np.array([m.N for m in meshes]); Es = np.array([m.E for m in meshes])
        Eds = np.array([m.Ed for m in meshes]); Eins = np.array([m.Ed_in for m in meshes])
        self.node_off = np.concatenate([[0], np.cumsum(Ns)]).astype(np.int32)
        self.elem_off = np.concatenate([[0], np.cumsum(Es)]).astype(np.int32)
        self.N, self.E = int(Ns.sum()), int(Es.sum())
        self.Ed, self.Ed_in = int(Eds.sum()), int(Eins.sum())
        in_off = np.concatenate([[0], np.cumsum(Eins)])
        bd_off = self.Ed_in + np.concatenate([[0], np.cumsum(Eds - Eins)])
        # packed row of every member edge (0-based)
        self.edge_rows = []
        for k, m in enumerate(meshes):
            j = np.arange(m.Ed)
            self.edge_rows.append(np.where(j < m.Ed_in, in_off[k] + j, bd_off[k] + (j - m.Ed_in)))
        self.scale_area = np.array([m.scale_area for m in meshes], dtype=np.float64)

        def cat(name):
            return np.ascontiguousarray(np.concatenate([getattr(m, name) for m in meshes]))

        def edges(name, width, dtype, fn=None):
            out = np.zeros((self.Ed, width), dtype=dtype)
            for k, m in enumerate(meshes):
                v = getattr(m, name)
                out[self.edge_rows[k]] = fn(k, v) if fn else v
            return out

        def edge_map(k, v):   # 1-based member edge numbers -> packed ones
            v = np.asarray(v, dtype=np.int64)
            return np.where(v > 0, self.edge_rows[k][np.maximum(v, 1) - 1] + 1, v).astype(np.int32)

        no, eo = self.node_off, self.elem_off
        a = {}
        a["index_nod2D"] = cat("index_nod2D")
        a["elem2D_nodes"] = np.concatenate([m.elem2D_nodes + no[k] for k, m in enumerate(meshes)]).astype(np.int32)
        a["edge_nodes"] = edges("edge_nodes", 2, np.int32, lambda k, v: v + no[k])
        a["edge_tri"] = edges("edge_tri", 2, np.int32, lambda k, v: _offset_pos(v, eo[k]))
        a["elem_edges"] = np.concatenate([edge_map(k, m.elem_edges) for k, m in enumerate(meshes)])
        a["elem_neighbors"] = np.concatenate([_offset_pos(m.elem_neighbors, eo[k]) for k, m in enumerate(meshes)])
        a["nod_in_elem2D_num"] = cat("nod_in_elem2D_num")
        wmax = max(m.c.nod_in_elem2D_max for m in meshes)
        nie = np.zeros((self.N, wmax), dtype=np.int32)
        for k, m in enumerate(meshes):
            v = m.nod_in_elem2D
            nie[no[k]:no[k + 1], :v.shape[1]] = _offset_pos(v, eo[k])
        a["nod_in_elem2D"] = nie
        with_updn = all(m.c.edge_up_dn_tri for m in meshes)
        if with_updn:
            a["edge_up_dn_tri"] = edges("edge_up_dn_tri", 2, np.int32, lambda k, v: _offset_pos(v, eo[k]))
        for name in ("coord_nod2D", "depth", "area", "elem_area", "elem_cos", "coriolis", "w_cv",
                     "gradient_sca", "gradient_vec", "ac"):
            a[name] = cat(name)
        a["edge_dxdy"] = edges("edge_dxdy", 2, np.float64)
        a["edge_cross_dxdy"] = edges("edge_cross_dxdy", 4, np.float64)
        a["sigma"] = np.ascontiguousarray(sig0)
        a["a_tp"] = np.ascontiguousarray(np.concatenate([m.a_tp for m in meshes], axis=1))
        obn = [m.in_obn for m in meshes if m.c.nobn > 0]
        a["in_obn"] = np.concatenate([m.in_obn + no[k] for k, m in enumerate(meshes) if m.c.nobn > 0]) \
            if obn else np.zeros(0, dtype=np.int32)
        riv = [m for m in meshes if m.c.n_rivers > 0]
        a["nod_rivers"] = np.concatenate([m.nod_rivers + no[k] for k, m in enumerate(meshes) if m.c.n_rivers > 0]) \
            if riv else np.zeros(0, dtype=np.int32)
        self.nobn = [m.c.nobn for m in meshes]
        self.n_rivers = [m.c.n_rivers for m in meshes]
        self._a = {k: np.ascontiguousarray(v) for k, v in a.items()}
        c = abi.Mesh()
        c.nod2D, c.elem2D, c.edge2D, c.edge2D_in, c.nsigma = self.N, self.E, self.Ed, self.Ed_in, self.NS
        c.nod_in_elem2D_max = wmax
        for name, _ in abi.Mesh._fields_:
            if name in self._a:
                v = self._a[name]
                setattr(c, name, abi.iptr(v) if v.dtype == np.int32 else abi.dptr(v))
        c.nobn, c.n_rivers = len(self._a["in_obn"]), len(self._a["nod_rivers"])
        if not with_updn:
            c.edge_up_dn_tri = None
        self.c = c

    def __getattr__(self, k):
        a = self.__dict__.get("_a")
        if a is not None and k in a:
            return a[k].copy()
        raise AttributeError(k)


class PackedCase:
    """Members (cases.Case of one level count and equal parameters but
    scale_area) as one case for model.GpuModel; `members` is the
    fesomc_members table the model is created with."""

    def __init__(self, member_cases, name="packed"):
        self.cases = list(member_cases)
        self.name = name
        p0 = self.cases[0].params
        for c in self.cases[1:]:
            for f, _ in abi.Params._fields_:
                if f in PER_MEMBER_PARAMS:
                    continue
                a, b = getattr(p0, f), getattr(c.params, f)
                if hasattr(a, "__len__"):
                    a, b = list(a), list(b)
                if a != b:
                    raise ValueError("packed members differ in parameter %s" % f)
        self.mesh = PackedMesh([c.mesh for c in self.cases])
        self.params = abi.Params()
        C.pointer(self.params)[0] = p0
        self.params.scale_area = float(self.mesh.scale_area[0])
        self.state0 = self._cat_state([c.state0 for c in self.cases])
        self.meta = {"members": [c.name for c in self.cases]}
        self._members_arrays = (np.ascontiguousarray(self.mesh.node_off), np.ascontiguousarray(self.mesh.elem_off),
                                np.ascontiguousarray(self.mesh.scale_area))
        m = abi.Members()
        m.n = len(self.cases)
        m.node_off = abi.iptr(self._members_arrays[0])
        m.elem_off = abi.iptr(self._members_arrays[1])
        m.scale_area = abi.dptr(self._members_arrays[2])
        self.members = m

    @staticmethod
    def _cat_state(states):
        return {k: np.concatenate([s[k] for s in states]) for k in states[0]}

    def new_state_arrays(self):
        return {k: v.copy() for k, v in self.state0.items()}

    def state_struct(self, arrays, time_jd, lfirst=1):
        return cases.Case.state_struct(self, arrays, time_jd, lfirst)

    def forcing_fn(self, nstep, time_jd):
        return self.pack_forcing([c.forcing_fn(nstep, time_jd) for c in self.cases])

    def pack_forcing(self, fdicts):
        """One forcing dict from the members' (same keys in every member)."""
        out = {}
        for k in fdicts[0]:
            vals = [f[k] for f in fdicts]
            if any(v is None for v in vals):
                if not all(v is None for v in vals):
                    raise ValueError("forcing %s given for some members only" % k)
                out[k] = None
            elif k in GLOBAL_FORCING:
                for v in vals[1:]:
                    if not np.array_equal(v, vals[0]):
                        raise ValueError("packed members need the same %s" % k)
                out[k] = np.asarray(vals[0], dtype=np.float64)
            elif k in OB_FORCING:
                out[k] = np.concatenate([np.asarray(v, dtype=np.float64).reshape(12, -1) for v in vals],
                                        axis=1).ravel()
            else:
                out[k] = np.concatenate([np.asarray(v, dtype=np.float64).ravel() for v in vals])
        return out

    def split_state(self, state):
        """Per-member state dicts of a packed state (sync_to_host order)."""
        no, eo = self.mesh.node_off, self.mesh.elem_off
        out = []
        for k, c in enumerate(self.cases):
            d = {}
            for name, v in state.items():
                if name.startswith("_"):
                    d[name] = v
                elif name in NODE_FIELDS:
                    w = len(c.state0[name]) // c.mesh.N
                    d[name] = v[no[k] * w:no[k + 1] * w]
                else:
                    w = len(c.state0[name]) // c.mesh.E
                    d[name] = v[eo[k] * w:eo[k + 1] * w]
            out.append(d)
        return out

    def split_runoff(self, runoff):
        off = np.concatenate([[0], np.cumsum(self.mesh.n_rivers)])
        return [runoff[off[k]:off[k + 1]] for k in range(len(self.cases))]


# fesomc_state fields per node (the rest are per element)
NODE_FIELDS = {"eta_n", "eta_n_1", "eta_n_2", "etaAB", "TF", "SF", "bt", "snu", "Kv", "Ri", "tke_dissip", "Wvel",
               "ssh_gp", "rho_c", "hpressure", "T_old", "S_old", "Tclim", "Sclim", "mask_wd_node"}
