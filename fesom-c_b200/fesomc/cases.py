"""Test cases for the FESOM-C time step: meshes, run parameters, initial
state and per-step forcing, laid out exactly as the reference's Fortran
driver leaves o_MESH / o_PARAM / o_ARRAYS before the main loop.

Two families:
  * le_medium(): the reference's own lock-exchange test case
    (test_cases/LE_medium; fv_run.dat values), read from the committed
    fixture tests/golden/le_medium.npz.
  * estuary(cfg): the synthetic estuary channel of the benchmark configs
    (structured quad grid, seeded 30 % triangle splits, sloping bathymetry
    with Gaussian-smoothed noise, M2 open-boundary tide, river inflow,
    optional uniform wind stress).
"""
import ctypes as C
import math
import os

import numpy as np

from . import abi

R_EARTH = 6400000.0
D_DE, D_GA, D_EP = 0.614, 0.088, 0.013        # AM4 weights, fv_ini.F90:143-146


class HostMesh:
    """Owns a fesomc_mesh_builder and numpy copies of its arrays."""

    def __init__(self, xy, index, elems, depth, *, cartesian, nsigma, coriolis_on=False, lat_deg=50.0,
                 ind_sigma=1, pow_sig=1.0, lev_bot=1.0, lev_sur=1.0, T_potential=False,
                 with_up_dn_tri=True, rivers=None, sponge_radius=None, lib=None):
        # lib: any object with the fesomc_mesh_* functions of the C-ABI (the
        # product library by default)
        lib = lib if lib is not None else abi.load()
        self.lib = lib
        xy = np.ascontiguousarray(xy, dtype=np.float64)
        index = np.ascontiguousarray(index, dtype=np.int32)
        elems = np.ascontiguousarray(elems, dtype=np.int32)
        depth = np.ascontiguousarray(depth, dtype=np.float64)
        opts = abi.MeshOpts(int(cartesian), int(coriolis_on), lat_deg, 360.0, nsigma, ind_sigma,
                            pow_sig, lev_bot, lev_sur, int(T_potential), int(with_up_dn_tri))
        h = C.c_void_p()
        abi.check(lib.fesomc_mesh_build(len(index), abi.dptr(xy), abi.iptr(index), len(elems),
                                        abi.iptr(elems), abi.dptr(depth), C.byref(opts), C.byref(h)),
                  "fesomc_mesh_build")
        self.handle = h
        if rivers is not None and len(rivers):
            r = np.ascontiguousarray(rivers, dtype=np.int32)
            abi.check(lib.fesomc_mesh_set_rivers(h, len(r), abi.iptr(r)), "fesomc_mesh_set_rivers")
        if sponge_radius:
            abi.check(lib.fesomc_mesh_set_sponge(h, float(sponge_radius)), "fesomc_mesh_set_sponge")
        self.c = abi.Mesh()
        abi.check(lib.fesomc_mesh_view(h, C.byref(self.c)), "fesomc_mesh_view")
        m = self.c
        self.N, self.E, self.Ed, self.Ed_in, self.NS = m.nod2D, m.elem2D, m.edge2D, m.edge2D_in, m.nsigma
        self.L = self.NS - 1
        self.scale_area = lib.fesomc_mesh_scale_area(h)

    def arr(self, name, shape, dtype=np.float64):
        p = getattr(self.c, name)
        n = int(np.prod(shape))
        if not p or n == 0:
            return None
        ctype = C.c_double if dtype == np.float64 else C.c_int32
        buf = C.cast(p, C.POINTER(ctype * n)).contents
        return np.frombuffer(buf, dtype=dtype).reshape(shape).copy()

    def __getattr__(self, k):
        shapes = {
            "index_nod2D": ((self.N,), np.int32), "elem2D_nodes": ((self.E, 4), np.int32),
            "edge_nodes": ((self.Ed, 2), np.int32), "edge_tri": ((self.Ed, 2), np.int32),
            "elem_edges": ((self.E, 4), np.int32), "elem_neighbors": ((self.E, 4), np.int32),
            "nod_in_elem2D_num": ((self.N,), np.int32),
            "nod_in_elem2D": ((self.N, self.c.nod_in_elem2D_max), np.int32),
            "edge_up_dn_tri": ((self.Ed, 2), np.int32), "coord_nod2D": ((self.N, 2), np.float64),
            "depth": ((self.N,), np.float64), "area": ((self.N,), np.float64),
            "elem_area": ((self.E,), np.float64), "elem_cos": ((self.E,), np.float64),
            "coriolis": ((self.E,), np.float64), "w_cv": ((self.E, 4), np.float64),
            "gradient_sca": ((self.E, 8), np.float64), "gradient_vec": ((self.E, 8), np.float64),
            "edge_dxdy": ((self.Ed, 2), np.float64), "edge_cross_dxdy": ((self.Ed, 4), np.float64),
            "sigma": ((self.NS,), np.float64), "a_tp": ((2, self.N), np.float64), "ac": ((self.N,), np.float64),
            "in_obn": ((self.c.nobn,), np.int32), "nod_rivers": ((self.c.n_rivers,), np.int32),
        }
        if k in shapes:
            shp, dt = shapes[k]
            return self.arr(k, shp, dt)
        raise AttributeError(k)

    def close(self):
        if self.handle:
            self.lib.fesomc_mesh_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def default_params(**kw):
    p = abi.Params()
    p.dt, p.dt_2D = 0.5, 0.1
    p.Dmin = 0.25
    p.C_d = 0.0
    p.beta, p.epsilon = 0.281105, 0.01          # fv_var.F90:108,110
    p.snul, p.z0b_min, p.z0s_min = 7.5e-4, 0.01, 0.02
    p.Pr_num, p.beta_scale, p.cka = 0.0001, 3.9, 0.4   # fv_var.F90:44,130,16
    p.tau_inv_filt, p.K_hor = 0.000046296, 0.010
    p.bih_3D, p.Abh0 = 0, 1000.0                  # LE_medium fv_run.dat:150,160
    p.filt_bi_3D, p.filt_bi_2D, p.tau_c = 0, 0, 0.4   # fv_run.dat:153,156,159
    p.bih_2D = 0                                   # fv_run.dat:157
    p.T_potential = 0
    # atmospheric forcing off; its shortwave settings as in LE_medium's
    # fv_run.dat:280-286 (type_swr_body 1, jer_const, R a b = 0.78 1.4 7.9)
    p.key_atm, p.type_swr_body, p.jer_const = 0, 1, 1
    p.Rjc, p.ajc, p.bjc = 0.78, 1.4, 7.9
    p.Cd_bz, p.Bp_bz = 10.0, 5.0
    p.clim_relax = 1.0 / (15.0 * 3600.0 * 24.0)
    p.relax2clim_ac = 1.0 / (60.0 * 3600.0 * 24.0)
    p.river_salinity = float(np.float32(0.2))   # REAL(4) literal 0.2 (fv_main.F90:1818)
    p.time_jd0 = 2457266.5
    p.mom_adv_2D, p.mom_adv_3D, p.vert_adv = 2, 1, 1
    p.im_vert_visc, p.im_vert_visc_fic, p.fic_point = 0, 1, 1
    p.tracer_adv, p.ver_mix = abi.TRACER_UPWIND, 3
    p.filt_2D = p.filt_3D = 0
    p.wet_dry_on = p.key_rivers = p.TF_presence = p.restart = 0
    p.cl_relax, p.cl_solid_boder_relax = 1, 0
    p.temp_on, p.salinity_on = 1, 0
    p.n_harm = 0
    for k, v in kw.items():
        setattr(p, k, v)
    p.Mt = int(p.dt / p.dt_2D)                   # fv_read_run.F90:1060
    return p


class Case:
    """Mesh + parameters + initial state + forcing generator."""

    def __init__(self, name, mesh, params, state, forcing_fn, meta=None):
        self.name, self.mesh, self.params, self.state0, self.forcing_fn = name, mesh, params, state, forcing_fn
        self.meta = meta or {}

    def new_state_arrays(self):
        return {k: v.copy() for k, v in self.state0.items()}

    def state_struct(self, arrays, time_jd, lfirst=1):
        s = abi.State()
        for k in abi.STATE_FIELDS:
            a = arrays.get(k)
            setattr(s, k, abi.dptr(a) if a is not None else None)
        s.lfirst = lfirst
        s.time_jd = time_jd
        return s


def initial_state(mesh, params, TF, SF, wet_dry_on):
    """initial_state (fv_ini.F90:113-150, 487-546) + wad_mask before the loop."""
    N, E, L, NS = mesh.N, mesh.E, mesh.L, mesh.NS
    depth = mesh.depth
    eta = np.zeros(N)
    neg = depth + eta < 0.0
    eta[neg] = -depth[neg]
    eta1, eta2 = eta.copy(), eta.copy()
    fe = 1.0 - D_DE - D_GA - D_EP
    etaAB = D_DE * eta + fe * eta + D_GA * eta1 + D_EP * eta2
    st = {
        "eta_n": eta, "eta_n_1": eta1, "eta_n_2": eta2, "etaAB": etaAB,
        "U_n_2D": np.zeros(2 * E), "U_n_1": np.zeros(2 * E), "U_n_2": np.zeros(2 * E),
        "U_filt_2D": np.zeros(E), "V_filt_2D": np.zeros(E),
        "U_n": np.zeros(L * E), "V_n": np.zeros(L * E), "U_rhsAB": np.zeros(L * E), "V_rhsAB": np.zeros(L * E),
        "U_n_filt": np.zeros(L * E), "V_n_filt": np.zeros(L * E),
        "TF": np.ascontiguousarray(TF.reshape(-1)), "SF": np.ascontiguousarray(SF.reshape(-1)),
        "bt": np.full(NS * N, 1.0e-8), "snu": np.full(NS * N, params.snul), "Kv": np.full(NS * N, params.snul),
        "Ri": np.zeros(NS * N), "tke_dissip": np.zeros(NS * N), "Av": np.full(NS * E, params.snul),
        "Wvel": np.zeros(NS * N), "ssh_gp": np.zeros(N),
        "rho_c": np.zeros(L * N), "hpressure": np.zeros(NS * N), "Bar_pr_2D": np.zeros(2 * E),
    }
    st["T_old"] = st["TF"].copy()
    st["S_old"] = st["SF"].copy()
    st["Tclim"] = st["TF"].copy()
    st["Sclim"] = st["SF"].copy()
    mask_wd = np.ones(E)
    mask_wd_node = np.ones(N)
    if wet_dry_on:
        en = mesh.elem2D_nodes - 1
        dmin4 = depth[en].min(axis=1)
        emax4 = etaAB[en].max(axis=1)
        mask_wd = np.where(dmin4 + emax4 > params.Dmin, 1.0, 0.0)
        mask_wd_node = np.where(depth + etaAB > params.Dmin, 1.0, 0.0)
    st["mask_wd"], st["mask_wd_node"] = mask_wd, mask_wd_node
    return st


def _fixture_path():
    return os.path.join(abi.REPO_DIR, "tests", "golden", "le_medium.npz")


def le_medium(nsigma=40, lib=None):
    """The reference's LE_medium lock-exchange case (fv_run.dat of the case).
    lib: the mesh builder to use (default: the product library)."""
    d = np.load(_fixture_path())
    depth = np.full(len(d["nod_index"]), 20.0)          # title 'LE' (fv_main.F90:915-916)
    mesh = HostMesh(d["nod_xy"], d["nod_index"], d["elem_nodes"], depth, cartesian=False,
                    nsigma=nsigma, coriolis_on=False, with_up_dn_tri=True, lib=lib)
    lib = lib if lib is not None else abi.load()
    p = default_params()
    p.scale_area = mesh.scale_area
    p.density_0 = 1000.0 + lib.fesomc_host_density_jm(20.0, 30.0, 0.0, 1000.0)
    L = mesh.L
    x = mesh.coord_nod2D[:, 0]
    tcol = np.where(x < 0.0, 5.0 / 0.28, 10.0 / 0.28)
    TF = np.repeat(tcol[:, None], L, axis=1)
    SF = np.zeros_like(TF)                               # SALINITY_ON = F: SF stays 0
    st = initial_state(mesh, p, TF, SF, wet_dry_on=False)
    E, N = mesh.E, mesh.N
    zeros_e, zeros_n = np.zeros(E), np.zeros(N)

    def forcing(step, time_jd):
        return {"taux": zeros_e, "tauy": zeros_e, "windx": zeros_n, "windy": zeros_n}

    return Case("le_medium", mesh, p, st, forcing, meta={"energy": d["energy"], "irep": 100})


# --------------------------------------------------------------------------
# synthetic estuary
# --------------------------------------------------------------------------
# Open-boundary settings of the estuary, both run-file parameters of the
# reference (fv_read_run.F90:877-898 and the SL_obn / SL_radius options).
# Without them the 80 m estuary diverges within a few hours of model time:
# an open-boundary node keeps its advective tracer tendency on inflow
# (fv_tracer.F90:300-330) but gets no flux through the open edge itself, so
# the tracer anomaly there grows exponentially (first at the shallow corner),
# and currents along the clamped-elevation boundary grow next to the far
# corner.  A relaxation to climatology on a 60 s time scale (faster than
# that growth, whose rate is of order u / dx) holds the boundary tracers,
# and a 5 km sponge layer (ac scaling of advection and viscosity, raised
# bottom drag) damps the boundary currents.
SPONGE_RADIUS = 5000.0                                   # m
OB_RELAX_S = 60.0                                        # clim_relax, relax2clim_ac time scale

ESTUARY_CFGS = {
    # name: (nx quads, ny quads, spacing m, nsigma, depth at y=0, depth at y=Ly, wind stress N/m2)
    "cfg0": (200, 80, 300.0, 11, 2.0, 25.0, 0.0),
    "cfg1": (1500, 700, 80.0, 21, 2.0, 40.0, 0.1),
    "small": (40, 16, 300.0, 11, 2.0, 25.0, 0.05),
    "medium": (300, 140, 150.0, 21, 2.0, 40.0, 0.1),
    # cfg1 generator at a quarter of the nodes: profiling captures
    "quarter": (700, 330, 170.0, 21, 2.0, 40.0, 0.1),
}


def estuary_geometry(nx, ny, dx, seed=20261203, split_frac=0.3, h0=2.0, h1=25.0, noise_sigma=0.5,
                     corr_len=2000.0):
    """Structured (nx+1)x(ny+1) node grid, nx*ny quads; a seeded 30 % of the
    quads are split into two triangles along a random diagonal.  Depth rises
    linearly in y plus Gaussian-smoothed white noise scaled to noise_sigma."""
    rng = np.random.default_rng(seed)
    ix, iy = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), indexing="xy")
    nid = (iy * (nx + 1) + ix + 1).astype(np.int64)      # 1-based, row-major in y
    x = ix * dx
    y = iy * dx
    xy = np.stack([x.ravel(), y.ravel()], axis=1).astype(np.float64)
    index = np.zeros((ny + 1, nx + 1), dtype=np.int32)
    index[0, :] = 1
    index[-1, :] = 1
    index[:, 0] = 1
    index[:, -1] = 2                                     # open boundary at x = Lx
    # quads, clockwise (n1 lower-left, n2 upper-left, n3 upper-right, n4 lower-right)
    n1 = nid[:-1, :-1].ravel()
    n2 = nid[1:, :-1].ravel()
    n3 = nid[1:, 1:].ravel()
    n4 = nid[:-1, 1:].ravel()
    nq = n1.size
    split = rng.random(nq) < split_frac
    diag = rng.random(nq) < 0.5
    elems = []
    q = ~split
    elems.append(np.stack([n1[q], n2[q], n3[q], n4[q]], axis=1))
    s13 = split & diag
    elems.append(np.stack([n1[s13], n2[s13], n3[s13], n1[s13]], axis=1))
    elems.append(np.stack([n1[s13], n3[s13], n4[s13], n1[s13]], axis=1))
    s24 = split & ~diag
    elems.append(np.stack([n1[s24], n2[s24], n4[s24], n1[s24]], axis=1))
    elems.append(np.stack([n2[s24], n3[s24], n4[s24], n2[s24]], axis=1))
    elems = np.concatenate(elems).astype(np.int32)
    # bathymetry
    Ly = ny * dx
    base = h0 + (h1 - h0) * (y / Ly)
    noise = rng.standard_normal((ny + 1, nx + 1))
    from scipy.ndimage import gaussian_filter
    sm = gaussian_filter(noise, sigma=corr_len / dx, mode="reflect")
    sd = sm.std()
    if sd > 0:
        sm = sm * (noise_sigma / sd)
    depth = (base + sm).ravel().astype(np.float64)
    return xy, index.ravel(), elems, depth, (nx + 1, ny + 1)


def estuary(cfg="cfg0", seed=20261203, tracer_adv=abi.TRACER_MUSCL, sponge_radius=SPONGE_RADIUS, **overrides):
    """One of the named estuary configurations (ESTUARY_CFGS).  lib=... (in
    overrides) selects the mesh builder, default the product library."""
    nx, ny, dx, nsigma, h0, h1, tau = ESTUARY_CFGS[cfg]
    # uniform stress, cross-shore (+y, from the shore towards deep water); an
    # along-channel stress towards the open boundary drives the shallow
    # shore corner at the open boundary unstable in the reference scheme
    # within a few hours of model time
    return estuary_case(cfg, nx, ny, dx, nsigma, h0, h1, stress=(0.0, tau), seed=seed, tracer_adv=tracer_adv,
                        sponge_radius=sponge_radius, **overrides)


def estuary_case(name, nx, ny, dx, nsigma, h0, h1, *, stress=(0.0, 0.0), m2_amp=1.2, m2_phase_deg=0.0,
                 noise_sigma=0.5, seed=20261203, tracer_adv=abi.TRACER_MUSCL, sponge_radius=SPONGE_RADIUS,
                 lib=None, atm=None, shuffle=None, **overrides):
    """Synthetic estuary: nx x ny quads at dx metres, 30 % split into
    triangles, depth h0 -> h1 across the channel plus smoothed noise of
    noise_sigma metres, river at x = 0, M2 tide of m2_amp metres and phase
    m2_phase_deg at the open boundary x = nx*dx, uniform wind stress
    (taux, tauy) in N/m2.  atm: atmospheric forcing (turns key_atm on), a
    dict of node fields or constants among qns, qsr (W/m2, downward), emp
    (E - P), mslp (Pa) and Rj, aj, bj (jer_const = 0), or a callable
    (mesh) -> such a dict, pushed with every step's forcing.  shuffle: a
    seed that numbers the nodes and lists the elements in random order (a
    mesh as it may come from a mesh generator's file, not row by row).
    Parameter overrides go to default_params."""
    xy, index, elems, depth, (nxn, nyn) = estuary_geometry(nx, ny, dx, seed=seed, h0=h0, h1=h1,
                                                            noise_sigma=noise_sigma)
    rivers = np.arange(0, nyn) * nxn + 1                 # every node on x = 0 (1-based)
    if shuffle is not None:
        rs = np.random.default_rng([seed, shuffle])
        pn = rs.permutation(len(index))                  # new node j is old node pn[j]
        new_of_old = np.empty(len(index), dtype=np.int64)
        new_of_old[pn] = np.arange(len(index))
        xy, index, depth = xy[pn], index[pn], depth[pn]
        elems = (new_of_old[elems - 1] + 1).astype(np.int32)[rs.permutation(len(elems))]
        rivers = new_of_old[rivers - 1] + 1
    # T_potential switches both the potential and the mesh's a_tp weights
    mesh = HostMesh(xy, index, elems, depth, cartesian=True, nsigma=nsigma, coriolis_on=True,
                    lat_deg=50.0, with_up_dn_tri=True, rivers=rivers, sponge_radius=sponge_radius,
                    T_potential=bool(overrides.get("T_potential", 0)), lib=lib)
    lib = lib if lib is not None else abi.load()
    kw = dict(dt=20.0, dt_2D=2.0, Dmin=1.0, C_d=0.0025, tracer_adv=tracer_adv, wet_dry_on=1,
              key_rivers=1, TF_presence=1, temp_on=1, salinity_on=1, filt_2D=1, filt_3D=1,
              river_salinity=5.0, clim_relax=1.0 / OB_RELAX_S, relax2clim_ac=1.0 / OB_RELAX_S)
    kw.update(overrides)
    if atm is not None:
        kw["key_atm"] = 1
    p = default_params(**kw)
    p.n_harm = 1
    p.harm_index[0] = 0                                  # M2
    p.scale_area = mesh.scale_area
    p.density_0 = 1000.0 + lib.fesomc_host_density_jm(12.0, 30.0, 0.0, 1000.0)
    N, E, L = mesh.N, mesh.E, mesh.L
    sig = mesh.sigma
    a = np.maximum(mesh.depth, p.Dmin)
    zbar = (1.0 - sig[None, :]) * a[:, None]
    Zmid = 0.5 * (zbar[:, :-1] + zbar[:, 1:])
    TF = 12.0 - 0.05 * Zmid                              # 0.5 C per 10 m
    SF = np.full((N, L), 30.0)
    st = initial_state(mesh, p, TF, SF, wet_dry_on=bool(p.wet_dry_on))
    nobn = mesh.c.nobn
    ampt = np.zeros((12, nobn))
    ampt[0, :] = m2_amp                                   # M2 amplitude, m
    fazt = np.zeros((12, nobn))
    fazt[0, :] = m2_phase_deg * (math.pi / 180.0)         # radians, as the OB harmonics take it
    amp_factor, phy_factor = np.ones(12), np.zeros(12)
    sx, sy = stress
    tau = math.hypot(sx, sy)
    taux, tauy = np.full(E, float(sx)), np.full(E, float(sy))
    # 10 m wind speed of the stress (rho_air 1.3, C_D 1.3e-3) for the surface
    # TKE flux, in the direction of the stress
    wspd = math.sqrt(tau / (1.3 * 1.3e-3)) if tau > 0 else 0.0
    windx = np.full(N, wspd * (sx / tau) if tau > 0 else 0.0)
    windy = np.full(N, wspd * (sy / tau) if tau > 0 else 0.0)
    nriv = mesh.c.n_rivers
    q_total = 500.0
    atm_fields = {}
    if atm is not None:
        a = atm(mesh) if callable(atm) else atm
        for k, v in a.items():
            atm_fields[k] = np.ascontiguousarray(np.broadcast_to(np.asarray(v, dtype=np.float64), (N,)))

    def forcing(step, time_jd):
        # rivers_do (fv_rivers.F90:263-299): constant runoff, 10-day ramp
        r = np.full(nriv, q_total / max(nriv, 1))
        if time_jd - p.time_jd0 < 10.0:
            r = r * (time_jd - p.time_jd0) / 10.0
        f = {"taux": taux, "tauy": tauy, "windx": windx, "windy": windy, "runoff_rivers": r,
             "ampt": ampt.reshape(-1).copy(), "fazt": fazt.reshape(-1).copy(),
             "amp_factor": amp_factor, "phy_factor": phy_factor}
        f.update(atm_fields)
        return f

    meta = {"nx": nx, "ny": ny, "dx": dx, "stress": (float(sx), float(sy)), "m2_amp": m2_amp,
            "m2_phase_deg": m2_phase_deg, "noise_sigma": noise_sigma}
    return Case(name, mesh, p, st, forcing, meta=meta)


# --------------------------------------------------------------------------
# perturbed estuary ensemble
# --------------------------------------------------------------------------
ENSEMBLE_NODES = (20_000, 250_000)


def ensemble_draw(index, seed=20261203, nodes_range=ENSEMBLE_NODES):
    """Parameters of ensemble member `index`: the cfg0 generator (300 m
    quads, 30 % split, depth 2 -> 25 m, aspect of the 200 x 80 grid) at a
    node count drawn log-uniformly in nodes_range, 11 or 21 sigma levels, M2
    amplitude 1.2 m +-20 %, phase +-15 degrees, uniform stress 0-0.2 N/m2 in
    a random direction, bathymetry noise sigma 0-1 m.  Each member draws
    from its own generator seeded by (seed, index)."""
    rng = np.random.default_rng([seed, index])
    lo, hi = nodes_range
    nodes = math.exp(rng.uniform(math.log(lo), math.log(hi)))
    ny1 = max(9, int(round(math.sqrt(nodes * 81.0 / 201.0))))
    nx1 = max(9, int(round(nodes / ny1)))
    nsigma = 11 if rng.random() < 0.5 else 21
    amp = 1.2 * (1.0 + rng.uniform(-0.2, 0.2))
    phase = rng.uniform(-15.0, 15.0)
    tau = rng.uniform(0.0, 0.2)
    th = rng.uniform(0.0, 2.0 * math.pi)
    noise = rng.uniform(0.0, 1.0)
    return {"nx": nx1 - 1, "ny": ny1 - 1, "nsigma": nsigma, "m2_amp": amp, "m2_phase_deg": phase,
            "stress": (tau * math.cos(th), tau * math.sin(th)), "noise_sigma": noise,
            "seed": seed + 7919 * (index + 1)}


def ensemble_member(index, seed=20261203, nodes_range=ENSEMBLE_NODES, **overrides):
    """Case of ensemble member `index` (ensemble_draw)."""
    d = ensemble_draw(index, seed, nodes_range)
    return estuary_case(f"member{index}", d["nx"], d["ny"], 300.0, d["nsigma"], 2.0, 25.0, stress=d["stress"],
                        m2_amp=d["m2_amp"], m2_phase_deg=d["m2_phase_deg"], noise_sigma=d["noise_sigma"],
                        seed=d["seed"], **overrides)


ATM_FIELDS = ("xwind", "ywind", "humidity", "shortwave", "longwave", "tair", "precipitation", "mslp")


def atm_coefficients(mesh, time_jd0, seed=3):
    """Synthetic atmospheric forcing for sbc_do (fesomc_gpu_set_atm_fields):
    the time-interpolation coefficients of the 8 fields per node (ATM_FIELDS
    order; m/s, kg/kg, W/m2, W/m2, K, kg/m2/s, Pa) for fields that vary over
    the mesh and drift over a day from time_jd0: value(t) = t * a + b, as
    getcoeffld (src/fv_sbc.F90:664-836) prepares them.  Returns (a, b), each
    8 values per node in the reference layout coef(i_totfl, nod2D)."""
    rng = np.random.default_rng(seed)
    N = mesh.N
    x = mesh.coord_nod2D[:, 0] / max(mesh.coord_nod2D[:, 0].max(), 1.0)
    v0 = np.stack([6.0 + 4.0 * x, -3.0 + 2.0 * rng.random(N), 0.004 + 0.002 * rng.random(N),
                   150.0 + 100.0 * x, 300.0 + 20.0 * rng.random(N), 281.0 + 4.0 * x,
                   2.0e-5 * rng.random(N), 101000.0 + 600.0 * x], axis=1)
    rate = np.stack([2.0 + 0 * x, -1.0 + 0 * x, 0.001 + 0 * x, 50.0 * x, 5.0 + 0 * x, 1.5 + 0 * x,
                     1.0e-6 + 0 * x, 100.0 + 0 * x], axis=1)
    return (np.ascontiguousarray(rate).reshape(-1),
            np.ascontiguousarray(v0 - time_jd0 * rate).reshape(-1))


def forcing_struct(fdict):
    """fesomc_forcing pointing at the arrays of fdict (kept alive by caller)."""
    f = abi.Forcing()
    for k in ("taux", "tauy", "windx", "windy", "runoff_rivers", "Tclim", "Sclim", "ampt", "fazt",
              "amp_factor", "phy_factor", "mslp", "emp", "qsr", "qns", "Rj", "aj", "bj"):
        a = fdict.get(k)
        if a is not None:
            a = np.ascontiguousarray(a, dtype=np.float64)
            fdict[k] = a
        setattr(f, k, abi.dptr(a) if a is not None else None)
    return f


def advance_time(time_jd, dt):
    """time_jd = time_jd + dt/86400 (fv_main.F90:400)."""
    return time_jd + dt / 86400.0
