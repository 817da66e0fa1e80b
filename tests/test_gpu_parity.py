"""GPU parity: the sm_100a FP64 path against the CPU oracle, called through
the C-ABI.  Both sides follow the reference's operation order without FMA
contraction, and the one transcendental of the step (the logarithm in
d3_end's bottom boundary value) is the same IEEE-only evaluation on both
(fesomc_log), so integer / mask results and every floating-point field are
compared for exact equality at every step count.  This is stricter than the
FP64 target of 1e-11 relative.

Every case is built twice: with the product library's host mesh builder for
the GPU run, and with the oracle's own restatement of the mesh set-up
(oracle/oracle_mesh.c) for the oracle run, so that nothing the oracle reads
comes from the product."""
import math

import numpy as np
import pytest


def half_unit_e16_7(v):
    """Half a unit in the last digit of Fortran format e16.7 (0.dddddddE+xx)."""
    return 0.5 * 10.0 ** (math.floor(math.log10(abs(v))) + 1 - 7)

pytestmark = pytest.mark.gpu

FIELDS = ["eta_n", "eta_n_1", "eta_n_2", "etaAB", "U_n_2D", "U_n_1", "U_n_2", "U_filt_2D", "V_filt_2D",
          "U_n", "V_n", "U_rhsAB", "V_rhsAB", "U_n_filt", "V_n_filt", "TF", "SF", "T_old", "S_old",
          "bt", "snu", "Kv", "Ri", "tke_dissip", "Av", "Wvel", "mask_wd", "mask_wd_node", "rho_c",
          "hpressure", "Bar_pr_2D"]


@pytest.fixture(scope="module")
def mods(built):
    import pyoracle
    from fesomc import abi, cases, model
    return abi, cases, model, pyoracle


def compare(sg, so):
    bad = []
    for f in FIELDS:
        a, b = sg[f], so[f]
        if not np.array_equal(a, b):
            bad.append((f, int(np.sum(a != b)), float(np.max(np.abs(a - b)))))
    return bad


def build_pair(mods, make):
    """make(lib) -> case; returns (case for the GPU, case for the oracle)."""
    abi, cases, model, pyoracle = mods
    return make(None), make(pyoracle.MeshLib(abi))


def run_pair(mods, make, steps, shapes=None):
    """steps of the GPU path (launch shapes / kernel forms `shapes`, by knob
    name) and of the oracle; returns (differing fields, the two energies)."""
    abi, cases, model, pyoracle = mods
    gcase, ocase = build_pair(mods, make)
    g = model.GpuModel(gcase)
    if shapes:
        from fesomc import autotune
        autotune.apply(g, shapes)
    o = pyoracle.Oracle(ocase, abi, cases)
    g.step(steps)
    o.step(steps)
    bad = compare(g.state(), o.state())
    eg, eo = g.energy(), o.energy()
    g.close()
    o.close()
    return bad, eg, eo


def est(cases, *a, **kw):
    """estuary case factory for build_pair / run_pair"""
    return lambda lib: cases.estuary(*a, lib=lib, **kw)


def le(cases, **params):
    """LE_medium factory (Mt = 4, the golden series' sub-step count) with
    parameter overrides"""
    def make(lib):
        c = cases.le_medium(lib=lib)
        c.params.Mt = 4
        for k, v in params.items():
            setattr(c.params, k, v)
        return c
    return make


def test_le_medium_bit_exact(mods):
    abi, cases, model, pyoracle = mods
    bad, eg, eo = run_pair(mods, le(cases), 20)
    assert bad == []
    assert abs(eg - eo) <= 1e-12 * abs(eo)


def test_estuary_muscl_wetdry_tides_rivers_bit_exact(mods):
    abi, cases, model, pyoracle = mods
    bad, eg, eo = run_pair(mods, est(cases, "small"), 30)
    assert bad == []
    assert abs(eg - eo) <= 1e-12 * abs(eo)


def test_estuary_upwind_implicit_visc_bit_exact(mods):
    abi, cases, model, pyoracle = mods
    case = est(cases, "small", tracer_adv=abi.TRACER_UPWIND, im_vert_visc=1, im_vert_visc_fic=0,
               filt_2D=0, filt_3D=0)
    bad, _, _ = run_pair(mods, case, 20)
    assert bad == []


def test_estuary_miura_bit_exact(mods):
    """solve_tracer_miura (temperature only, salinity passes through
    advection) with wetting/drying, tides and rivers."""
    abi, cases, model, pyoracle = mods
    bad, eg, eo = run_pair(mods, est(cases, "small", tracer_adv=abi.TRACER_MIURA), 20)
    assert bad == []
    assert abs(eg - eo) <= 1e-12 * abs(eo)


def test_le_medium_miura_bit_exact(mods):
    abi, cases, model, pyoracle = mods
    bad, _, _ = run_pair(mods, le(cases, tracer_adv=abi.TRACER_MIURA), 20)
    assert bad == []


def test_estuary_both_vertical_viscosities_and_fic_points(mods):
    abi, cases, model, pyoracle = mods
    for fic in (0, 2):
        bad, _, _ = run_pair(mods, est(cases, "small", im_vert_visc=1, im_vert_visc_fic=1, fic_point=fic), 10)
        assert bad == [], fic


def test_estuary_medium_21_levels(mods):
    """42k nodes x 20 layers, 20 internal steps, exact."""
    abi, cases, model, pyoracle = mods
    bad, _, _ = run_pair(mods, est(cases, "medium"), 20)
    assert bad == []


def test_le_long_run_bit_exact(mods):
    abi, cases, model, pyoracle = mods
    bad, eg, eo = run_pair(mods, le(cases), 200)
    assert bad == []
    # the energy integral is a parallel compensated sum on the device and a
    # serial sum in the oracle: equal state, round-off-level difference
    assert abs(eg - eo) <= 1e-12 * abs(eo)


def test_estuary_upwind_implicit_visc_long_run(mods):
    """The configuration whose state first exposed a one-ulp difference of the
    device log against libm's, run ten times longer than the other cases."""
    abi, cases, model, pyoracle = mods
    case = est(cases, "small", tracer_adv=abi.TRACER_UPWIND, im_vert_visc=1, im_vert_visc_fic=0,
               filt_2D=0, filt_3D=0)
    bad, _, _ = run_pair(mods, case, 200)
    assert bad == []


# the LE golden series (energy_tocheck.dat of the reference's LE_medium test
# case, one row per 100 steps, 7 printed digits): rows the GPU must track,
# and rows over which the oracle, on its own mesh, runs beside it
GOLDEN_ROWS_GPU = 2000
GOLDEN_ROWS_ORACLE = 150


def test_le_golden_energy_series(mods):
    """The GPU tracks the reference's printed energy over 2000 rows (200,000
    steps, 1.16 model days); over the first 150 rows the oracle runs beside
    it and both energies agree to 1e-12.  The first row whose energy no longer
    rounds to the printed 7 digits (if any) is named in the failure."""
    abi, cases, model, pyoracle = mods
    gcase, ocase = build_pair(mods, le(cases))
    gold = gcase.meta["energy"]
    assert len(gold) >= GOLDEN_ROWS_GPU
    g = model.GpuModel(gcase)
    o = pyoracle.Oracle(ocase, abi, cases)
    off = []
    try:
        for row in range(GOLDEN_ROWS_GPU):
            g.run(100)                       # LE has no forcing: graph replay
            eg = g.energy()
            if row < GOLDEN_ROWS_ORACLE:
                o.step(100)
                eo = o.energy()
                assert abs(eg - eo) <= 1e-12 * abs(eo), row
            if abs(eg - gold[row, 1]) > half_unit_e16_7(gold[row, 1]):
                off.append((row, eg, float(gold[row, 1])))
    finally:
        g.close()
        o.close()
    assert off == [], "first departing row %d (%r), %d rows off" % (off[0][0], off[0][1:], len(off))


def test_cfg0_two_tidal_days(mods):
    """The reference's CPU-sized configuration (201 x 81 nodes at 300 m, 11
    sigma levels, MUSCL, wetting/drying, M2 tide, river) over its stated run,
    2 tidal days = 8,942 internal steps with the forcing of every step pushed
    from the host, GPU against the oracle: wet/dry masks equal, and every
    field within 1e-11 of its magnitude (the comparison is exact in practice;
    the fields that differ at all are part of the failure text)."""
    abi, cases, model, pyoracle = mods
    steps = int(round(2 * 2 * 12.42 * 3600.0 / 20.0))        # 2 tidal days of 20 s steps
    assert steps == 8942
    gcase, ocase = build_pair(mods, est(cases, "cfg0"))
    g = model.GpuModel(gcase)
    o = pyoracle.Oracle(ocase, abi, cases)
    try:
        assert g.step(steps) == 0
        assert o.step(steps) == 0
        sg, so = g.state(), o.state()
        eg, eo = g.energy(), o.energy()
    finally:
        g.close()
        o.close()
    assert sg["_time_jd"] == so["_time_jd"]
    for f in ("mask_wd", "mask_wd_node"):
        assert np.array_equal(sg[f], so[f]), f
    differing = compare(sg, so)
    for f in FIELDS:
        scale = max(float(np.abs(so[f]).max()), 1e-300)
        assert float(np.abs(sg[f] - so[f]).max()) <= 1e-11 * scale, (f, differing)
    assert differing == [], differing
    assert abs(eg - eo) <= 1e-12 * abs(eo)


def test_cfg1_bit_exact(mods):
    """The 1.05M-node, 21-level benchmark mesh (1501 x 701 nodes at 80 m, 30 %
    of quads split, MUSCL, wetting/drying, tide, river, 0.1 N/m2 wind),
    4 internal steps, GPU against the oracle, exact."""
    abi, cases, model, pyoracle = mods
    gcase, ocase = build_pair(mods, est(cases, "cfg1"))
    g = model.GpuModel(gcase)
    o = pyoracle.Oracle(ocase, abi, cases)
    try:
        g.step(4)
        o.step(4)
        bad = compare(g.state(), o.state())
        eg, eo = g.energy(), o.energy()
    finally:
        g.close()
        o.close()
    assert bad == []
    assert abs(eg - eo) <= 1e-12 * abs(eo)


def test_graph_run_equals_stepwise(mods):
    """fesomc_gpu_run (forcing of the first step held, graph replay) equals
    fesomc_gpu_step when the forcing does not change (LE has none)."""
    abi, cases, model, pyoracle = mods
    case = cases.le_medium()
    a = model.GpuModel(case)
    b = model.GpuModel(case)
    a.step(12)
    b.run(12)
    sa, sb = a.state(), b.state()
    for f in FIELDS:
        assert np.array_equal(sa[f], sb[f]), f
    a.close()
    b.close()


def test_deterministic_repeat(mods):
    abi, cases, model, pyoracle = mods
    case = cases.estuary("small")
    res = []
    for _ in range(2):
        g = model.GpuModel(case)
        g.step(15)
        res.append(g.state())
        g.close()
    for f in FIELDS:
        assert np.array_equal(res[0][f], res[1][f]), f


def test_negative_salinity_reported(mods):
    """Host-injected river water of absurd negative salinity drives S < 0."""
    abi, cases, model, pyoracle = mods
    case = cases.estuary("small", river_salinity=-1.0e9)
    g = model.GpuModel(case)
    rc = g.step(1, check=False)
    assert rc == 5          # FESOMC_ENEGSALT
    g.close()


def test_low_temperature_reported(mods):
    abi, cases, model, pyoracle = mods
    case = cases.estuary("small")
    L = case.mesh.L
    case.state0["TF"][L * 7: L * 9] = -10.0
    case.state0["T_old"][L * 7: L * 9] = -10.0
    g = model.GpuModel(case)
    rc = g.step(1, check=False)
    assert rc == 6          # FESOMC_ELOWTEMP
    g.close()


def test_sync_roundtrip(mods):
    abi, cases, model, pyoracle = mods
    case = cases.estuary("small")
    g = model.GpuModel(case)
    g.step(3)
    s = g.state()
    import ctypes as C
    s2 = {k: (v * 1.0) for k, v in s.items() if k != "_time_jd"}
    st = case.state_struct(s2, s["_time_jd"], lfirst=0)
    abi.check(g.lib.fesomc_gpu_sync_from_host(g.h, abi.F_ALL, C.byref(st)))
    s3 = g.state()
    for f in FIELDS:
        assert np.array_equal(s[f], s3[f]), f
    g.close()


def test_estuary_biharmonic_bit_exact(mods):
    """biharmonic_viscosity (two edge Laplacians, vel_lapl_gradients) on the
    small estuary with the sponge factor, 30 steps."""
    abi, cases, model, pyoracle = mods
    bad, eg, eo = run_pair(mods, est(cases, "small", bih_3D=1, Abh0=1e4), 30)
    assert bad == []


def test_le_biharmonic_bit_exact(mods):
    abi, cases, model, pyoracle = mods
    bad, _, _ = run_pair(mods, le(cases, bih_3D=1), 20)
    assert bad == []


def test_biharmonic_2d_bit_exact(mods):
    """biharmonic_2D (bih_2D: two 2D Laplacians per sub-step, the second
    one's gradients from vel_gradients_2D) on the small estuary, 30 steps,
    and on LE, 20 steps."""
    abi, cases, model, pyoracle = mods
    bad, _, _ = run_pair(mods, est(cases, "small", bih_2D=1, Abh0=1e4), 30)
    assert bad == []
    bad, _, _ = run_pair(mods, le(cases, bih_2D=1), 20)
    assert bad == []


def test_tidal_potential_bit_exact(mods):
    """T_potential: the potential kernel (all 11 equilibrium harmonics, the
    shared IEEE-only sine and cosine) gives the oracle's ssh_gp, and the run
    that feels it stays bit-exact, 30 steps."""
    abi, cases, model, pyoracle = mods
    def make(lib):
        case = cases.estuary("small", T_potential=1, lib=lib)
        case.params.n_harm = 11
        for j in range(11):
            case.params.harm_index[j] = j
        return case
    gcase, ocase = build_pair(mods, make)
    g = model.GpuModel(gcase)
    o = pyoracle.Oracle(ocase, abi, cases)
    g.step(30)
    o.step(30)
    sg, so = g.state(), o.state()
    g.close()
    o.close()
    assert np.abs(so["ssh_gp"]).max() > 0.0
    assert np.array_equal(sg["ssh_gp"], so["ssh_gp"])
    assert compare(sg, so) == []


@pytest.mark.parametrize("nsigma", [64, 127])
def test_estuary_many_levels_bit_exact(mods, nsigma):
    """Level counts far above the configurations (127 is the largest the
    library takes): the generic d3_end, the column blocks with few entities
    per block and the 128-level solver variants, 10 steps."""
    abi, cases, model, pyoracle = mods
    def make(lib):
        return cases.estuary_case("small%d" % nsigma, 40, 16, 300.0, nsigma, 2.0, 25.0, stress=(0.0, 0.05), lib=lib)
    bad, _, _ = run_pair(mods, make, 10)
    assert bad == []


def test_estuary_filter2x_bit_exact(mods):
    """viscosity_filt2x_3D and viscosity_filt2x_2D (filt_bi_3D / filt_bi_2D)
    on the small estuary, 30 steps, and on LE, 20 steps."""
    abi, cases, model, pyoracle = mods
    bad, _, _ = run_pair(mods, est(cases, "small", filt_bi_3D=1, filt_bi_2D=1, tau_c=0.4), 30)
    assert bad == []
    bad, _, _ = run_pair(mods, le(cases, filt_bi_3D=1, filt_bi_2D=1), 20)
    assert bad == []


def test_cfg0_bit_exact(mods):
    """The reference's CPU-sized configuration (201 x 81 nodes at 300 m, 11
    sigma levels, MUSCL, wetting/drying, tide, river), 100 internal steps."""
    abi, cases, model, pyoracle = mods
    bad, eg, eo = run_pair(mods, est(cases, "cfg0"), 100)
    assert bad == []
    assert abs(eg - eo) <= 1e-12 * abs(eo)


def test_cfg1_scale_properties(mods):
    """The 1.05M-node, 21-level benchmark mesh: finite state, masks in {0,1},
    bit-identical repeat, and kernel launches counted."""
    abi, cases, model, pyoracle = mods
    case = cases.estuary("cfg1")
    out = []
    for _ in range(2):
        g = model.GpuModel(case)
        g.run(3)
        s = g.state(abi.F_ETA | abi.F_TS | abi.F_MASK | abi.F_UV2D)
        assert g.kernel_launches() > 100
        out.append(s)
        g.close()
    s = out[0]
    for k in ("eta_n", "TF", "SF", "U_n_2D"):
        assert np.all(np.isfinite(s[k]))
        assert np.array_equal(out[0][k], out[1][k])
    assert set(np.unique(s["mask_wd"])) <= {0.0, 1.0}


def _atm_varied(mesh):
    """Shortwave, non-solar flux, E - P and a sea-level pressure gradient
    that vary over the estuary (seeded)."""
    rng = np.random.default_rng(11)
    x = mesh.coord_nod2D[:, 0] / mesh.coord_nod2D[:, 0].max()
    return {"qsr": 250.0 + 50.0 * rng.random(mesh.N), "qns": -60.0 + 20.0 * x,
            "emp": 2.0e-5 * (x - 0.5), "mslp": 101325.0 + 400.0 * x}


def _atm_per_node(mesh):
    f = _atm_varied(mesh)
    rng = np.random.default_rng(12)
    f.update(Rj=0.58 + 0.2 * rng.random(mesh.N), aj=0.35 + rng.random(mesh.N), bj=5.0 + 20.0 * rng.random(mesh.N))
    return f


@pytest.mark.parametrize("variant", ["cfg4_heat_loss", "jerlov_const", "soloviev", "jerlov_per_node"])
def test_key_atm_bit_exact(mods, variant):
    """Atmospheric forcing (key_atm): the sea-level pressure and E - P in
    the elevation gradient of the sub-cycle and in the surface pressure force
    of the 3D step, and the shortwave / non-solar heat and E - P freshwater
    sources of the tracer column solve, 20 steps on the small estuary, exact.
    cfg4_heat_loss is the learned-closure configuration's -100 W/m2 surface
    heat flux; the others exercise both shortwave profiles and per-node
    Jerlov water types."""
    abi, cases, model, pyoracle = mods
    atm, kw = {
        "cfg4_heat_loss": ({"qns": -100.0, "qsr": 0.0, "emp": 0.0}, {}),
        "jerlov_const": (_atm_varied, {}),
        "soloviev": (_atm_varied, {"type_swr_body": 2}),
        "jerlov_per_node": (_atm_per_node, {"jer_const": 0}),
    }[variant]
    bad, eg, eo = run_pair(mods, est(cases, "small", atm=atm, **kw), 20)
    assert bad == []
    assert abs(eg - eo) <= 1e-12 * abs(eo)


def _estuary21(cases, **kw):
    """the small estuary with 21 sigma levels (cfg1's level count)"""
    return lambda lib: cases.estuary_case("small21", 40, 16, 300.0, 21, 2.0, 25.0, stress=(0.0, 0.05), lib=lib,
                                          **kw)


@pytest.mark.parametrize("variant", ["rivers_split_local", "atm_split_shared", "atm_per_node_split",
                                     "reg6_11", "reg8_11_atm", "reg6_21", "reg8_21", "one_kernel_forms_21",
                                     "tile64_atm_21", "implvisc_direct_21"])
def test_two_kernel_forms_bit_exact(mods, variant):
    """The kernel forms beside the defaults against the oracle: d3_end in
    one kernel and as set-up + sweep (sweep arrays in local memory, in
    shared memory, in registers for 11 and 21 levels), the tracers' vertical
    diffusion with directly read columns and on tiles of 128 or 64 columns
    (10 and 20 layers), the implicit vertical viscosity with directly read
    columns (the tiles are the default), with the river salinity source and
    with atmospheric heat and freshwater sources in the column solve, 20
    steps, exact."""
    abi, cases, model, pyoracle = mods
    make, shapes = {
        "rivers_split_local": (est(cases, "small"), {"d3end_arrays": 3, "vdiff_form": 2}),
        "atm_split_shared": (est(cases, "small", atm=_atm_varied, type_swr_body=2),
                             {"d3end_arrays": 4, "vdiff_form": 2}),
        "atm_per_node_split": (est(cases, "small", atm=_atm_per_node, jer_const=0),
                               {"d3end_arrays": 3, "vdiff_form": 2}),
        "reg6_11": (est(cases, "small"), {"d3end_arrays": 5}),
        "reg8_11_atm": (est(cases, "small", atm=_atm_varied), {"d3end_arrays": 6, "vdiff_form": 2}),
        "reg6_21": (_estuary21(cases), {"d3end_arrays": 5, "vdiff_form": 2}),
        "reg8_21": (_estuary21(cases), {"d3end_arrays": 6}),
        "one_kernel_forms_21": (_estuary21(cases), {"d3end_arrays": 1, "vdiff_form": 1}),
        "tile64_atm_21": (_estuary21(cases, atm=_atm_varied), {"vdiff_form": 3}),
        "implvisc_direct_21": (_estuary21(cases), {"implvisc_form": 1, "vdiff_form": 2}),
    }[variant]
    bad, eg, eo = run_pair(mods, make, 20, shapes)
    assert bad == []
    assert abs(eg - eo) <= 1e-12 * abs(eo)


@pytest.mark.parametrize("net_flux,sfc", [(0, 0), (1, 1)])
def test_device_surface_fluxes_bit_exact(mods, net_flux, sfc):
    """sbc_do on the device (fesomc_gpu_set_atm_fields: the atmospheric
    fields at every step's time, the Large & Yeager bulk formulae of
    apply_atm_fluxes / core_coeff_2z, the stress onto the elements) against
    the oracle's restatement, 20 steps on the small estuary, exact; with the
    longwave as a net flux and the mesh stored along the Hilbert curve in
    the second case."""
    abi, cases, model, pyoracle = mods
    gcase, ocase = build_pair(mods, est(cases, "small", atm={"qns": 0.0}))
    gcase.params.sfc_order = sfc
    a, b = cases.atm_coefficients(gcase.mesh, gcase.params.time_jd0)
    g = model.GpuModel(gcase)
    o = pyoracle.Oracle(ocase, abi, cases)
    try:
        g.set_atm_fields(a, b, net_flux, 1.0)
        o.set_atm_fields(a, b, net_flux, 1.0)
        g.step(20)
        o.step(20)
        assert compare(g.state(), o.state()) == []
        eg, eo = g.energy(), o.energy()
        assert abs(eg - eo) <= 1e-12 * abs(eo)
    finally:
        g.close()
        o.close()


def test_device_surface_fluxes_refused_without_key_atm(mods):
    abi, cases, model, pyoracle = mods
    g = model.GpuModel(cases.estuary("small"))
    try:
        a, b = cases.atm_coefficients(g.case.mesh, g.case.params.time_jd0)
        assert g.lib.fesomc_gpu_set_atm_fields(g.h, abi.dptr(a), abi.dptr(b), 0, 1.0) == 1
    finally:
        g.close()


def test_key_atm_changes_the_run_and_fp32_form_runs(mods):
    """The surface heat loss cools the estuary against the run without it,
    and the FP32 form runs the same forcing (finite, within 0.01 C of FP64)."""
    abi, cases, model, pyoracle = mods
    heat = {"qns": -100.0, "qsr": 0.0, "emp": 0.0}
    out = {}
    for name, atm, fp32 in (("off", None, 0), ("on", heat, 0), ("on32", heat, 1)):
        c = cases.estuary("small", atm=atm)
        c.params.fp32_form = fp32
        g = model.GpuModel(c)
        g.step(20)
        out[name] = g.state()
        g.close()
    wet = out["on"]["mask_wd_node"] > 0
    L = c.mesh.L
    top = lambda s: s["TF"].reshape(-1, L)[wet, 0]
    assert np.mean(top(out["on"]) - top(out["off"])) < -1e-4
    assert np.all(np.isfinite(out["on32"]["TF"]))
    assert np.max(np.abs(out["on32"]["TF"] - out["on"]["TF"])) < 0.01


def test_key_atm_per_node_water_types_required(mods):
    """With jer_const = 0 the per-node Rj, aj, bj must come with the forcing
    before the first step (FESOMC_ESTATE otherwise)."""
    abi, cases, model, pyoracle = mods
    c = cases.estuary("small", atm={"qns": -100.0}, jer_const=0)
    g = model.GpuModel(c)
    try:
        assert g.step(1, check=False) == 4
    finally:
        g.close()


@pytest.mark.parametrize("shuffle", [None, 5])
def test_sfc_storage_order_bit_exact(mods, shuffle):
    """Nodes, elements and edges stored along a Hilbert curve (sfc_order = 1)
    give the oracle's bits, on the estuary as generated (row by row) and with
    its nodes and elements numbered at random (a mesh in file order); the
    oracle runs in the reference numbering of the same mesh."""
    abi, cases, model, pyoracle = mods
    bad, eg, eo = run_pair(mods, est(cases, "small", shuffle=shuffle, sfc_order=1), 30)
    assert bad == []
    assert abs(eg - eo) <= 1e-12 * abs(eo)
    if shuffle is not None:
        bad, _, _ = run_pair(mods, est(cases, "small", shuffle=shuffle), 30)
        assert bad == []


def test_sfc_storage_order_le_potential_snapshot_fp32(mods):
    """Storage order on LE (spherical), with the tidal potential and device
    forcing, through the asynchronous snapshot, and in the FP32 form (which
    gives the same bits in both orders)."""
    abi, cases, model, pyoracle = mods
    bad, _, _ = run_pair(mods, le(cases, sfc_order=1), 20)
    assert bad == []
    out = []
    for sfc in (0, 1):
        case = cases.estuary("small", T_potential=1, sfc_order=sfc)
        case.params.fp32_form = 1
        g = model.GpuModel(case)
        g.set_forcing(case.forcing_fn(1, cases.advance_time(g.time_jd, case.params.dt)))
        base = np.ascontiguousarray(case.forcing_fn(1, case.params.time_jd0 + 20.0)["runoff_rivers"])
        abi.check(g.lib.fesomc_gpu_set_device_forcing(g.h, abi.dptr(base), 1))
        g.run(15)
        g.snapshot_begin()
        snap = g.snapshot_end()
        st = g.state()
        g.close()
        for f in FIELDS:
            assert np.array_equal(snap[f], st[f]), f
        out.append(st)
    for f in FIELDS:
        assert np.array_equal(out[0][f], out[1][f]), f
