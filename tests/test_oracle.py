"""CPU oracle: pinned against the reference's golden energy series and
checked for conservation on the CPU (no GPU)."""
import math

import numpy as np
import pytest


def half_unit_e16_7(v):
    """Half a unit in the last digit of Fortran format e16.7 (0.dddddddE+xx)."""
    return 0.5 * 10.0 ** (math.floor(math.log10(abs(v))) + 1 - 7)


class _OracleCases:
    """cases.* with the oracle's own mesh restatement as the builder, so that
    nothing in these tests goes through the product library."""

    def __init__(self, cases, lib):
        self._c, self._lib = cases, lib

    def le_medium(self, **kw):
        return self._c.le_medium(lib=self._lib, **kw)

    def estuary(self, *a, **kw):
        return self._c.estuary(*a, lib=self._lib, **kw)

    def __getattr__(self, k):
        return getattr(self._c, k)


@pytest.fixture(scope="module")
def mods():
    import pyoracle
    from fesomc import abi, cases
    pyoracle.build()
    return abi, _OracleCases(cases, pyoracle.MeshLib(abi)), pyoracle


# rows of the golden series checked here (100 steps each, about a second of
# oracle time per row); the GPU suite checks the oracle and the GPU further on
GOLDEN_ROWS_CPU = 30


def test_mt_from_ieee_division():
    # Mt = int(dt/dt_2D) (fv_read_run.F90:1060) is 5 for dt=0.5, dt_2D=0.1 in
    # IEEE double arithmetic; the golden LE series corresponds to 4 sub-steps
    assert int(0.5 / 0.1) == 5


def test_le_energy_matches_reference_golden(mods):
    """energy_tocheck.dat of test_cases/LE_medium, printed with 7 significant
    digits every 100 steps; reproduced with Mt = 4 sub-steps."""
    abi, cases, pyoracle = mods
    case = cases.le_medium()
    case.params.Mt = 4
    gold = case.meta["energy"]
    o = pyoracle.Oracle(case, abi, cases)
    for row in range(GOLDEN_ROWS_CPU):
        o.step(100)
        days = o.time_jd - case.params.time_jd0
        # the day column identifies the row (time_jd accumulates dt/86400 on
        # top of JD0, so its last printed digits carry that round-off); the
        # energy is printed as 0.dddddddE+xx and must round to the printed value
        assert abs(days - gold[row, 0]) < 1e-6 * gold[row, 0], row
        assert abs(o.energy() - gold[row, 1]) <= half_unit_e16_7(gold[row, 1]), row
    o.close()


def test_le_energy_with_five_substeps_differs(mods):
    abi, cases, pyoracle = mods
    case = cases.le_medium()
    assert case.params.Mt == 5
    o = pyoracle.Oracle(case, abi, cases)
    o.step(100)
    assert o.energy() / case.meta["energy"][0, 1] > 1.2
    o.close()


def test_le_volume_conserved(mods):
    abi, cases, pyoracle = mods
    case = cases.le_medium()
    area = case.mesh.area
    o = pyoracle.Oracle(case, abi, cases)
    v0 = np.sum(area * (case.mesh.depth + o.state()["eta_n"]))
    o.step(40)
    v1 = np.sum(area * (case.mesh.depth + o.state()["eta_n"]))
    assert abs(v1 - v0) / v0 < 1e-13
    o.close()


def test_estuary_small_stable(mods):
    abi, cases, pyoracle = mods
    case = cases.estuary("small")
    o = pyoracle.Oracle(case, abi, cases)
    rc = o.step(30)
    s = o.state()
    assert rc == 0
    for k in ("eta_n", "U_n", "TF", "SF", "snu"):
        assert np.all(np.isfinite(s[k]))
    assert set(np.unique(s["mask_wd"])) <= {0.0, 1.0}
    assert (s["mask_wd"] == 0).sum() > 0          # wetting/drying active
    assert 0 < s["snu"].min() and s["snu"].max() <= 0.2
    o.close()


def test_estuary_miura_oracle_advects_temperature_only(mods):
    """tracer_adv = 4 advances T with the Miura scheme and leaves S to the
    river source and vertical diffusion (fv_main.F90:1790-1799)."""
    abi, cases, pyoracle = mods
    case = cases.estuary("small", tracer_adv=abi.TRACER_MIURA, key_rivers=0)
    o = pyoracle.Oracle(case, abi, cases)
    s0 = o.state()
    rc = o.step(10)
    s = o.state()
    assert rc == 0
    assert np.all(np.isfinite(s["TF"]))
    assert not np.array_equal(s["TF"], s0["TF"])
    # without rivers, S only diffuses vertically: column means are kept
    L = case.mesh.L
    m0 = s0["SF"].reshape(-1, L).mean(axis=1)
    m1 = s["SF"].reshape(-1, L).mean(axis=1)
    assert np.max(np.abs(m1 - m0)) < 0.05
    o.close()


def test_estuary_oracle_negative_salinity_flag(mods):
    """A river source of absurdly negative salinity (injected on the host)
    drives salinity below zero; the check of fv_tracer.F90:1469-1473 (which
    stops the reference) is reported through the status word."""
    abi, cases, pyoracle = mods
    case = cases.estuary("small", river_salinity=-1.0e9)
    o = pyoracle.Oracle(case, abi, cases)
    rc = o.step(1)
    assert rc & abi.ST_NEGSALT
    o.close()


def test_estuary_oracle_low_temperature_flag(mods):
    abi, cases, pyoracle = mods
    case = cases.estuary("small")
    L = case.mesh.L
    case.state0["TF"][L * 7: L * 9] = -10.0
    case.state0["T_old"][L * 7: L * 9] = -10.0
    o = pyoracle.Oracle(case, abi, cases)
    rc = o.step(1)
    assert rc & abi.ST_LOWTEMP
    o.close()


def test_shared_log_within_one_ulp_of_libm(mods):
    """fesomc_log (the IEEE-only logarithm of d3_end's bottom boundary value,
    shared by the oracle and the device kernels) against the C library's log:
    at most one ulp apart, over the closure's argument range and beyond."""
    abi, cases, pyoracle = mods
    lib = pyoracle.load(abi)
    rng = np.random.default_rng(5)
    xs = np.concatenate([np.exp(rng.uniform(-700.0, 700.0, 20000)),    # whole range
                         1.0 + rng.uniform(-0.3, 0.3, 20000),          # near 1
                         1.0 + rng.uniform(0.0, 2000.0, 20000),        # delta_b / z0b_min
                         [1.0, 2.0, 0.5, 5e-324, 1e-310, 1.7976931348623157e308,
                          np.nextafter(1.0, 2.0), np.nextafter(1.0, 0.0)]])
    ours = np.array([lib.oracle_log(float(x)) for x in xs])
    ref = np.array([math.log(float(x)) for x in xs])
    ulps = np.abs(ours.view(np.int64) - ref.view(np.int64))
    assert ulps.max() <= 1
    assert np.mean(ulps != 0) < 0.01
    assert lib.oracle_log(1.0) == 0.0
    assert lib.oracle_log(0.0) == -math.inf
    assert math.isnan(lib.oracle_log(-1.0)) and math.isnan(lib.oracle_log(math.nan))
    assert lib.oracle_log(math.inf) == math.inf


def test_shared_cos_within_one_ulp_of_libm(mods):
    """fesomc_cos (the IEEE-only cosine of the harmonic open-boundary
    elevation, shared by the oracle, the host forcing path and the device
    forcing kernel) against the C library's cos: at most one ulp apart over
    the phases a tide reaches, NaN beyond its range."""
    abi, cases, pyoracle = mods
    lib = pyoracle.load(abi)
    rng = np.random.default_rng(7)
    xs = np.concatenate([rng.uniform(-1000.0, 1000.0, 20000), rng.uniform(-4.0, 4.0, 20000),
                         rng.uniform(-1.5e6, 1.5e6, 5000), [0.0, 1e-300, math.pi / 2, math.pi, -math.pi]])
    ours = np.array([lib.oracle_cos(float(x)) for x in xs])
    ref = np.array([math.cos(float(x)) for x in xs])
    ulps = np.abs(ours.view(np.int64) - ref.view(np.int64))
    # near a zero of cos an ulp of the result is tiny: compare those absolutely
    ok = (ulps <= 1) | (np.abs(ours - ref) <= 2.3e-16)
    assert ok.all()
    assert np.mean(ulps != 0) < 0.1
    assert lib.oracle_cos(0.0) == 1.0
    assert math.isnan(lib.oracle_cos(2e6)) and math.isnan(lib.oracle_cos(math.inf))


def test_shared_atan_within_four_ulp_of_libm(mods):
    """fesomc_atan (psi_m of the bulk transfer coefficients, shared by the
    oracle and the device surface-flux kernel) against the C library's
    atan: at most 4 ulp apart over 12 decades of argument, exact at the
    reduction points."""
    abi, cases, pyoracle = mods
    lib = pyoracle.load(abi)
    rng = np.random.default_rng(11)
    xs = np.concatenate([rng.uniform(-4.0, 4.0, 20000), np.exp(rng.uniform(-14.0, 14.0, 20000)),
                         -np.exp(rng.uniform(-14.0, 14.0, 5000)), [0.0, 1.0, -1.0, 1e-300, 1e300]])
    ours = np.array([lib.oracle_atan(float(x)) for x in xs])
    ref = np.array([math.atan(float(x)) for x in xs])
    ulps = np.abs(ours.view(np.int64) - ref.view(np.int64))
    assert ulps.max() <= 4
    assert lib.oracle_atan(1.0) == math.atan(1.0) and lib.oracle_atan(0.0) == 0.0
    assert lib.oracle_atan(math.inf) == math.pi / 2 and math.isnan(lib.oracle_atan(math.nan))


def test_bulk_surface_fluxes_in_range(mods):
    """The oracle's sbc_do (bulk formulae of apply_atm_fluxes and
    core_coeff_2z, src/fv_sbc.F90:368-662): with 6-10 m/s winds over a
    12 C sea, the stress is of order rho_a Cd U^2 (Cd about 1.2e-3), it
    points along the wind, the sea loses heat to the colder, drier air
    through evaporation and sensible heat, and E - P is evaporation less
    precipitation."""
    abi, cases, pyoracle = mods
    c = cases.estuary("small", atm={"qns": 0.0})
    o = pyoracle.Oracle(c, abi, cases)
    try:
        a, b = cases.atm_coefficients(c.mesh, c.params.time_jd0)
        o.set_atm_fields(a, b, net_flux=0, prec_coef=1.0)
        o.step(1)
        t = o.time_jd
        atm = (t * a + b).reshape(-1, 8)
        wx = o.array("windx")
        assert np.array_equal(wx, atm[:, 0])
        tx, ty = o.array("taux"), o.array("tauy")
        speed2 = (atm[:, 0] ** 2 + atm[:, 1] ** 2).mean()
        assert 0.5e-3 < np.abs(tx).mean() / (1.3 * speed2 ** 0.5 * np.abs(atm[:, 0]).mean()) < 3e-3
        assert (tx > 0).all() and (ty < 0).mean() > 0.5
        qns = o.array("qns")
        assert np.isfinite(qns).all() and (qns < 0).all()
        emp = o.array("emp")
        assert (emp > -atm[:, 6]).all()          # evaporation over the drier air
        assert np.allclose(o.array("qsr"), (1.0 - float(np.float32(0.1))) * atm[:, 3])
        assert np.array_equal(o.array("mslp"), atm[:, 7])
    finally:
        o.close()


def test_shared_sin_within_one_ulp_of_libm(mods):
    """fesomc_sin (the equilibrium tide of the tidal potential) against the C
    library's sin, as the cosine above."""
    abi, cases, pyoracle = mods
    lib = pyoracle.load(abi)
    rng = np.random.default_rng(8)
    xs = np.concatenate([rng.uniform(-4.0, 4.0, 20000), rng.uniform(-1000.0, 1000.0, 10000),
                         [0.0, 1e-300, -1e-300, math.pi / 2, math.pi, 0.5 * 3.14159265358979]])
    ours = np.array([lib.oracle_sin(float(x)) for x in xs])
    ref = np.array([math.sin(float(x)) for x in xs])
    ulps = np.abs(ours.view(np.int64) - ref.view(np.int64))
    ok = (ulps <= 1) | (np.abs(ours - ref) <= 2.3e-16)
    assert ok.all()
    assert lib.oracle_sin(0.0) == 0.0 and lib.oracle_sin(1e-300) == 1e-300
    assert math.isnan(lib.oracle_sin(2e6))


def potential_numpy(time_jd, time_jd0, coord, ath):
    """potential (fv_tide_potential.F90:1-107) in numpy with the C library's
    sine and cosine: an independent restatement that pins the oracle's."""
    pi = 3.14159265358979
    rad = pi / 180.0
    Apt = np.array([0.242334, 0.112841, 0.046398, 0.030704, 0.141565, 0.100514, 0.046843, 0.019256,
                    0.041742, 0.022026, 0.019446])
    Fpt = np.array([1.40519e-4, 1.45444e-4, 1.37880e-4, 1.45842e-4, 0.72921e-4, 0.67598e-4, 0.72523e-4,
                    0.64959e-4, 0.53234e-5, 0.26392e-5, 0.03982e-5])

    def c360(fr):
        iz = int(fr / 360.0)
        return fr - iz * 360.0 if iz >= 1 else fr

    DY = time_jd - 2442413.5
    TY = (27392.500528 + 1.0000000356 * DY) / 36525.0
    h0 = c360(279.69668 + 36000.768930485 * TY + 3.03e-4 * TY ** 2)
    s0 = c360(270.434358 + 481267.88314137 * TY - 0.001133 * TY ** 2 + 1.9e-6 * TY ** 3)
    p0 = c360(334.329653 + 4069.0340329575 * TY - 0.010325 * TY ** 2 - 1.2e-5 * TY ** 3)
    sxi = np.array([(h0 - s0) * 2 * rad, 0.0, (2 * h0 - 3 * s0 + p0) * rad, 2 * h0 * rad, (h0 + 90) * rad,
                    (h0 - 2 * s0 - 90) * rad, (h0 - 90) * rad, (h0 - 3 * s0 + p0 - 90) * rad, 2 * s0 * rad,
                    (s0 - p0) * rad, 2 * h0 * rad])
    lon, lat = coord[:, 0], coord[:, 1]
    colat = 0.5 * pi - lat
    out = np.zeros(len(lon))
    for j in range(11):
        arg_t = Fpt[j] * (DY * 86400.0 - sxi[j] / Fpt[j]) + sxi[j]
        if j < 4:
            out += ath[j] * Apt[j] * np.sin(colat) ** 2 * np.cos(arg_t + 2 * lon)
        elif j < 8:
            out += ath[j] * Apt[j] * np.sin(2 * colat) * np.cos(arg_t + lon)
        else:
            out += ath[j] * Apt[j] * (3 * np.sin(colat) ** 2 - 2) * np.cos(arg_t)
    if time_jd - time_jd0 < 5.0:
        out = out * (time_jd - time_jd0) / 5.0
    return out


def test_tidal_potential_oracle(mods):
    """T_potential: the oracle's ssh_gp after a step equals the numpy
    restatement to rounding (the two use different sines and cosines), with
    all 11 harmonics and with M2 alone, and the potential changes the run."""
    abi, cases, pyoracle = mods
    c = cases.estuary("small", T_potential=1)
    c.params.n_harm = 11
    for j in range(11):
        c.params.harm_index[j] = j
    coord = c.mesh.arr("coord_nod2D", (c.mesh.N, 2)).copy()
    o = pyoracle.Oracle(c, abi, cases)
    o.step(3)
    s = o.state()
    o.close()
    ref = potential_numpy(o.time_jd, c.params.time_jd0, coord, np.ones(11))
    assert np.abs(ref).max() > 0.0
    assert np.allclose(s["ssh_gp"], ref, rtol=0.0, atol=1e-12 * np.abs(ref).max())
    # only the listed harmonics
    c1 = cases.estuary("small", T_potential=1)
    o = pyoracle.Oracle(c1, abi, cases)
    o.step(3)
    s1 = o.state()
    o.close()
    ath = np.zeros(11)
    ath[0] = 1.0
    ref1 = potential_numpy(o.time_jd, c1.params.time_jd0, coord, ath)
    assert np.allclose(s1["ssh_gp"], ref1, rtol=0.0, atol=1e-12 * np.abs(ref1).max())
    c0 = cases.estuary("small")
    o = pyoracle.Oracle(c0, abi, cases)
    o.step(3)
    s0 = o.state()
    o.close()
    assert not np.array_equal(s0["U_n_2D"], s1["U_n_2D"])
    assert np.all(s0["ssh_gp"] == 0.0)


def test_estuary_biharmonic_oracle(mods):
    """biharmonic_viscosity (bih_3D): active, finite, and linear in Abh0 for
    a small viscosity (the damping of a fixed flow field doubles with it)."""
    abi, cases, pyoracle = mods
    out = {}
    for ab in (0.0, 1e3, 1e4):
        c = cases.estuary("small", bih_3D=1 if ab else 0, Abh0=ab if ab else 1000.0)
        o = pyoracle.Oracle(c, abi, cases)
        o.step(30)
        out[ab] = o.state()
        o.close()
    d3 = np.abs(out[1e3]["U_n"] - out[0.0]["U_n"]).max()
    d4 = np.abs(out[1e4]["U_n"] - out[0.0]["U_n"]).max()
    assert np.isfinite(out[1e4]["U_n"]).all()
    assert d3 > 0.0
    assert 5.0 < d4 / d3 < 15.0


def test_estuary_biharmonic_2d_oracle(mods):
    """biharmonic_2D (bih_2D): changes the barotropic velocity, stays finite,
    and its effect grows with Abh0."""
    abi, cases, pyoracle = mods
    out = {}
    for ab in (0.0, 1e3, 1e4):
        c = cases.estuary("small", bih_2D=1 if ab else 0, Abh0=ab if ab else 1000.0)
        o = pyoracle.Oracle(c, abi, cases)
        o.step(20)
        out[ab] = o.state()
        o.close()
    d3 = np.abs(out[1e3]["U_n_2D"] - out[0.0]["U_n_2D"]).max()
    d4 = np.abs(out[1e4]["U_n_2D"] - out[0.0]["U_n_2D"]).max()
    assert np.isfinite(out[1e4]["U_n_2D"]).all() and np.isfinite(out[1e4]["eta_n"]).all()
    assert 0.0 < d3 < d4


def test_estuary_filter2x_oracle(mods):
    """viscosity_filt2x_3D / _2D: each switch changes the run, which stays
    finite."""
    abi, cases, pyoracle = mods
    out = {}
    for key, kw in (("none", {}), ("3d", {"filt_bi_3D": 1}), ("2d", {"filt_bi_2D": 1})):
        c = cases.estuary("small", tau_c=0.4, **kw)
        o = pyoracle.Oracle(c, abi, cases)
        o.step(20)
        out[key] = o.state()
        o.close()
    for key in ("3d", "2d"):
        assert np.isfinite(out[key]["U_n"]).all()
        assert not np.array_equal(out[key]["U_n"], out["none"]["U_n"])


def test_shared_exp_within_one_ulp_of_libm(mods):
    """fesomc_exp (the IEEE-only exponential of the shortwave absorption
    profiles, shared by the oracle and the device kernels) against the C
    library's exp: at most one ulp apart over the normal range; subnormal
    results and the over/underflow ends included."""
    abi, cases, pyoracle = mods
    lib = pyoracle.load(abi)
    rng = np.random.default_rng(6)
    xs = np.concatenate([rng.uniform(-700.0, 700.0, 20000),         # whole normal range
                         rng.uniform(-60.0, 0.0, 20000),            # z / a of the profiles
                         rng.uniform(-1e-3, 1e-3, 5000),
                         [0.0, -0.0, 1.0, -1.0, 709.78, -708.3, 1e-300, -1e-300]])
    ours = np.array([lib.oracle_exp(float(x)) for x in xs])
    ref = np.array([math.exp(float(x)) for x in xs])
    ulps = np.abs(ours.view(np.int64) - ref.view(np.int64))
    assert ulps.max() <= 1
    assert np.mean(ulps != 0) < 0.1
    assert lib.oracle_exp(0.0) == 1.0
    for x in (-710.0, -720.0, -740.0):
        assert abs(lib.oracle_exp(x) - math.exp(x)) <= 2 * 5e-324 + 2e-16 * math.exp(x)
    assert lib.oracle_exp(-800.0) == 0.0 and lib.oracle_exp(800.0) == math.inf
    assert math.isnan(lib.oracle_exp(math.nan))


def test_sw_cp_unesco_check_value(mods):
    """sw_cp (fv_tracer.F90:1775-1908) against the UNESCO 1983 check value
    (Fofonoff and Millard, Unesco Tech. Pap. Mar. Sci. 44): cp = 3849.500
    J/(kg K) at S = 40, T68 = 40 C, p = 10000 dbar (1000 bar, the routine's
    unit); and pure water at the surface at 0 C: the polynomial's 4217.4."""
    abi, cases, pyoracle = mods
    lib = pyoracle.load(abi)
    assert abs(lib.oracle_sw_cp(40.0, 40.0 / 1.00024, 1000.0) - 3849.500) < 0.01
    assert abs(lib.oracle_sw_cp(0.0, 0.0, 0.0) - 4217.4) < 1e-9
    # the routine clamps negative temperature and salinity to zero
    assert lib.oracle_sw_cp(-1.0, -2.0, 0.0) == lib.oracle_sw_cp(0.0, 0.0, 0.0)


def test_surface_heat_flux_cools_the_top_layer(mods):
    """key_atm with a -100 W/m2 non-solar flux (the learned-closure forcing):
    after one step the wet top layer is cooler than in the same run with a
    zero flux, by up to dt * qns / (rho c_p Jc) (the heat source of the top
    layer, fv_tracer.F90:1686-1690, spread down by the implicit diffusion),
    and the domain heat content drops by about dt * qns * wet area / (rho
    c_p)."""
    abi, cases, pyoracle = mods
    runs = []
    for qns in (0.0, -100.0):
        c = cases.estuary("small", atm={"qns": qns, "qsr": 0.0, "emp": 0.0})
        o = pyoracle.Oracle(c, abi, cases)
        o.step(1)
        runs.append((c, o.state()))
        o.close()
    (c, s0), (_, s1) = runs
    m, L, dt = c.mesh, c.mesh.L, c.params.dt
    T0 = s0["TF"].reshape(m.N, L)
    T1 = s1["TF"].reshape(m.N, L)
    wet = s0["mask_wd_node"] > 0
    dT = T1 - T0
    assert np.all(dT[wet, 0] < 0.0)
    H = np.maximum(m.depth + s0["eta_n"], c.params.Dmin)
    jc = H * (m.sigma[0] - m.sigma[1])
    rho_cp = 1025.0 * 3990.0
    expect = dt * (-100.0) / (rho_cp * jc)
    ratio = dT[wet, 0] / expect[wet]
    assert np.median(ratio) > 0.3 and ratio.max() < 1.1
    heat = np.sum(m.area[wet, None] * (dT[wet] * (H[wet, None] * (m.sigma[:-1] - m.sigma[1:])[None, :])))
    assert abs(heat / (dt * -100.0 * m.area[wet].sum() / rho_cp) - 1.0) < 0.05
