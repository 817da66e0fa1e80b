"""Forcing on the device (fesomc_gpu_set_device_forcing): the open-boundary
tide and the ramped river runoff evaluated by the forcing kernels give the
same bits as the host path, which computes them per step and uploads them,
in both precision forms."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STEPS = 40
FIELDS = ["eta_n", "eta_n_1", "etaAB", "U_n_2D", "U_n", "V_n", "TF", "SF", "Wvel", "Kv", "mask_wd_node",
          "ssh_gp"]


@pytest.mark.parametrize("fp32,potential", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_device_forcing_matches_host_forcing(built, fp32, potential):
    """With T_potential the potential kernel reads the device clock, which
    the host path uploads each step and device forcing advances itself."""
    from fesomc import abi, cases, model
    case = cases.estuary("small", T_potential=potential)
    case.params.fp32_form = fp32
    # host path: the forcing of every step pushed from the host
    g = model.GpuModel(case)
    try:
        g.step(STEPS)
        ref = g.state()
    finally:
        g.close()
    # device path: stress and harmonics pushed once, then the device
    # evaluates tide and runoff itself
    g = model.GpuModel(case)
    try:
        g.set_forcing(case.forcing_fn(1, cases.advance_time(g.time_jd, case.params.dt)))
        base = np.ascontiguousarray(case.forcing_fn(1, case.params.time_jd0 + 20.0)["runoff_rivers"])
        assert base.max() > 0.0
        abi.check(g.lib.fesomc_gpu_set_device_forcing(g.h, abi.dptr(base), 1), "fesomc_gpu_set_device_forcing")
        abi.check(g.lib.fesomc_gpu_run(g.h, 0, STEPS // 2), "fesomc_gpu_run")
        abi.check(g.lib.fesomc_gpu_run(g.h, 0, STEPS - STEPS // 2), "fesomc_gpu_run")
        got = g.state()
    finally:
        g.close()
    assert got["_time_jd"] == ref["_time_jd"]
    for f in FIELDS:
        assert np.array_equal(got[f], ref[f]), f


@pytest.mark.parametrize("potential", [0, 1])
def test_device_forcing_matches_oracle(built, potential):
    """The forcing kernels (open-boundary tide of every sub-step, ramped river
    runoff, and with T_potential the equilibrium tide) against the oracle,
    which evaluates the same forcing on the host each step from the case's
    forcing routines (rivers_do / obc harmonics, oracle_set_forcing); the
    oracle runs on its own mesh restatement.  Exact."""
    import pyoracle
    from fesomc import abi, cases, model
    case = cases.estuary("small", T_potential=potential)
    ocase = cases.estuary("small", T_potential=potential, lib=pyoracle.MeshLib(abi))
    g = model.GpuModel(case)
    o = pyoracle.Oracle(ocase, abi, cases)
    try:
        g.set_forcing(case.forcing_fn(1, cases.advance_time(g.time_jd, case.params.dt)))
        base = np.ascontiguousarray(case.forcing_fn(1, case.params.time_jd0 + 20.0)["runoff_rivers"])
        abi.check(g.lib.fesomc_gpu_set_device_forcing(g.h, abi.dptr(base), 1), "fesomc_gpu_set_device_forcing")
        abi.check(g.lib.fesomc_gpu_run(g.h, 0, STEPS), "fesomc_gpu_run")
        got = g.state()
        assert o.step(STEPS) == 0
        ref = o.state()
    finally:
        g.close()
        o.close()
    assert got["_time_jd"] == ref["_time_jd"]
    if potential:
        assert np.abs(ref["ssh_gp"]).max() > 0.0
    for f in FIELDS:
        assert np.array_equal(got[f], ref[f]), f


def test_device_forcing_needs_river_base(built):
    from fesomc import cases, model
    case = cases.estuary("small")
    g = model.GpuModel(case)
    try:
        assert g.lib.fesomc_gpu_set_device_forcing(g.h, None, 1) == 1
        assert g.lib.fesomc_gpu_set_device_forcing(None, None, 0) == 1
    finally:
        g.close()


def test_restart_with_device_forcing_and_potential(built):
    """A restart into a fresh model on device forcing with the tidal
    potential: the device clock follows the restart time, and the run
    continues bit for bit."""
    from fesomc import abi, cases, model
    case = cases.estuary("small", T_potential=1)
    base = np.ascontiguousarray(case.forcing_fn(1, case.params.time_jd0 + 20.0)["runoff_rivers"])
    a = model.GpuModel(case)
    c = model.GpuModel(case)
    try:
        for g in (a, c):
            g.set_forcing(case.forcing_fn(1, cases.advance_time(g.time_jd, case.params.dt)))
            abi.check(g.lib.fesomc_gpu_set_device_forcing(g.h, abi.dptr(base), 1), "fesomc_gpu_set_device_forcing")
        abi.check(a.lib.fesomc_gpu_run(a.h, 0, 10), "fesomc_gpu_run")
        snap = a.state()
        abi.check(a.lib.fesomc_gpu_run(a.h, 0, 10), "fesomc_gpu_run")
        ref = a.state()
        arrays = {k: v for k, v in snap.items() if k != "_time_jd"}
        st = case.state_struct(arrays, snap["_time_jd"], lfirst=0)
        abi.check(c.lib.fesomc_gpu_sync_from_host(c.h, abi.F_ALL, C.byref(st)), "sync_from_host")
        abi.check(c.lib.fesomc_gpu_run(c.h, 0, 10), "fesomc_gpu_run")
        got = c.state()
    finally:
        a.close()
        c.close()
    assert got["_time_jd"] == ref["_time_jd"]
    for f in FIELDS:
        assert np.array_equal(got[f], ref[f]), f
