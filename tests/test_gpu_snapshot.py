"""Asynchronous output (fesomc_gpu_snapshot_begin / _end): the snapshot holds
the state at the moment it was begun, bit for bit, while the model keeps
stepping, and taking it does not disturb the run; in both precision forms."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ["eta_n", "U_n_2D", "U_filt_2D", "U_n", "V_n", "TF", "SF", "T_old", "bt", "Kv", "Wvel", "mask_wd",
          "rho_c", "Bar_pr_2D"]


@pytest.mark.parametrize("fp32", [0, 1])
def test_snapshot_is_the_state_when_begun(built, fp32):
    from fesomc import abi, cases, model
    case = cases.estuary("small")
    case.params.fp32_form = fp32
    a = model.GpuModel(case)
    b = model.GpuModel(case)
    try:
        a.step(10)
        a.snapshot_begin(abi.F_ALL)
        a.step(5)                     # stepping goes on while the copy runs
        snap = a.snapshot_end()
        b.step(10)
        ref = b.state()
        assert snap["_time_jd"] == ref["_time_jd"]
        for f in FIELDS:
            assert np.array_equal(snap[f], ref[f]), f
        b.step(5)
        after_a, after_b = a.state(), b.state()
        for f in FIELDS:
            assert np.array_equal(after_a[f], after_b[f]), f
    finally:
        a.close()
        b.close()


@pytest.mark.parametrize("fp32", [0, 1])
def test_restart_from_snapshot_is_bit_exact(built, fp32):
    """The restart path (write_restart_separate / a restart read): a full
    snapshot taken while the run goes on, loaded into a fresh model, which
    then continues exactly as the original run."""
    import ctypes as C
    from fesomc import abi, cases, model
    case = cases.estuary("small")
    case.params.fp32_form = fp32
    a = model.GpuModel(case)
    c = model.GpuModel(case)
    try:
        a.step(10)
        a.snapshot_begin(abi.F_ALL)
        a.step(10)
        snap = a.snapshot_end()
        ref = a.state()
        arrays = {k: v for k, v in snap.items() if k != "_time_jd"}
        st = case.state_struct(arrays, snap["_time_jd"], lfirst=0)
        abi.check(c.lib.fesomc_gpu_sync_from_host(c.h, abi.F_ALL, C.byref(st)), "sync_from_host")
        c.nstep, c.time_jd = 10, snap["_time_jd"]
        c.step(10)
        got = c.state()
        assert got["_time_jd"] == ref["_time_jd"]
        for f in FIELDS:
            assert np.array_equal(got[f], ref[f]), f
    finally:
        a.close()
        c.close()


def test_snapshot_order_is_checked(built):
    from fesomc import abi, cases, model
    case = cases.estuary("small")
    g = model.GpuModel(case)
    try:
        assert g.lib.fesomc_gpu_snapshot_end(g.h) == 4                # none pending
        g.snapshot_begin(abi.F_ETA)
        arrays, st = g._snap
        assert g.lib.fesomc_gpu_snapshot_begin(g.h, abi.F_ETA, st) == 4  # one at a time
        snap = g.snapshot_end()
        assert np.array_equal(snap["eta_n"], g.state(abi.F_ETA)["eta_n"])
    finally:
        g.close()
