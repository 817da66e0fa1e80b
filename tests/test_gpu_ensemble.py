"""fesomc_ensemble_run: members of different sizes and precision forms
advanced concurrently on one GPU give the same bits as each member advanced
alone, and the timed form reports a device time."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ["eta_n", "U_n_2D", "U_n", "V_n", "TF", "SF", "Wvel", "Kv", "mask_wd_node"]
NODES = (600, 4000)
STEPS = 12


def _members():
    from fesomc import cases
    out = []
    for i in range(4):
        c = cases.ensemble_member(i, nodes_range=NODES)
        c.params.fp32_form = i % 2
        out.append(c)
    return out


def _alone(case, steps):
    from fesomc import abi, cases, model
    g = model.GpuModel(case)
    try:
        g.set_forcing(case.forcing_fn(1, cases.advance_time(g.time_jd, case.params.dt)))
        base = np.ascontiguousarray(case.forcing_fn(1, case.params.time_jd0 + 20.0)["runoff_rivers"])
        abi.check(g.lib.fesomc_gpu_set_device_forcing(g.h, abi.dptr(base), 1), "fesomc_gpu_set_device_forcing")
        abi.check(g.lib.fesomc_gpu_run(g.h, 0, steps), "fesomc_gpu_run")
        return g.state()
    finally:
        g.close()


def test_concurrent_members_match_members_alone(built):
    from fesomc import ensemble
    members = _members()
    ens = ensemble.Ensemble(members)
    try:
        ms, status = ens.run(STEPS // 2, timed=True)
        assert ms > 0.0 and status == [0] * len(members)
        _, status = ens.run(STEPS - STEPS // 2)
        assert status == [0] * len(members)
        got = [ens.member(i).state() for i in range(len(members))]
    finally:
        ens.close()
    for i, c in enumerate(_members()):
        ref = _alone(c, STEPS)
        for f in FIELDS:
            assert np.array_equal(got[i][f], ref[f]), (i, f)


def test_ensemble_rejects_bad_arguments(built):
    from fesomc import abi, ensemble
    lib = abi.load()
    members = _members()[:1]
    ens = ensemble.Ensemble(members)
    try:
        h = ens._handles
        assert lib.fesomc_ensemble_run(h, 0, 1, None, None) == 1
        assert lib.fesomc_ensemble_run(h, 1, -1, None, None) == 1
        dup = (C.c_void_p * 2)(h[0], h[0])
        assert lib.fesomc_ensemble_run(dup, 2, 1, None, None) == 1
    finally:
        ens.close()
