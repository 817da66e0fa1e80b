"""Packed members (fesomc_gpu_init_packed): every member of a packed model
advances bit for bit as it does alone, in both precision forms and both
storage orders, with host forcing per step and with forcing on the device;
the packed ensemble reports per-member states and statuses."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NODES = (600, 4000)


def _members(n, nsigma, fp32=0, sfc=0):
    from fesomc import cases
    out, i = [], 0
    while len(out) < n:
        c = cases.ensemble_member(i, nodes_range=NODES)
        i += 1
        if c.mesh.NS == nsigma:
            c.params.fp32_form = fp32
            c.params.sfc_order = sfc
            out.append(c)
    return out


def _assert_same(got, ref, tag):
    for f, v in ref.items():
        if f.startswith("_"):
            continue
        assert np.array_equal(got[f], v), (tag, f)


@pytest.mark.parametrize("fp32,sfc", [(0, 0), (1, 0), (0, 1)])
def test_packed_members_step_like_members_alone(built, fp32, sfc):
    from fesomc import model, packed
    steps = 6
    pc = packed.PackedCase(_members(3, 21, fp32, sfc))
    g = model.GpuModel(pc)
    try:
        assert g.step(steps) == 0
        parts = pc.split_state(g.state())
    finally:
        g.close()
    for k, c in enumerate(_members(3, 21, fp32, sfc)):
        a = model.GpuModel(c)
        try:
            assert a.step(steps) == 0
            _assert_same(parts[k], a.state(), (fp32, sfc, k))
        finally:
            a.close()


def test_packed_ensemble_on_device_forcing_matches_members_alone(built):
    from fesomc import abi, cases, ensemble, model
    steps = 10
    members = _members(2, 21, 1) + _members(2, 11, 0)
    ens = ensemble.PackedEnsemble(members)
    try:
        assert len(ens.packs) == 2
        ms, status = ens.run(steps, timed=True)
        assert ms > 0.0 and status == [0] * len(members)
        got = [ens.member_state(i) for i in range(len(members))]
    finally:
        ens.close()
    for i, c in enumerate(_members(2, 21, 1) + _members(2, 11, 0)):
        g = model.GpuModel(c)
        try:
            g.set_forcing(c.forcing_fn(1, cases.advance_time(g.time_jd, c.params.dt)))
            base = np.ascontiguousarray(c.forcing_fn(1, c.params.time_jd0 + 20.0)["runoff_rivers"])
            abi.check(g.lib.fesomc_gpu_set_device_forcing(g.h, abi.dptr(base), 1), "fesomc_gpu_set_device_forcing")
            abi.check(g.lib.fesomc_gpu_run(g.h, 0, steps), "fesomc_gpu_run")
            _assert_same(got[i], g.state(), i)
        finally:
            g.close()
