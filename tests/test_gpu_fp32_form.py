"""The FP32 form (fesomc_params.fp32_form = 1): level fields, mesh geometry
and the 3D arithmetic in FP32, the barotropic sub-cycle and the energy
integral in FP64.  It is compared with the plain FP64 path on the same case
through the C-ABI.  Tolerances follow the form's error budget against the
FP64 path (SSH RMS 1 mm, T/S 0.01) scaled to these short runs, and the
domain volume, whose
accumulation stays FP64, is held to round-off in a closed basin."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SSH_RMS_MAX = 1.0e-3      # m
TS_MAX = 1.0e-2           # degC / psu
VOLUME_REL = 1.0e-13


@pytest.fixture(scope="module")
def mods(built):
    from fesomc import abi, cases, model
    return abi, cases, model


def run(mods, case, steps, fp32):
    abi, cases, model = mods
    case.params.fp32_form = 1 if fp32 else 0
    g = model.GpuModel(case)
    g.step(steps)
    st = g.state()
    e = g.energy()
    g.close()
    return st, e


def test_estuary_fp32_form_within_budget(mods):
    abi, cases, model = mods
    a, ea = run(mods, cases.estuary("small"), 60, False)
    b, eb = run(mods, cases.estuary("small"), 60, True)
    wet = a["mask_wd_node"] > 0
    ssh_rms = np.sqrt(np.mean((a["eta_n"][wet] - b["eta_n"][wet]) ** 2))
    assert ssh_rms < SSH_RMS_MAX
    assert np.max(np.abs(a["TF"] - b["TF"])) < TS_MAX
    assert np.max(np.abs(a["SF"] - b["SF"])) < TS_MAX
    assert np.array_equal(a["mask_wd"], b["mask_wd"])
    assert abs(ea - eb) <= 1e-3 * abs(ea)
    # the FP32 form really runs in FP32: the fields are not bit-identical
    assert not np.array_equal(a["TF"], b["TF"])


def test_closed_basin_volume_fp32_form(mods):
    abi, cases, model = mods
    case = cases.le_medium()
    case.params.Mt = 4
    case.params.fp32_form = 1
    area = case.mesh.area
    g = model.GpuModel(case)
    v0 = np.sum(area * (case.mesh.depth + g.state(abi.F_ETA)["eta_n"]))
    g.step(40)
    v1 = np.sum(area * (case.mesh.depth + g.state(abi.F_ETA)["eta_n"]))
    g.close()
    assert abs(v1 - v0) / v0 < VOLUME_REL


@pytest.mark.parametrize("scheme", ["upwind", "miura"])
def test_fp32_form_other_tracer_schemes(mods, scheme):
    abi, cases, model = mods
    adv = abi.TRACER_UPWIND if scheme == "upwind" else abi.TRACER_MIURA
    a, _ = run(mods, cases.estuary("small", tracer_adv=adv), 30, False)
    b, _ = run(mods, cases.estuary("small", tracer_adv=adv), 30, True)
    assert np.max(np.abs(a["TF"] - b["TF"])) < TS_MAX
    assert np.max(np.abs(a["SF"] - b["SF"])) < TS_MAX


def test_fp32_form_biharmonic(mods):
    a, _ = run(mods, mods[1].estuary("small", bih_3D=1, Abh0=1e4), 30, False)
    b, _ = run(mods, mods[1].estuary("small", bih_3D=1, Abh0=1e4), 30, True)
    assert np.max(np.abs(a["TF"] - b["TF"])) < TS_MAX
    assert np.max(np.abs(a["U_n"] - b["U_n"])) < 1e-3
    a, _ = run(mods, mods[1].estuary("small", bih_2D=1, Abh0=1e4), 30, False)
    b, _ = run(mods, mods[1].estuary("small", bih_2D=1, Abh0=1e4), 30, True)
    assert np.max(np.abs(a["TF"] - b["TF"])) < TS_MAX
    assert np.max(np.abs(a["U_n_2D"] - b["U_n_2D"])) < 1e-3
