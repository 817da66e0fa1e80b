"""Launch-shape knobs on the GPU: any accepted setting gives the same bits
as the defaults (both precision forms, MUSCL and upwind tracers), bad
settings are refused without changing anything, and the autotuner's search
returns shapes within the limits."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STEPS = 5


def _case(fp32, adv=None):
    from fesomc import abi, cases
    c = cases.estuary("small")
    c.params.fp32_form = fp32
    if adv is not None:
        c.params.tracer_adv = adv
    return c


def _run(case, shapes=None):
    from fesomc import autotune, model
    g = model.GpuModel(case)
    try:
        if shapes is not None:
            autotune.apply(g, shapes)
        assert g.step(STEPS) == 0
        return g.state()
    finally:
        g.close()


@pytest.mark.parametrize("fp32,adv", [(0, None), (1, None), (0, 1)])
def test_every_shape_gives_the_same_bits(built, fp32, adv):
    from fesomc import autotune, model
    ref = _run(_case(fp32, adv))
    g = model.GpuModel(_case(fp32, adv))
    try:
        _, lim = autotune.get(g)
    finally:
        g.close()
    small = {k: (1 if k in autotune.FORMS else 64) for k in lim}
    large = dict(lim)
    for shapes in (small, large):
        got = _run(_case(fp32, adv), shapes)
        for f, v in ref.items():
            if not f.startswith("_"):
                assert np.array_equal(got[f], v), (shapes, f)


def test_bad_shapes_are_refused(built):
    from fesomc import autotune, model
    g = model.GpuModel(_case(0))
    try:
        cur, lim = autotune.get(g)
        n = len(cur)
        for k, bad in (("velrhs", 33), ("velrhs", lim["velrhs"] + 32), ("columns", lim["columns"] + 1),
                       ("av", -32)):
            vals = dict(cur)
            vals[k] = bad
            arr = (C.c_int32 * n)(*[vals[name] for name, _ in autotune.knobs(g.lib)])
            assert g.lib.fesomc_gpu_tune_set(g.h, arr) == 1
            assert autotune.get(g)[0] == cur
    finally:
        g.close()


def test_search_returns_shapes_within_limits(built, tmp_path):
    from fesomc import autotune, model
    case = _case(1)
    shapes, rep = autotune.shapes_for(case, path=str(tmp_path / "s.json"), steps=2, warmup=1)
    assert rep["cached"] is False and rep["trials"] > 0
    g = model.GpuModel(case)
    try:
        _, lim = autotune.get(g)
        autotune.apply(g, shapes)
        assert autotune.get(g)[0] == shapes
    finally:
        g.close()
    assert all(0 < shapes[k] <= lim[k] for k in shapes)
    again, rep2 = autotune.shapes_for(case, path=str(tmp_path / "s.json"))
    assert rep2["cached"] is True and again == shapes
