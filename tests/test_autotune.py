"""Launch-shape knobs and the autotuner's cache on the host: the library
names every knob and the profile records that time it (no GPU needed), the
records are ones the step reports, and the cache merges the shipped table
with the user's file and writes entries atomically."""
import json
import os
import re

from conftest import ROOT


def test_knobs_and_their_records(built):
    from fesomc import autotune
    ks = autotune.knobs(built)
    names = [n for n, _ in ks]
    assert len(ks) == built.fesomc_gpu_tune_knobs() >= 20 and len(set(names)) == len(names)
    assert "columns" in names and "velrhs" in names and "muscl_h" in names
    # every record is a profile record name of the step (model.cu rec(m, "...") calls)
    src = open(os.path.join(ROOT, "fesom-c_b200", "csrc", "model.cu")).read()
    recs = set(re.findall(r'rec\(m, "(\w+)"', src))
    for n, rr in ks:
        assert rr and all(r in recs for r in rr), (n, rr)
    assert built.fesomc_gpu_tune_knob(len(ks), None, 0, None, 0) == 1        # EINVAL


def test_cache_roundtrip(tmp_path, built):
    from fesomc import autotune, cases
    case = cases.estuary("small")
    key = autotune.cache_key(case)
    assert re.fullmatch(r"N\d+-E\d+-Ed\d+-NS\d+-f(32|64)-adv\d+-mix\d+-sfc\d", key)
    path = str(tmp_path / "shapes.json")
    assert key not in autotune.load_cache(path)
    autotune.save_entry(key, {"velrhs": 128, "columns": 4}, path)
    autotune.save_entry("other", {"velrhs": 64}, path)
    got = autotune.load_cache(path)
    assert got[key] == {"velrhs": 128, "columns": 4} and got["other"] == {"velrhs": 64}
    assert json.load(open(path))[key]["columns"] == 4
    shapes, rep = autotune.shapes_for(case, path=path)
    assert rep == {"cached": True} and shapes["velrhs"] == 128


def test_shipped_table_is_valid_json():
    from fesomc import autotune
    if os.path.exists(autotune.SHIPPED):
        data = json.load(open(autotune.SHIPPED))
        for k, v in data.items():
            assert re.fullmatch(r"N\d+-E\d+-Ed\d+-NS\d+-f(32|64)-adv\d+-mix\d+-sfc\d", k)
            assert all(isinstance(x, int) and x >= 0 for x in v.values())
