"""The C-ABI library loads on a CPU-only host and exports every entry point
declared in include/fesomc_gpu.h (no GPU compute is issued here)."""
import ctypes as C
import os
import re

from conftest import ROOT


def header_functions():
    txt = open(os.path.join(ROOT, "include", "fesomc_gpu.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(fesomc_\w+)\s*\(", txt)))


def test_header_functions_found():
    fns = header_functions()
    assert "fesomc_gpu_init" in fns and "fesomc_gpu_step" in fns and "fesomc_mesh_build" in fns
    assert len(fns) >= 20


def test_library_exports_every_declared_symbol(built):
    lib = C.CDLL(os.path.join(ROOT, "fesom-c_b200", "libfesomc_gpu.so"))
    missing = [f for f in header_functions() if not hasattr(lib, f)]
    assert missing == []


def test_python_signatures_match_header(built):
    from fesomc import abi
    assert sorted(abi.SIGNATURES) == header_functions()
    assert built.missing_symbols == []


def test_error_strings(built):
    for code in range(0, 10):
        assert built.fesomc_gpu_error_string(code)
    assert b"salinity" in built.fesomc_gpu_error_string(5)


def test_init_rejects_bad_arguments_without_gpu(built):
    from fesomc import abi
    h = C.c_void_p()
    assert built.fesomc_gpu_init(None, None, None, C.byref(h)) == 1
    m = abi.Mesh()
    m.nsigma = 3     # fewer than 5 sigma levels is rejected before any CUDA call
    m.nod2D = 10
    m.elem2D = 5
    p = abi.Params()
    s = abi.State()
    assert built.fesomc_gpu_init(C.byref(m), C.byref(p), C.byref(s), C.byref(h)) == 1


def test_init_rejects_more_than_one_rank_without_gpu(built):
    """The whole mesh lives on one GPU (no halo exchange): a driver that runs
    with npes > 1 ranks is refused before any CUDA call."""
    from fesomc import abi, cases
    case = cases.estuary("small")
    arrays = case.new_state_arrays()
    st = case.state_struct(arrays, case.params.time_jd0)
    h = C.c_void_p()
    case.params.npes = 2
    assert built.fesomc_gpu_init(C.byref(case.mesh.c), C.byref(case.params), C.byref(st), C.byref(h)) == 1
    assert not h.value


def test_host_density_matches_oracle(built):
    import pyoracle
    from fesomc import abi
    olib = pyoracle.load(abi)
    for t, s, p in [(17.857142857142858, 0.0, 0.0), (35.714285714285715, 0.0, -12.0), (12.0, 30.0, -3.5),
                    (3.0, 35.5, -3000.0)]:
        assert built.fesomc_host_density_jm(t, s, p, 1000.0) == olib.oracle_densityJM(t, s, p, 1000.0)
    # pure water near 17.9 C and 35.7 C (independent sanity of the EOS restatement)
    assert abs(built.fesomc_host_density_jm(17.857142857142858, 0.0, 0.0, 0.0) - 998.62) < 0.01
    assert abs(built.fesomc_host_density_jm(35.714285714285715, 0.0, 0.0, 0.0) - 993.79) < 0.01


def test_init_rejects_bad_atmospheric_options_without_gpu(built):
    """key_atm must be 0/1, type_swr_body 1 or 2 and jer_const 0/1
    (fv_read_run.F90:799-803)."""
    from fesomc import cases
    case = cases.estuary("small")
    arrays = case.new_state_arrays()
    st = case.state_struct(arrays, case.params.time_jd0)
    h = C.c_void_p()
    for bad in ({"key_atm": 2}, {"key_atm": 1, "type_swr_body": 3}, {"key_atm": 1, "jer_const": 2}, {"sfc_order": 2}):
        p = cases.default_params(**bad)
        p.scale_area, p.density_0 = case.params.scale_area, case.params.density_0
        assert built.fesomc_gpu_init(C.byref(case.mesh.c), C.byref(p), C.byref(st), C.byref(h)) == 1, bad
