"""ctypes mirror of include/fesomc_gpu.h.

The structures below are field-for-field copies of the C declarations; the
loader finds the in-tree shared library built by fesomc.build.
"""
import ctypes as C
import os

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
ROOT_DIR = os.path.dirname(PKG_DIR)              # fesom-c_b200/
REPO_DIR = os.path.dirname(ROOT_DIR)
LIB_PATH = os.path.join(ROOT_DIR, "libfesomc_gpu.so")

i32p = C.POINTER(C.c_int32)
f64p = C.POINTER(C.c_double)
f32p = C.POINTER(C.c_float)

FESOMC_OK = 0
ERRORS = {1: "EINVAL", 2: "ENOMEM", 3: "ECUDA", 4: "ESTATE", 5: "ENEGSALT", 6: "ELOWTEMP",
          7: "ENONFINITE", 8: "ENOTCONV", 9: "EMESH"}

F_ETA, F_UV2D, F_UV3D, F_TS, F_MIX, F_WVEL, F_MASK, F_CLIM, F_DIAG = (
    0x1, 0x2, 0x4, 0x8, 0x10, 0x20, 0x40, 0x80, 0x100)
F_ALL = 0xFFFF
ST_NEGSALT, ST_LOWTEMP, ST_NONFINITE, ST_NOTCONV = 0x1, 0x2, 0x4, 0x8
TRACER_UPWIND, TRACER_MUSCL, TRACER_MIURA = 1, 2, 4


class Mesh(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("nod2D", "elem2D", "edge2D", "edge2D_in", "nsigma",
                                         "nod_in_elem2D_max")] + \
        [(n, i32p) for n in ("index_nod2D", "elem2D_nodes", "edge_nodes", "edge_tri", "elem_edges",
                             "elem_neighbors", "nod_in_elem2D_num", "nod_in_elem2D", "edge_up_dn_tri")] + \
        [(n, f64p) for n in ("coord_nod2D", "depth", "area", "elem_area", "elem_cos", "coriolis", "w_cv",
                             "gradient_sca", "gradient_vec", "edge_dxdy", "edge_cross_dxdy", "sigma",
                             "a_tp", "ac")] + \
        [("nobn", C.c_int32), ("in_obn", i32p), ("n_rivers", C.c_int32), ("nod_rivers", i32p)]


class Params(C.Structure):
    _fields_ = [("dt", C.c_double), ("dt_2D", C.c_double), ("Mt", C.c_int32), ("Dmin", C.c_double),
                ("C_d", C.c_double), ("beta", C.c_double), ("epsilon", C.c_double),
                ("density_0", C.c_double), ("scale_area", C.c_double)] + \
        [(n, C.c_double) for n in ("snul", "z0b_min", "z0s_min", "Pr_num", "beta_scale", "cka",
                                   "tau_inv_filt", "K_hor", "Cd_bz", "Bp_bz", "clim_relax",
                                   "relax2clim_ac", "river_salinity", "time_jd0")] + \
        [(n, C.c_int32) for n in ("mom_adv_2D", "mom_adv_3D", "vert_adv", "im_vert_visc",
                                  "im_vert_visc_fic", "fic_point", "tracer_adv", "ver_mix", "filt_2D",
                                  "filt_3D", "wet_dry_on", "key_rivers", "TF_presence", "restart",
                                  "cl_relax", "cl_solid_boder_relax", "temp_on", "salinity_on",
                                  "n_harm")] + \
        [("harm_index", C.c_int32 * 12), ("fp32_form", C.c_int32), ("bih_3D", C.c_int32), ("Abh0", C.c_double),
                                  ("filt_bi_3D", C.c_int32), ("filt_bi_2D", C.c_int32), ("tau_c", C.c_double),
                                  ("bih_2D", C.c_int32), ("T_potential", C.c_int32), ("npes", C.c_int32),
                                  ("key_atm", C.c_int32), ("type_swr_body", C.c_int32), ("jer_const", C.c_int32),
                                  ("Rjc", C.c_double), ("ajc", C.c_double), ("bjc", C.c_double),
                                  ("sfc_order", C.c_int32)]


STATE_FIELDS = ["eta_n", "eta_n_1", "eta_n_2", "etaAB", "U_n_2D", "U_n_1", "U_n_2", "U_filt_2D",
                "V_filt_2D", "U_n", "V_n", "U_rhsAB", "V_rhsAB", "U_n_filt", "V_n_filt", "TF", "SF",
                "T_old", "S_old", "Tclim", "Sclim", "bt", "snu", "Kv", "Ri", "tke_dissip", "Av", "Wvel",
                "mask_wd", "mask_wd_node", "ssh_gp", "rho_c", "hpressure", "Bar_pr_2D"]


class State(C.Structure):
    _fields_ = [(n, f64p) for n in STATE_FIELDS] + [("lfirst", C.c_int32), ("time_jd", C.c_double)]


class Forcing(C.Structure):
    _fields_ = [(n, f64p) for n in ("taux", "tauy", "windx", "windy", "runoff_rivers", "Tclim", "Sclim",
                                    "ampt", "fazt", "amp_factor", "phy_factor", "mslp", "emp", "qsr", "qns",
                                    "Rj", "aj", "bj")]


class MeshOpts(C.Structure):
    _fields_ = [("cartesian", C.c_int32), ("coriolis_on", C.c_int32), ("lat_cartesian_deg", C.c_double),
                ("cyclic_length_deg", C.c_double), ("nsigma", C.c_int32), ("ind_sigma", C.c_int32),
                ("pow_sig", C.c_double), ("lev_bot", C.c_double), ("lev_sur", C.c_double),
                ("T_potential", C.c_int32), ("with_up_dn_tri", C.c_int32)]


class Members(C.Structure):
    _fields_ = [("n", C.c_int32), ("node_off", i32p), ("elem_off", i32p), ("scale_area", f64p)]


class ClosureReport(C.Structure):
    _fields_ = [(n, C.c_int64) for n in ("steps", "judge_steps", "wet_columns", "out_of_envelope", "dry_columns",
                                         "judge_values")] + [("judge_rms_log", C.c_double), ("judge_max_log", C.c_double)]


# Every symbol include/fesomc_gpu.h declares, with its ctypes signature.
SIGNATURES = {
    "fesomc_gpu_init": (C.c_int, [C.POINTER(Mesh), C.POINTER(Params), C.POINTER(State), C.POINTER(C.c_void_p)]),
    "fesomc_gpu_set_forcing": (C.c_int, [C.c_void_p, C.POINTER(Forcing)]),
    "fesomc_gpu_set_device_forcing": (C.c_int, [C.c_void_p, f64p, C.c_int32]),
    "fesomc_gpu_step": (C.c_int, [C.c_void_p, C.c_int32]),
    "fesomc_gpu_run": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
    "fesomc_gpu_sync_to_host": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(State)]),
    "fesomc_gpu_sync_from_host": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(State)]),
    "fesomc_gpu_set_tracer_range": (C.c_int, [C.c_void_p, f64p]),
    "fesomc_gpu_set_atm_fields": (C.c_int, [C.c_void_p, f64p, f64p, C.c_int32, C.c_double]),
    "fesomc_gpu_halo_plan": (C.c_int, [C.c_void_p, C.c_int32, i32p, C.c_int32, i32p, C.POINTER(C.c_void_p)]),
    "fesomc_gpu_halo_size": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "fesomc_gpu_halo_pack": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "fesomc_gpu_halo_unpack": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "fesomc_gpu_halo_range": (C.c_int, [C.c_void_p, C.c_void_p, f64p]),
    "fesomc_gpu_halo_free": (None, [C.c_void_p]),
    "fesomc_gpu_snapshot_begin": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(State)]),
    "fesomc_gpu_snapshot_end": (C.c_int, [C.c_void_p]),
    "fesomc_gpu_energy": (C.c_int, [C.c_void_p, f64p]),
    "fesomc_gpu_last_status": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint32), i32p]),
    "fesomc_gpu_finalize": (C.c_int, [C.c_void_p]),
    "fesomc_gpu_error_string": (C.c_char_p, [C.c_int]),
    "fesomc_mesh_build": (C.c_int, [C.c_int32, f64p, i32p, C.c_int32, i32p, f64p, C.POINTER(MeshOpts),
                                    C.POINTER(C.c_void_p)]),
    "fesomc_mesh_view": (C.c_int, [C.c_void_p, C.POINTER(Mesh)]),
    "fesomc_mesh_scale_area": (C.c_double, [C.c_void_p]),
    "fesomc_mesh_set_rivers": (C.c_int, [C.c_void_p, C.c_int32, i32p]),
    "fesomc_mesh_set_sponge": (C.c_int, [C.c_void_p, C.c_double]),
    "fesomc_mesh_free": (None, [C.c_void_p]),
    "fesomc_gpu_time_run": (C.c_int, [C.c_void_p, C.c_int32, f64p]),
    "fesomc_gpu_d3end_iterations": (C.c_int, [C.c_void_p, C.c_int32, i32p]),
    "fesomc_gpu_profile": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, i32p, C.c_char_p, f64p, f64p,
                                     C.POINTER(C.c_int64)]),
    "fesomc_ensemble_run": (C.c_int, [C.POINTER(C.c_void_p), C.c_int32, C.c_int32, f64p, i32p]),
    "fesomc_gpu_tune_knobs": (C.c_int, []),
    "fesomc_closure_set_rules": (C.c_int, [C.c_void_p, C.c_int32]),
    "fesomc_gpu_tune_knob": (C.c_int, [C.c_int32, C.c_char_p, C.c_int32, C.c_char_p, C.c_int32]),
    "fesomc_gpu_tune_get": (C.c_int, [C.c_void_p, i32p, i32p]),
    "fesomc_gpu_tune_set": (C.c_int, [C.c_void_p, i32p]),
    "fesomc_gpu_init_packed": (C.c_int, [C.POINTER(Mesh), C.POINTER(Params), C.POINTER(State), C.POINTER(Members),
                                         C.POINTER(C.c_void_p)]),
    "fesomc_gpu_set_device": (C.c_int, [C.c_int32]),
    "fesomc_closure_create": (C.c_int, [C.c_int32, C.c_int64, C.c_uint64, C.POINTER(C.c_void_p)]),
    "fesomc_closure_free": (None, [C.c_void_p]),
    "fesomc_closure_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64), i32p, i32p]),
    "fesomc_closure_harvest": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32]),
    "fesomc_closure_fit": (C.c_int, [C.c_void_p]),
    "fesomc_closure_train": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_float, C.c_uint64, f32p]),
    "fesomc_closure_params": (C.c_int, [C.c_void_p, f32p, f32p]),
    "fesomc_closure_norm": (C.c_int, [C.c_void_p, f32p, f32p]),
    "fesomc_closure_forward": (C.c_int, [C.c_void_p, f32p, C.c_int64, f32p, C.c_int32]),
    "fesomc_closure_grad": (C.c_int, [C.c_void_p, f32p, f32p, C.c_int32, f64p, f32p]),
    "fesomc_closure_attach": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32]),
    "fesomc_closure_stats": (C.c_int, [C.c_void_p, C.POINTER(ClosureReport)]),
    "fesomc_closure_time": (C.c_int, [C.c_void_p, C.c_int64, C.c_int32, C.c_int32, f64p]),
    "fesomc_gpu_version": (C.c_char_p, []),
    "fesomc_gpu_kernel_launches": (C.c_int64, [C.c_void_p]),
    "fesomc_host_density_jm": (C.c_double, [C.c_double, C.c_double, C.c_double, C.c_double]),
    "fesomc_energy_device": (C.c_int, [C.c_int32, C.c_int32, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, f64p]),
}

_lib = None


def load(path=None):
    """Load the in-tree C-ABI library (raises if it was not built)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"fesomc: C-ABI library not built ({p}); run fesomc.build.build()")
    lib = C.CDLL(p)
    lib.missing_symbols = []
    for name, (res, args) in SIGNATURES.items():
        try:
            fn = getattr(lib, name)
        except AttributeError:
            lib.missing_symbols.append(name)
            continue
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(rc, what="fesomc call"):
    if rc != FESOMC_OK:
        raise RuntimeError(f"{what} failed: {ERRORS.get(rc, rc)}")


def dptr(a):
    """double* to a C-contiguous float64 numpy array (or NULL)."""
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(f64p)


def fptr(a):
    """float* to a C-contiguous float32 numpy array (or NULL)."""
    if a is None:
        return None
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(f32p)


def iptr(a):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(i32p)
