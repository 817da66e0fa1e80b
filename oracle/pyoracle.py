"""ctypes binding of the CPU oracle (test infrastructure only).

Used by tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py
as the checker; never by the GPU product path.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")


def build():
    r = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    return LIB


_lib = None


def load(abi):
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        lib = C.CDLL(LIB)
        lib.oracle_create.restype = C.c_void_p
        lib.oracle_create.argtypes = [C.POINTER(abi.Mesh), C.POINTER(abi.Params), C.POINTER(abi.State)]
        lib.oracle_set_forcing.restype = C.c_int
        lib.oracle_set_forcing.argtypes = [C.c_void_p, C.POINTER(abi.Forcing)]
        lib.oracle_step.restype = C.c_int
        lib.oracle_step.argtypes = [C.c_void_p]
        lib.oracle_energy.restype = C.c_double
        lib.oracle_energy.argtypes = [C.c_void_p]
        lib.oracle_get_state.restype = None
        lib.oracle_get_state.argtypes = [C.c_void_p, C.POINTER(abi.State)]
        lib.oracle_array.restype = C.POINTER(C.c_double)
        lib.oracle_array.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_int64)]
        lib.oracle_free.restype = None
        lib.oracle_free.argtypes = [C.c_void_p]
        lib.oracle_notconv.restype = C.c_int
        lib.oracle_notconv.argtypes = [C.c_void_p]
        lib.oracle_T_aver.restype = C.c_double
        lib.oracle_T_aver.argtypes = [C.c_void_p]
        lib.oracle_densityJM.restype = C.c_double
        lib.oracle_densityJM.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double]
        lib.oracle_log.restype = C.c_double
        lib.oracle_log.argtypes = [C.c_double]
        lib.oracle_atm_fluxes.restype = C.c_int
        lib.oracle_atm_fluxes.argtypes = [C.c_void_p, abi.f64p, abi.f64p, C.c_int, C.c_double, C.c_double]
        lib.oracle_atan.restype = C.c_double
        lib.oracle_atan.argtypes = [C.c_double]
        lib.oracle_cos.restype = C.c_double
        lib.oracle_cos.argtypes = [C.c_double]
        lib.oracle_sin.restype = C.c_double
        lib.oracle_sin.argtypes = [C.c_double]
        lib.oracle_exp.restype = C.c_double
        lib.oracle_exp.argtypes = [C.c_double]
        lib.oracle_sw_cp.restype = C.c_double
        lib.oracle_sw_cp.argtypes = [C.c_double, C.c_double, C.c_double]
        lib.oracle_mesh_build.restype = C.c_int
        lib.oracle_mesh_build.argtypes = [C.c_int32, abi.f64p, abi.i32p, C.c_int32, abi.i32p, abi.f64p,
                                          C.POINTER(abi.MeshOpts), C.POINTER(C.c_void_p)]
        lib.oracle_mesh_view.restype = C.c_int
        lib.oracle_mesh_view.argtypes = [C.c_void_p, C.POINTER(abi.Mesh)]
        lib.oracle_mesh_scale_area.restype = C.c_double
        lib.oracle_mesh_scale_area.argtypes = [C.c_void_p]
        lib.oracle_mesh_set_rivers.restype = C.c_int
        lib.oracle_mesh_set_rivers.argtypes = [C.c_void_p, C.c_int32, abi.i32p]
        lib.oracle_mesh_set_sponge.restype = C.c_int
        lib.oracle_mesh_set_sponge.argtypes = [C.c_void_p, C.c_double]
        lib.oracle_mesh_free.restype = None
        lib.oracle_mesh_free.argtypes = [C.c_void_p]
        f32p = C.POINTER(C.c_float)
        lib.oracle_mlp_nparams.restype = C.c_int64
        lib.oracle_mlp_nparams.argtypes = [C.c_int]
        lib.oracle_mlp_forward.restype = C.c_int
        lib.oracle_mlp_forward.argtypes = [C.c_int, f32p, f32p, C.c_int, f32p]
        lib.oracle_mlp_grad.restype = C.c_int
        lib.oracle_mlp_grad.argtypes = [C.c_int, f32p, f32p, f32p, C.c_int, C.POINTER(C.c_double),
                                        C.POINTER(C.c_double)]
        lib.oracle_mlp_adam.restype = None
        lib.oracle_mlp_adam.argtypes = [C.c_int64, f32p, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                        C.POINTER(C.c_double), C.c_int, C.c_double]
        _lib = lib
    return _lib


class MeshLib:
    """The oracle's own mesh restatement (oracle_mesh.c) under the names of
    the product's host mesh builder, so that cases.* can build a case's mesh,
    sigma levels and density_0 without loading the product library:
    cases.estuary(cfg, lib=pyoracle.MeshLib(abi))."""

    def __init__(self, abi):
        lib = load(abi)
        self.missing_symbols = []
        self.fesomc_mesh_build = lib.oracle_mesh_build
        self.fesomc_mesh_view = lib.oracle_mesh_view
        self.fesomc_mesh_scale_area = lib.oracle_mesh_scale_area
        self.fesomc_mesh_set_rivers = lib.oracle_mesh_set_rivers
        self.fesomc_mesh_set_sponge = lib.oracle_mesh_set_sponge
        self.fesomc_mesh_free = lib.oracle_mesh_free
        self.fesomc_host_density_jm = lib.oracle_densityJM


class Oracle:
    """One oracle model instance driven like the reference main loop."""

    def __init__(self, case, abi, cases_mod):
        self.lib = load(abi)
        self.case, self.abi, self.cm = case, abi, cases_mod
        self.arrays = case.new_state_arrays()
        st = case.state_struct(self.arrays, case.params.time_jd0, lfirst=1)
        self.h = self.lib.oracle_create(C.byref(case.mesh.c), C.byref(case.params), C.byref(st))
        if not self.h:
            raise RuntimeError("oracle_create failed")
        self.time_jd = case.params.time_jd0
        self.nstep = 0
        self.atm = None

    def set_atm_fields(self, coef_a, coef_b, net_flux=0, prec_coef=1.0):
        """sbc_do before every step from the time-interpolation coefficients
        (8 per node, reference layout), as fesomc_gpu_set_atm_fields."""
        self.atm = (np.ascontiguousarray(coef_a, dtype=np.float64), np.ascontiguousarray(coef_b, dtype=np.float64),
                    int(net_flux), float(prec_coef))

    def step(self, nsteps=1):
        rc = 0
        for _ in range(nsteps):
            self.nstep += 1
            t_next = self.cm.advance_time(self.time_jd, self.case.params.dt)
            f = self.case.forcing_fn(self.nstep, t_next)
            fs = self.cm.forcing_struct(f)
            self.lib.oracle_set_forcing(self.h, C.byref(fs))
            if self.atm is not None:
                a, b, nf, pc = self.atm
                self.lib.oracle_atm_fluxes(self.h, a.ctypes.data_as(C.POINTER(C.c_double)),
                                           b.ctypes.data_as(C.POINTER(C.c_double)), nf, pc, t_next)
            rc |= self.lib.oracle_step(self.h)
            self.time_jd = t_next
        return rc

    def energy(self):
        return self.lib.oracle_energy(self.h)

    def state(self):
        out = {k: np.empty_like(v) for k, v in self.case.state0.items()}
        st = self.case.state_struct(out, 0.0)
        self.lib.oracle_get_state(self.h, C.byref(st))
        out["_time_jd"] = st.time_jd
        return out

    def array(self, name):
        n = C.c_int64()
        p = self.lib.oracle_array(self.h, name.encode(), C.byref(n))
        if not p:
            raise KeyError(name)
        return np.ctypeslib.as_array(p, shape=(n.value,)).copy()

    def close(self):
        if self.h:
            self.lib.oracle_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def mlp_nparams(abi, nsigma):
    return load(abi).oracle_mlp_nparams(nsigma)


def mlp_forward(abi, nsigma, params, X):
    """The closure network on the CPU (double accumulation): Y = net(X)."""
    lib = load(abi)
    p, X = _f32(params), _f32(X)
    Y = np.empty((X.shape[0], nsigma), dtype=np.float32)
    f = C.POINTER(C.c_float)
    if lib.oracle_mlp_forward(nsigma, p.ctypes.data_as(f), X.ctypes.data_as(f), X.shape[0], Y.ctypes.data_as(f)):
        raise RuntimeError("oracle_mlp_forward failed")
    return Y


def mlp_grad(abi, nsigma, params, X, T):
    """Mean squared error of the closure network and its exact gradient."""
    lib = load(abi)
    p, X, T = _f32(params), _f32(X), _f32(T)
    g = np.empty(p.size, dtype=np.float64)
    loss = C.c_double()
    f = C.POINTER(C.c_float)
    if lib.oracle_mlp_grad(nsigma, p.ctypes.data_as(f), X.ctypes.data_as(f), T.ctypes.data_as(f), X.shape[0],
                           C.byref(loss), g.ctypes.data_as(C.POINTER(C.c_double))):
        raise RuntimeError("oracle_mlp_grad failed")
    return loss.value, g
