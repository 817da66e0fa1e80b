"""Host-side driver of the GPU time step, mirroring the reference main loop
(src/fv_main.F90:388-742): per internal step, advance time_jd, let the
forcing routines fill o_ARRAYS (rivers_do / sbc_do / obc_do), call the time
step, and pull state back for diagnostics and output.
"""
import ctypes as C

import numpy as np

from . import abi, cases


class GpuModel:
    """One model instance on the current CUDA device, driven through the C-ABI."""

    def __init__(self, case):
        self.lib = abi.load()
        if self.lib.missing_symbols:
            raise RuntimeError("C-ABI library lacks symbols: %s" % self.lib.missing_symbols)
        self.case = case
        self.arrays = case.new_state_arrays()
        st = case.state_struct(self.arrays, case.params.time_jd0, lfirst=1)
        h = C.c_void_p()
        members = getattr(case, "members", None)   # packed members (packed.PackedCase)
        if members is not None:
            abi.check(self.lib.fesomc_gpu_init_packed(C.byref(case.mesh.c), C.byref(case.params), C.byref(st),
                                                      C.byref(members), C.byref(h)), "fesomc_gpu_init_packed")
        else:
            abi.check(self.lib.fesomc_gpu_init(C.byref(case.mesh.c), C.byref(case.params), C.byref(st), C.byref(h)),
                      "fesomc_gpu_init")
        self.h = h
        self.time_jd = case.params.time_jd0
        self.nstep = 0

    def set_atm_fields(self, coef_a, coef_b, net_flux=0, prec_coef=1.0):
        """sbc_do on the device from the atmospheric fields' time-interpolation
        coefficients (fesomc_gpu_set_atm_fields)."""
        a = np.ascontiguousarray(coef_a, dtype=np.float64)
        b = np.ascontiguousarray(coef_b, dtype=np.float64)
        abi.check(self.lib.fesomc_gpu_set_atm_fields(self.h, abi.dptr(a), abi.dptr(b), int(net_flux),
                                                      float(prec_coef)), "fesomc_gpu_set_atm_fields")

    def set_forcing(self, fdict):
        f = cases.forcing_struct(fdict)
        abi.check(self.lib.fesomc_gpu_set_forcing(self.h, C.byref(f)), "fesomc_gpu_set_forcing")

    def step(self, nsteps=1, check=True):
        """Advance nsteps internal steps, pushing the case's forcing before each."""
        rc_all = 0
        for _ in range(nsteps):
            self.nstep += 1
            t_next = cases.advance_time(self.time_jd, self.case.params.dt)
            self.set_forcing(self.case.forcing_fn(self.nstep, t_next))
            rc = self.lib.fesomc_gpu_step(self.h, self.nstep)
            self.time_jd = t_next
            if rc and check:
                abi.check(rc, "fesomc_gpu_step")
            rc_all = rc_all or rc
        return rc_all

    def run(self, nsteps, check=True):
        """Advance nsteps with the forcing of the first of them held fixed
        (one launch sequence, no per-step host round trip)."""
        t_next = cases.advance_time(self.time_jd, self.case.params.dt)
        self.set_forcing(self.case.forcing_fn(self.nstep + 1, t_next))
        rc = self.lib.fesomc_gpu_run(self.h, self.nstep + 1, nsteps)
        for _ in range(nsteps):
            self.time_jd = cases.advance_time(self.time_jd, self.case.params.dt)
        self.nstep += nsteps
        if rc and check:
            abi.check(rc, "fesomc_gpu_run")
        return rc

    def state(self, mask=abi.F_ALL):
        out = {k: np.empty_like(v) for k, v in self.case.state0.items()}
        st = self.case.state_struct(out, 0.0)
        abi.check(self.lib.fesomc_gpu_sync_to_host(self.h, mask, C.byref(st)), "fesomc_gpu_sync_to_host")
        out["_time_jd"] = st.time_jd
        return out

    def energy(self):
        e = C.c_double()
        abi.check(self.lib.fesomc_gpu_energy(self.h, C.byref(e)), "fesomc_gpu_energy")
        return e.value

    def snapshot_begin(self, mask=abi.F_ALL):
        """Start an asynchronous copy of the masked fields (state after every
        step enqueued so far) into host arrays this object keeps (page-locked
        by the library on first use); stepping may go on meanwhile."""
        if getattr(self, "_snap", None) is None:
            arrays = {k: np.empty_like(v) for k, v in self.case.state0.items()}
            self._snap = (arrays, self.case.state_struct(arrays, 0.0))
        abi.check(self.lib.fesomc_gpu_snapshot_begin(self.h, mask, C.byref(self._snap[1])),
                  "fesomc_gpu_snapshot_begin")

    def snapshot_end(self):
        """Wait for the snapshot started by snapshot_begin and return a copy."""
        abi.check(self.lib.fesomc_gpu_snapshot_end(self.h), "fesomc_gpu_snapshot_end")
        arrays, st = self._snap
        out = {k: v.copy() for k, v in arrays.items()}
        out["_time_jd"] = st.time_jd
        return out

    def status(self):
        s, nc = C.c_uint32(), C.c_int32()
        self.lib.fesomc_gpu_last_status(self.h, C.byref(s), C.byref(nc))
        return s.value, nc.value

    def kernel_launches(self):
        return self.lib.fesomc_gpu_kernel_launches(self.h)

    def close(self):
        if getattr(self, "h", None):
            self.lib.fesomc_gpu_finalize(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
