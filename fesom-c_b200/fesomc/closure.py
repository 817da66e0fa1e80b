"""Host driver of the learned vertical-mixing closure (fesomc_closure_* in
include/fesomc_gpu.h): harvest columns from the plain closure d3_end
(src/fv_mixing.F90:73-347) while a model steps, fit the normalisation and the
training envelope, train on the GPU, and attach the network to a model's
time step.  No counterpart in the reference."""
import ctypes as C

import numpy as np

from . import abi

# rows of the statistics (norm): input mean, input sd, target mean, target
# sd, envelope low, envelope high (normalised inputs), lowest and highest
# target (log bt)
STAT_ROWS = 8


class Closure:
    """One network (and its training set) for meshes with nsigma levels."""

    def __init__(self, nsigma, capacity=0, seed=20261204):
        self.lib = abi.load()
        h = C.c_void_p()
        abi.check(self.lib.fesomc_closure_create(nsigma, int(capacity), seed, C.byref(h)), "fesomc_closure_create")
        self.h = h
        n_in, n_out = C.c_int32(), C.c_int32()
        np_ = C.c_int64()
        abi.check(self.lib.fesomc_closure_info(h, None, C.byref(np_), C.byref(n_in), C.byref(n_out)))
        self.nsigma, self.n_in, self.n_out, self.nparams = nsigma, n_in.value, n_out.value, np_.value

    def harvested(self):
        n = C.c_int64()
        abi.check(self.lib.fesomc_closure_info(self.h, C.byref(n), None, None, None))
        return n.value

    def harvest(self, model, nsteps, every=1):
        """Advance model (a fesomc.model.GpuModel, forcing as last set) by
        nsteps with the plain closure, harvesting every 'every'-th step."""
        rc = self.lib.fesomc_closure_harvest(self.h, model.h, nsteps, every)
        for _ in range(nsteps):
            model.time_jd += model.case.params.dt / 86400.0
        model.nstep += nsteps
        abi.check(rc, "fesomc_closure_harvest")

    def set_rules(self, unstable=False, boundary=False):
        """Fallback rules beyond the envelope, used from the next attach on:
        unstable -- statically unstable columns (N^2 < 0) to the plain closure;
        boundary -- columns at solid / open boundary nodes to the plain closure."""
        rules = (1 if unstable else 0) | (2 if boundary else 0)
        abi.check(self.lib.fesomc_closure_set_rules(self.h, rules), "fesomc_closure_set_rules")

    def fit(self):
        abi.check(self.lib.fesomc_closure_fit(self.h), "fesomc_closure_fit")

    def train(self, epochs, batch=4096, lr=1e-3, seed=1):
        losses = np.zeros(max(epochs, 1), dtype=np.float32)
        abi.check(self.lib.fesomc_closure_train(self.h, epochs, batch, lr, seed, abi.fptr(losses)),
                  "fesomc_closure_train")
        return losses[:epochs]

    def params(self, value=None):
        if value is not None:
            v = np.ascontiguousarray(value, dtype=np.float32)
            assert v.size == self.nparams
            abi.check(self.lib.fesomc_closure_params(self.h, None, abi.fptr(v)))
            return v
        out = np.empty(self.nparams, dtype=np.float32)
        abi.check(self.lib.fesomc_closure_params(self.h, abi.fptr(out), None))
        return out

    def norm(self, value=None):
        w = max(self.n_in, self.n_out)
        if value is not None:
            v = np.ascontiguousarray(value, dtype=np.float32).reshape(-1)
            assert v.size == STAT_ROWS * w
            abi.check(self.lib.fesomc_closure_norm(self.h, None, abi.fptr(v)))
            return v.reshape(STAT_ROWS, w)
        out = np.empty(STAT_ROWS * w, dtype=np.float32)
        abi.check(self.lib.fesomc_closure_norm(self.h, abi.fptr(out), None))
        return out.reshape(STAT_ROWS, w)

    def forward(self, X, bf16=False):
        """The network on normalised inputs; bf16: on the tensor cores."""
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.empty((X.shape[0], self.n_out), dtype=np.float32)
        abi.check(self.lib.fesomc_closure_forward(self.h, abi.fptr(X), X.shape[0], abi.fptr(Y), int(bf16)),
                  "fesomc_closure_forward")
        return Y

    def grad(self, X, T):
        X = np.ascontiguousarray(X, dtype=np.float32)
        T = np.ascontiguousarray(T, dtype=np.float32)
        g = np.empty(self.nparams, dtype=np.float32)
        loss = C.c_double()
        abi.check(self.lib.fesomc_closure_grad(self.h, abi.fptr(X), abi.fptr(T), X.shape[0], C.byref(loss),
                                               abi.fptr(g)), "fesomc_closure_grad")
        return loss.value, g

    def attach(self, model, judge_every=0, bf16=True):
        """The model's steps use this network (inference on the tensor cores
        unless bf16 is False); every judge_every-th step runs the plain
        closure and compares."""
        abi.check(self.lib.fesomc_closure_attach(model.h, self.h, judge_every, int(bf16)), "fesomc_closure_attach")

    @staticmethod
    def detach(model):
        abi.check(abi.load().fesomc_closure_attach(model.h, None, 0, 0), "fesomc_closure_attach")

    def time(self, ncol, reps=10, bf16=True):
        """Mean device ms of one pass over ncol device-resident columns."""
        ms = C.c_double()
        abi.check(self.lib.fesomc_closure_time(self.h, int(ncol), reps, int(bf16), C.byref(ms)), "fesomc_closure_time")
        return ms.value

    @staticmethod
    def stats(model):
        r = abi.ClosureReport()
        abi.check(abi.load().fesomc_closure_stats(model.h, C.byref(r)), "fesomc_closure_stats")
        return {k: getattr(r, k) for k, _ in abi.ClosureReport._fields_}

    def close(self):
        if getattr(self, "h", None):
            self.lib.fesomc_closure_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
