"""Ensembles of independent model instances.

On one GPU the members advance concurrently through fesomc_ensemble_run:
each member keeps its own stream and captured step graph, and the library
interleaves one step of every member per round, so small meshes that cannot
fill 148 SMs alone overlap with each other.  Across GPUs (one process per
GPU) the members are dealt out by longest-processing-time bin packing on
their cost N * L * steps; there is no exchange between members.

The reference runs one mesh per executable; an ensemble there is a set of
separate runs.
"""
import ctypes as C

import numpy as np

from . import abi, cases, model, packed

# member step statuses that fesomc_ensemble_run reports per member
STEP_STATUSES = {k for k, v in abi.ERRORS.items() if v in ("ENEGSALT", "ELOWTEMP", "ENONFINITE")}


def member_cost(case, steps=1):
    """Work of one member: node-level updates over `steps` internal steps."""
    return case.mesh.N * case.mesh.L * steps


def lpt_partition(costs, bins):
    """Longest-processing-time bin packing: members in order of decreasing
    cost (ties by index), each to the least loaded bin (ties by bin index).
    Returns one list of member indices per bin, each in assignment order
    (largest first).  Deterministic, so every rank computes the same plan."""
    if bins < 1:
        raise ValueError("bins must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0] * bins
    plan = [[] for _ in range(bins)]
    for i in order:
        b = min(range(bins), key=lambda k: (load[k], k))
        plan[b].append(i)
        load[b] += costs[i]
    return plan


class Ensemble:
    """Members (cases) on the current GPU, advanced together.  Each member's
    stress and wind are pushed once and held; its open-boundary tide and its
    river runoff (ramped over the first 10 days) are evaluated on the GPU at
    every step (fesomc_gpu_set_device_forcing)."""

    def __init__(self, member_cases):
        self.lib = abi.load()
        order = sorted(range(len(member_cases)), key=lambda i: (-member_cost(member_cases[i]), i))
        self.cases = [member_cases[i] for i in order]
        self.index = order                       # position -> caller's member index
        self.models = []
        try:
            for c in self.cases:
                g = model.GpuModel(c)
                t_next = cases.advance_time(g.time_jd, c.params.dt)
                g.set_forcing(c.forcing_fn(1, t_next))
                self.models.append(g)
                base = np.ascontiguousarray(c.forcing_fn(1, c.params.time_jd0 + 20.0)["runoff_rivers"],
                                            dtype=np.float64)
                abi.check(self.lib.fesomc_gpu_set_device_forcing(g.h, abi.dptr(base) if base.size else None, 1),
                          "fesomc_gpu_set_device_forcing")
        except Exception:
            self.close()
            raise
        self._handles = (C.c_void_p * len(self.models))(*[g.h.value for g in self.models])

    def _advance_clock(self, nsteps):
        for g in self.models:
            for _ in range(nsteps):
                g.time_jd = cases.advance_time(g.time_jd, g.case.params.dt)
            g.nstep += nsteps

    def run(self, nsteps, timed=False):
        """All members concurrently; returns (device ms or None, statuses in
        the caller's member order)."""
        n = len(self.models)
        st = (C.c_int32 * n)()
        ms = C.c_double()
        rc = self.lib.fesomc_ensemble_run(self._handles, n, nsteps, C.byref(ms) if timed else None, st)
        self._advance_clock(nsteps)
        if rc != abi.FESOMC_OK and rc not in STEP_STATUSES:
            abi.check(rc, "fesomc_ensemble_run")
        status = [0] * n
        for pos, i in enumerate(self.index):
            status[i] = st[pos]
        return (ms.value if timed else None), status

    def run_one_at_a_time(self, nsteps):
        """The same steps member after member, each on an otherwise idle GPU;
        returns the summed device ms and the statuses (caller's order)."""
        total = 0.0
        status = [0] * len(self.models)
        for pos, g in enumerate(self.models):
            ms = C.c_double()
            rc = self.lib.fesomc_gpu_time_run(g.h, nsteps, C.byref(ms))
            status[self.index[pos]] = rc
            total += ms.value
        self._advance_clock(nsteps)
        return total, status

    def member(self, i):
        """GpuModel of the caller's member i."""
        return self.models[self.index.index(i)]

    def close(self):
        for g in self.models:
            g.close()
        self.models = []


class PackedEnsemble(Ensemble):
    """The members packed into one model per level count (packed.PackedCase):
    every kernel of a step covers all members of a pack in one launch, and
    the packs (at most two here: 11 and 21 levels) run side by side as in
    Ensemble.  Statuses and states are reported per member."""

    def __init__(self, member_cases):
        groups = {}
        for i, c in enumerate(member_cases):
            groups.setdefault(c.mesh.NS, []).append(i)
        self.groups = [groups[k] for k in sorted(groups)]
        self.n_members = len(member_cases)
        self.packs = [packed.PackedCase([member_cases[i] for i in g], name="pack%d" % k)
                      for k, g in enumerate(self.groups)]
        super().__init__(self.packs)

    def _spread(self, pack_status):
        status = [0] * self.n_members
        for g, st in zip(self.groups, pack_status):
            for i in g:
                status[i] = st
        return status

    def run(self, nsteps, timed=False):
        ms, st = super().run(nsteps, timed)
        return ms, self._spread(st)

    def run_one_at_a_time(self, nsteps):
        ms, st = super().run_one_at_a_time(nsteps)
        return ms, self._spread(st)

    def member_state(self, i, mask=abi.F_ALL):
        """State of the caller's member i, split from its pack."""
        for k, g in enumerate(self.groups):
            if i in g:
                pack = self.packs[k]
                return pack.split_state(Ensemble.member(self, k).state(mask))[g.index(i)]
        raise IndexError(i)

