"""Launch-shape autotuner over the knobs of fesomc_gpu_tune_* (threads per
block of the kernels whose results do not depend on the block shape, and
entities per block of the column kernels).

The search is a coordinate descent: each knob in turn is tried at its
candidate values while the others hold, each value timed with
fesomc_gpu_profile (device time of the knob's own kernels per step) on a
scratch model of the same case, so the model a caller tunes for is never
advanced.  A value replaces the current one only when it is faster by more
than `margin`.  Any setting gives the same bits, so tuning changes speed
only.

Results are cached per mesh size (nodes, elements, edges), level count,
precision form, tracer scheme and storage order in a JSON file: the user's cache
(FESOMC_LAUNCH_SHAPES, default ~/.cache/fesomc/launch_shapes.json), seeded
by the shapes measured on a B200 that ship with the package
(launch_shapes_b200.json).
"""
import ctypes as C
import json
import os
import tempfile
import time

import numpy as np

from . import abi, cases, model

THREADS = (64, 128, 256, 512, 1024)
COLUMNS = (1, 2, 4, 8, 16, 32)
# d3_end: local-memory arrays, shared-memory arrays, set-up and sweep kernels
# (the sweep's arrays in local memory, in shared memory, or in registers at
# 6 or 8 resident blocks per SM)
D3END_ARRAYS = (1, 2, 3, 4, 5, 6)
# tracer_impl_vert_diff: columns read directly, or tiles of 128 or 64 columns
# staged in shared memory
VDIFF_FORMS = (1, 2, 3)
# the knobs that pick a form rather than a block size
# momentum_vert_impl_visc_tmp: columns read directly, or tiles of 64 columns
IMPLVISC_FORMS = (1, 2)
FORMS = {"columns": COLUMNS, "d3end_arrays": D3END_ARRAYS, "vdiff_form": VDIFF_FORMS,
         "implvisc_form": IMPLVISC_FORMS}
SHIPPED = os.path.join(os.path.dirname(os.path.abspath(__file__)), "launch_shapes_b200.json")


def cache_path():
    return os.environ.get("FESOMC_LAUNCH_SHAPES",
                          os.path.join(os.path.expanduser("~"), ".cache", "fesomc", "launch_shapes.json"))


def cache_key(case):
    m, p = case.mesh, case.params
    return "N%d-E%d-Ed%d-NS%d-%s-adv%d-mix%d-sfc%d" % (m.N, m.E, m.Ed, m.NS, "f32" if p.fp32_form else "f64",
                                                       p.tracer_adv, p.ver_mix, p.sfc_order)


def load_cache(path=None):
    """The cached shapes: the shipped table updated by the user's cache."""
    out = {}
    for f in (SHIPPED, path or cache_path()):
        try:
            with open(f) as fh:
                out.update(json.load(fh))
        except (OSError, ValueError):
            pass
    return out


def save_entry(key, shapes, path=None):
    """Adds one entry to the user's cache (written atomically)."""
    path = path or cache_path()
    data = {}
    try:
        with open(path) as fh:
            data = json.load(fh)
    except (OSError, ValueError):
        pass
    data[key] = shapes
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    fd, tmp = tempfile.mkstemp(dir=os.path.dirname(path) or ".", suffix=".tmp")
    with os.fdopen(fd, "w") as fh:
        json.dump(data, fh, indent=1, sort_keys=True)
    os.replace(tmp, path)


def knobs(lib=None):
    """[(name, [profile records])] in knob order."""
    lib = lib or abi.load()
    out = []
    for k in range(lib.fesomc_gpu_tune_knobs()):
        name, recs = C.create_string_buffer(64), C.create_string_buffer(256)
        abi.check(lib.fesomc_gpu_tune_knob(k, name, 64, recs, 256), "fesomc_gpu_tune_knob")
        out.append((name.value.decode(), recs.value.decode().split(",")))
    return out


def get(g):
    """(values, limits) of a GpuModel, by knob name."""
    names = [n for n, _ in knobs(g.lib)]
    v = (C.c_int32 * len(names))()
    lim = (C.c_int32 * len(names))()
    abi.check(g.lib.fesomc_gpu_tune_get(g.h, v, lim), "fesomc_gpu_tune_get")
    return dict(zip(names, list(v))), dict(zip(names, list(lim)))


def apply(g, shapes):
    """Sets the knobs named in shapes (others keep their value)."""
    names = [n for n, _ in knobs(g.lib)]
    cur, _ = get(g)
    cur.update({k: int(v) for k, v in shapes.items() if k in cur})
    arr = (C.c_int32 * len(names))(*[cur[n] for n in names])
    abi.check(g.lib.fesomc_gpu_tune_set(g.h, arr), "fesomc_gpu_tune_set")


def profile(g, steps):
    """Device ms per step of every profile record."""
    maxk = 128
    nk = C.c_int32()
    names = C.create_string_buffer(32 * maxk)
    ms = (C.c_double * maxk)()
    nbytes = (C.c_double * maxk)()
    launches = (C.c_int64 * maxk)()
    abi.check(g.lib.fesomc_gpu_profile(g.h, steps, maxk, C.byref(nk), names, ms, nbytes, launches),
              "fesomc_gpu_profile")
    out = {}
    for i in range(nk.value):
        nm = names.raw[32 * i:32 * i + 32].split(b"\0", 1)[0].decode()
        out[nm] = ms[i] * launches[i] / steps
    return out


def search(case, steps=3, warmup=2, margin=0.02, log=None):
    """Coordinate descent on a scratch model of `case`; returns (shapes by
    knob name, report)."""
    t0 = time.perf_counter()
    g = model.GpuModel(case)
    try:
        g.run(warmup)
        ks = knobs(g.lib)
        cur, lim = get(g)
        before = profile(g, steps)
        trials = 0
        for name, recs in ks:
            cands = FORMS.get(name, THREADS)
            cands = [c for c in cands if c <= lim[name]]

            def t_of(v):
                apply(g, {name: v})
                p = profile(g, steps)
                return sum(p.get(r, 0.0) for r in recs)

            best_v, best_t = cur[name], t_of(cur[name])
            for v in cands:
                if v == cur[name]:
                    continue
                t = t_of(v)
                trials += 1
                if t < best_t * (1.0 - margin):
                    best_v, best_t = v, t
            apply(g, {name: best_v})
            cur[name] = best_v
            if log:
                log("%-12s -> %4d  (%.4f ms/step)" % (name, best_v, best_t))
        after = profile(g, steps)
    finally:
        g.close()
    total = lambda p: sum(v for k, v in p.items())
    report = {"trials": trials, "seconds": time.perf_counter() - t0, "ms_per_step_before": total(before),
              "ms_per_step_after": total(after)}
    return cur, report


def shapes_for(case, refresh=False, path=None, **kw):
    """Cached shapes of the case's size, searched (and cached) when absent."""
    key = cache_key(case)
    if not refresh:
        hit = load_cache(path).get(key)
        if hit is not None:
            return hit, {"cached": True}
    shapes, report = search(case, **kw)
    save_entry(key, shapes, path)
    report["cached"] = False
    return shapes, report
