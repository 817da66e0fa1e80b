"""Benchmark of the FESOM-C internal time step on B200 (sm_100a, FP64).

Workload: the 1.05M-node, 21-sigma-level synthetic estuary (1501 x 701
nodes at 80 m spacing, 30 % of quads split into triangles, MUSCL tracers,
wetting/drying, M2 open-boundary tide, river inflow, 0.1 N/m2 wind stress),
one "step" = one internal time step of oce_timestep case(3) with its 10
external sub-steps.  Metric: node*level updates per second
(nod2D * (nsigma-1) * steps / seconds), whole job.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 (launched by torch.distributed.run) runs N independent replicas, one
per GPU: the single-mesh time step does not shard across GPUs.
--impl reference times the CPU implementation of the same time step on the
host cores (the oracle restatement of the reference, OpenMP over all cores;
the Fortran reference cannot be compiled in this image).
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "fesom-c_b200"))

METRIC = "node·level updates/s"
UNIT = "node-level updates/s"
HBM_FALLBACK_GBS = 6650.0


def dist_info():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", HBM_FALLBACK_GBS)), "measured"
    return HBM_FALLBACK_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    def __init__(self, gpu):
        self.gpu = gpu
        self.path = tempfile.mktemp(suffix=".csv")
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        sms, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            with open(self.path) as f:
                for line in f:
                    parts = [x.strip() for x in line.split(",")]
                    if len(parts) < 9:
                        continue
                    try:
                        sm = float(parts[1])
                        mx = float(parts[2])
                    except ValueError:
                        continue
                    sms.append(sm)
                    for nm, v in zip(names, parts[5:9]):
                        if v.lower() == "active":
                            reasons.add(nm)
            os.unlink(self.path)
        except Exception:
            pass
        if not sms:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": 0}
        return {"sm_mhz": statistics.median(sms), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sms)}


BUILD_OPTS = {}   # storage-order options of the run (--mesh-order, --shuffle)


def build_case(cfg, lib=None):
    from fesomc import cases
    return cases.estuary(cfg, lib=lib, **BUILD_OPTS)


def oracle_case(cfg):
    """The workload built by the oracle's own mesh restatement: the CPU legs
    never load the product library."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from fesomc import abi
    return build_case(cfg, lib=pyoracle.MeshLib(abi))


def host_cpu():
    """CPU model, physical cores and the hardware threads this process may use."""
    model, cores = None, set()
    phys = core = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                k, _, v = line.partition(":")
                k, v = k.strip(), v.strip()
                if k == "model name" and model is None:
                    model = v
                elif k == "physical id":
                    phys = v
                elif k == "core id":
                    core = v
                elif not k and phys is not None:
                    cores.add((phys, core))
                    phys = core = None
        if phys is not None:
            cores.add((phys, core))
    except OSError:
        pass
    try:
        threads = len(os.sched_getaffinity(0))
    except AttributeError:
        threads = os.cpu_count() or 1
    return {"model": model, "physical_cores": len(cores) or None, "threads_available": threads}


def cases_sponge_km(case):
    from fesomc import cases
    return cases.SPONGE_RADIUS / 1000.0


def workload_config(case, cfg):
    m = case.mesh
    state_gb = (m.N * m.L * 8 * 19 + m.E * m.L * 8 * 20 + m.N * m.NS * 8 * 7) / 1e9
    nx, ny = case.meta["nx"], case.meta["ny"]
    return {
        "workload": f"{cfg}: synthetic estuary {nx + 1}x{ny + 1} nodes ({case.meta['dx']:.0f} m), "
                    f"{m.NS} sigma levels, 30% quads split, MUSCL tracers, wetting/drying, "
                    f"M2 open-boundary tide, river 500 m3/s, cross-shore wind stress 0.1 N/m2, "
                    f"{cases_sponge_km(case):.0f} km open-boundary sponge; one step = one internal "
                    f"step (dt {case.params.dt:.0f} s) with {case.params.Mt} external sub-steps",
        "nodes": m.N, "elements": m.E, "edges": m.Ed, "levels": m.L,
        "dt_s": case.params.dt, "substeps": case.params.Mt,
        "l2": f"inputs larger than L2 (device state ~{state_gb:.1f} GB per replica, no flush needed)",
        "parallelism": "replicas (one independent mesh per GPU)",
        "numbering": ("nodes and elements numbered at random (seed %d)" % BUILD_OPTS["shuffle"]
                      if BUILD_OPTS.get("shuffle") is not None else "generator order (row by row)"),
        "storage_order": "Hilbert curve" if BUILD_OPTS.get("sfc_order") else "mesh numbering",
    }


def cpu_oracle_rate(case, steps, budget_s=60.0, warmup=1):
    """Oracle restatement on all host cores: node*level updates/s over a
    bounded number of internal steps after `warmup` untimed ones."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from fesomc import abi, cases
    o = pyoracle.Oracle(case, abi, cases)
    o.step(max(warmup, 0))
    done, t0 = 0, time.perf_counter()
    while done < steps:
        o.step(1)
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    o.close()
    m = case.mesh
    return m.N * m.L * done / dt, done, dt


def run_reference(args, ws, rank):
    """The reference arm: the oracle restatement of the time step (the
    Fortran reference cannot be built in this image) on all host threads,
    its case built by the oracle's own mesh restatement, so that no product
    code is loaded.  --warmup untimed steps (at most 5), then up to --steps
    timed steps within a time budget (a bounded sample of the workload)."""
    if rank != 0:
        return
    cfg = args.config
    case = oracle_case(cfg)
    cpu = host_cpu()
    cores = cpu["threads_available"]
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    budget = min(150.0, 8.0 * max(args.steps, 1))
    warm = min(args.warmup, 5)
    rate, done, dt = cpu_oracle_rate(case, max(args.steps, 1), budget_s=budget, warmup=warm)
    sample = (f"{done} internal steps of {cfg} after {warm} untimed steps ({dt:.1f} s), CPU restatement of the "
              f"reference time step (oracle port) with OpenMP over {cores} threads")
    line = {
        "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus, "steps": done,
        "warmup": warm, "ms_per_step": 1000.0 * dt / max(done, 1), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": workload_config(case, cfg),
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample,
                         "cpu": cpu},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def traffic_from_profiles(kernel):
    """DRAM bytes per launch of 'kernel' from the committed ncu summary
    (line 'traffic_bytes_per_launch <kernel> <bytes>'), or None."""
    pdir = os.path.join(ROOT, "profiles")
    if not os.path.isdir(pdir):
        return None
    for fn in sorted(os.listdir(pdir)):
        if not fn.endswith((".md", ".txt")):
            continue
        with open(os.path.join(pdir, fn)) as f:
            for line in f:
                parts = line.strip().strip("`").split()
                if len(parts) == 3 and parts[0] == "traffic_bytes_per_launch" and parts[1] == kernel:
                    try:
                        return float(parts[2])
                    except ValueError:
                        pass
    return None


def run_ours(args, ws, rank, local):
    from fesomc import abi, build, cases, model, replicas
    if not os.path.exists(abi.LIB_PATH):
        build.build_library()
    lib = abi.load()
    if lib.missing_symbols:
        raise RuntimeError("missing symbols %s" % lib.missing_symbols)
    if ws > 1:
        import torch
        torch.cuda.set_device(local)
    reps = replicas.Replicas(ws, "nccl")
    abi.check(lib.fesomc_gpu_set_device(local), "fesomc_gpu_set_device")
    cfg = args.config
    case = build_case(cfg)
    case.params.fp32_form = 1 if args.fp32_form else 0
    shapes, tune_rep = None, None
    if args.launch_shapes != "default":
        from fesomc import autotune
        try:
            shapes, tune_rep = autotune.shapes_for(case, refresh=args.launch_shapes == "search")
        except Exception as ex:        # timing stays valid with the default shapes
            shapes, tune_rep = None, {"error": repr(ex)}
    if args.shape:
        # explicit knob values on top of the chosen shapes
        from fesomc import autotune
        shapes = dict(shapes or {})
        for kv in args.shape:
            k, v = kv.split("=")
            shapes[k] = int(v)
    g = model.GpuModel(case)
    if shapes:
        autotune.apply(g, shapes)
    m = case.mesh
    units_per_step = m.N * m.L
    barrier, max_over_ranks = reps.barrier, reps.max

    # forcing of the run: constant stress / wind, ramped river runoff per step
    t_next = cases.advance_time(g.time_jd, case.params.dt)
    g.set_forcing(case.forcing_fn(1, t_next))
    g.run(args.warmup)
    # ---- end to end through the C-ABI: per step the host pushes the step's
    # forcing that the reference recomputes each step (rivers_do runoff; the
    # open-boundary tide table is staged by the library from pinned memory),
    # advances one step (status word read back) and reads the energy diagnostic
    rivers = case.mesh.c.n_rivers
    nobn = case.mesh.c.nobn
    h2d = 8 * (rivers + nobn * case.params.Mt)
    d2h = 4 + 4 + 3 * 8
    e = C.c_double()
    barrier()
    t0 = time.perf_counter()
    for k in range(args.steps):
        t_next = cases.advance_time(g.time_jd, case.params.dt)
        fd = case.forcing_fn(g.nstep + 1, t_next)
        f = cases.forcing_struct({"runoff_rivers": fd["runoff_rivers"]})
        abi.check(lib.fesomc_gpu_set_forcing(g.h, C.byref(f)), "set_forcing")
        abi.check(lib.fesomc_gpu_step(g.h, g.nstep + 1), "step")
        abi.check(lib.fesomc_gpu_energy(g.h, C.byref(e)), "energy")
        g.time_jd = t_next
        g.nstep += 1
    t_e2e = max_over_ranks(time.perf_counter() - t0)
    e2e_value = replicas.whole_job_rate(units_per_step, args.steps, ws, t_e2e)
    # ---- device-timed region: K internal steps, inputs resident in HBM; the
    # step's forcing (open-boundary tide, ramped river runoff) is evaluated on
    # the device, so no step copies anything from the host
    device_forcing(lib, abi, g, case)
    barrier()
    ms = C.c_double()
    launches0 = g.kernel_launches()
    with ClockSampler(local) as cs:
        abi.check(lib.fesomc_gpu_time_run(g.h, args.steps, C.byref(ms)), "fesomc_gpu_time_run")
    timed_launches = g.kernel_launches() - launches0
    clocks = cs.summary()
    for _ in range(args.steps):
        g.time_jd = cases.advance_time(g.time_jd, case.params.dt)
    g.nstep += args.steps
    t_dev = max_over_ranks(ms.value / 1000.0)
    barrier()
    value = replicas.whole_job_rate(units_per_step, args.steps, ws, t_dev)
    # ---- per-kernel device times with events (eager launches) for the roofline
    nk = C.c_int32()
    maxk = 64
    names = C.create_string_buffer(32 * maxk)
    kms = (C.c_double * maxk)()
    kbytes = (C.c_double * maxk)()
    klaunch = (C.c_int64 * maxk)()
    nprof = 2
    abi.check(lib.fesomc_gpu_profile(g.h, nprof, maxk, C.byref(nk), names, kms, kbytes, klaunch), "profile")
    kernels = []
    total = 0.0
    for i in range(nk.value):
        nm = names.raw[32 * i: 32 * i + 32].split(b"\0", 1)[0].decode()
        per_step = kms[i] * klaunch[i] / nprof
        total += per_step
        kernels.append({"kernel": nm, "ms_per_launch": kms[i], "launches_per_step": klaunch[i] // nprof,
                        "bytes_per_launch": kbytes[i],
                        "gbs": (kbytes[i] / (kms[i] * 1e-3) / 1e9) if kms[i] > 0 else None,
                        "ms_per_step": per_step})
    for k in kernels:
        k["share"] = k["ms_per_step"] / total if total > 0 else None
    kernels.sort(key=lambda k: -k["ms_per_step"])
    dom = kernels[0]
    peak, peak_kind = measured_peaks()
    achieved = dom["gbs"]
    roof = {"bound": "hbm", "kernel": dom["kernel"], "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": peak_kind,
            "traffic": traffic_from_profiles(dom["kernel"]),
            "bytes_per_launch": dom["bytes_per_launch"], "ms_per_launch": dom["ms_per_launch"],
            "share_of_step": dom["share"]}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * t_dev / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if args.fp32_form else "f64",
        "data": "synthetic",
        "config": workload_config(case, cfg),
        "forcing": "timed region: open-boundary tide and ramped river runoff evaluated on the GPU each step "
                   "(fesomc_gpu_set_device_forcing); e2e: host forcing path, the step's runoff and tide table "
                   "copied from pinned host memory",
        "clocks": clocks,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": 1000.0 * t_e2e / args.steps},
        "gpu_launches": int(timed_launches),
        "launch_shapes": {"source": args.launch_shapes, "shapes": shapes, "tuning": tune_rep},
        "roofline": roof,
        "kernels": [{k: (round(v, 6) if isinstance(v, float) else v) for k, v in kk.items()} for kk in kernels],
    }
    # d3_end sweeps per column in one more step: the mean, and the mean over
    # warps (32 consecutive columns) of their largest count, which a warp
    # waits for
    import numpy as np
    its = np.empty(m.N, dtype=np.int32)
    if lib.fesomc_gpu_d3end_iterations(g.h, 1, its.ctypes.data_as(C.POINTER(C.c_int32))) == 0:
        w = its[: (m.N // 32) * 32].reshape(-1, 32)
        line["d3end_iterations"] = {"mean": float(its.mean()), "max": int(its.max()),
                                    "warp_max_mean": float(w.max(axis=1).mean()),
                                    "lane_efficiency": float(its[: w.size].mean() / w.max(axis=1).mean()),
                                    "step": "the step after the timed region"}
    g.close()
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = host_cpu()
        cores = cpu["threads_available"]
        os.environ.setdefault("OMP_NUM_THREADS", str(cores))
        rate, done, dt = cpu_oracle_rate(oracle_case(cfg), 8, budget_s=30.0)
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port", "cpu": cpu,
                                "sample": f"{done} internal steps of {cfg} after 1 untimed step "
                                          f"({dt:.1f} s), CPU restatement (oracle port, own mesh "
                                          f"restatement) with OpenMP over {cores} threads"}
    reps.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


M2_PERIOD_S = 12.42 * 3600.0      # fv_var.F90:171
TIDAL_DAY_S = 2.0 * M2_PERIOD_S    # two M2 periods


def device_forcing(lib, abi, g, case):
    """Tide and ramped river runoff of the estuary evaluated on the GPU each
    step (the runoff the case's forcing reaches after its 10-day ramp)."""
    import numpy as np
    base = np.ascontiguousarray(case.forcing_fn(1, case.params.time_jd0 + 20.0)["runoff_rivers"], dtype=np.float64)
    abi.check(lib.fesomc_gpu_set_device_forcing(g.h, abi.dptr(base) if base.size else None, 1),
              "fesomc_gpu_set_device_forcing")


def run_compare_forms(args):
    """Chosen (FP32) form against the plain FP64 path on one GPU: both
    models advance the same number of internal steps from the same state
    (device-timed, forcing held), in chunks of --chunk steps; after each
    chunk the prognostic fields are compared.  Prints one JSON line with the
    wall time per simulated tidal day of each form, their ratio, the RMS /
    max differences at the end and after every chunk."""
    import numpy as np
    from fesomc import abi, build, cases, model
    if not os.path.exists(abi.LIB_PATH):
        build.build_library()
    lib = abi.load()
    cfg = args.config
    chunk = args.chunk if args.chunk > 0 else args.steps
    models = []
    shapes_used = {}
    for form in (0, 1):
        case = build_case(cfg)
        case.params.fp32_form = form
        shapes = None
        if args.launch_shapes != "default":
            from fesomc import autotune
            shapes, _ = autotune.shapes_for(case, refresh=args.launch_shapes == "search")
        g = model.GpuModel(case)
        if shapes:
            autotune.apply(g, shapes)
        shapes_used["fp32" if form else "fp64"] = shapes
        t_next = cases.advance_time(g.time_jd, case.params.dt)
        g.set_forcing(case.forcing_fn(1, t_next))
        device_forcing(lib, abi, g, case)
        models.append(g)
    m = case.mesh
    L = m.L
    dt = case.params.dt

    def rms(x):
        return float(np.sqrt(np.mean(x * x)))

    def compare():
        (a, b) = (g.state() for g in models)
        va, vb = (float(np.sum(m.area * (m.depth + s["eta_n"]))) for s in (a, b))
        wet = (a["mask_wd_node"] > 0) & (b["mask_wd_node"] > 0)
        wetn = np.repeat(wet, L)
        return {
            "ssh_rms_m": rms(a["eta_n"][wet] - b["eta_n"][wet]),
            "ssh_max_m": float(np.max(np.abs(a["eta_n"][wet] - b["eta_n"][wet]))),
            "u_rms_m_s": rms(a["U_n"] - b["U_n"]), "u_max_m_s": float(np.max(np.abs(a["U_n"] - b["U_n"]))),
            "v_rms_m_s": rms(a["V_n"] - b["V_n"]), "v_max_m_s": float(np.max(np.abs(a["V_n"] - b["V_n"]))),
            "T_rms_C": rms(a["TF"][wetn] - b["TF"][wetn]),
            "T_max_C": float(np.max(np.abs(a["TF"][wetn] - b["TF"][wetn]))),
            "S_rms_psu": rms(a["SF"][wetn] - b["SF"][wetn]),
            "S_max_psu": float(np.max(np.abs(a["SF"][wetn] - b["SF"][wetn]))),
            "volume_rel": abs(vb - va) / va,
            "wet_nodes_differing": int(np.sum(a["mask_wd_node"] != b["mask_wd_node"])),
        }

    total_ms = [0.0, 0.0]
    done = 0
    per_chunk = []
    failure = None
    while done < args.steps and failure is None:
        n = min(chunk, args.steps - done)
        for form, g in enumerate(models):
            ms = C.c_double()
            rc = lib.fesomc_gpu_time_run(g.h, n, C.byref(ms))
            if rc != abi.FESOMC_OK:
                failure = f"form {form} stopped with {abi.ERRORS.get(rc, rc)} in steps {done + 1}-{done + n}"
                break
            total_ms[form] += ms.value
        if failure is None:
            done += n
            e = compare()
            per_chunk.append({"steps": done, "ssh_rms_m": e["ssh_rms_m"], "T_max_C": e["T_max_C"],
                              "S_max_psu": e["S_max_psu"], "u_max_m_s": e["u_max_m_s"]})
    errors = compare() if failure is None else None
    for g in models:
        g.close()
    steps_per_day = TIDAL_DAY_S / dt
    ms0, ms1 = (t / max(done, 1) for t in total_ms)
    line = {
        "metric": "chosen vs plain FP64 per simulated tidal day", "config": workload_config(case, cfg),
        "steps": done, "simulated_s": done * dt, "m2_cycles": done * dt / M2_PERIOD_S,
        "plain_fp64": {"ms_per_step": ms0, "s_per_tidal_day": ms0 * steps_per_day / 1000.0},
        "chosen_fp32": {"ms_per_step": ms1, "s_per_tidal_day": ms1 * steps_per_day / 1000.0},
        "speedup": ms0 / ms1 if ms1 > 0 else None, "errors_vs_fp64": errors, "per_chunk": per_chunk,
        "launch_shapes": shapes_used,
        "notes": "device-timed graph replay, both runs from the same initial state; stress and wind held, open-boundary "
                 "tide and ramped river runoff evaluated on the GPU each step",
    }
    if failure:
        line["failure"] = failure
    print(json.dumps(line), flush=True)


def run_ensemble(args, ws, rank, local):
    """Perturbed estuary ensemble (--ensemble M members, FP32 form unless
    --fp64): each rank takes its longest-processing-time share of the
    members, advances them concurrently (fesomc_ensemble_run) for --steps
    internal steps after --warmup, then the same steps member after member,
    then packed into one model per level count (packed.PackedCase).  Prints
    one JSON line: aggregate node-level updates/s of the three ways (max
    device time over ranks; `value` is the packed one) and their ratios."""
    from fesomc import abi, build, cases, ensemble, replicas
    if not os.path.exists(abi.LIB_PATH):
        build.build_library()
    lib = abi.load()
    if ws > 1:
        import torch
        torch.cuda.set_device(local)
    reps = replicas.Replicas(ws, "nccl")
    abi.check(lib.fesomc_gpu_set_device(local), "fesomc_gpu_set_device")
    draws = [cases.ensemble_draw(i) for i in range(args.ensemble)]
    costs = [(d["nx"] + 1) * (d["ny"] + 1) * (d["nsigma"] - 1) for d in draws]
    mine = ensemble.lpt_partition(costs, ws)[rank]
    members = []
    for i in mine:
        c = cases.ensemble_member(i)
        c.params.fp32_form = 0 if args.fp64 else 1
        members.append(c)
    ens = ensemble.Ensemble(members)
    ens.run(args.warmup)
    reps.barrier()
    ms_conc, st_conc = ens.run(args.steps, timed=True)
    t_conc = reps.max(ms_conc / 1000.0)
    reps.barrier()
    ms_seq, st_seq = ens.run_one_at_a_time(args.steps)
    t_seq = reps.max(ms_seq / 1000.0)
    ens.close()
    # the same members packed into one model per level count: one launch of
    # every kernel covers all members of a pack
    pens = ensemble.PackedEnsemble(members)
    pens.run(args.warmup)
    reps.barrier()
    ms_pack, st_pack = pens.run(args.steps, timed=True)
    t_pack = reps.max(ms_pack / 1000.0)
    packs = [len(g) for g in pens.groups]
    pens.close()
    reps.close()
    ok = all(s == 0 for s in st_conc + st_seq + st_pack)
    total_units = sum(costs)                     # all members, all ranks
    if rank != 0:
        return
    conc = total_units * args.steps / t_conc
    seq = total_units * args.steps / t_seq
    pack = total_units * args.steps / t_pack
    sizes = [(d["nx"] + 1) * (d["ny"] + 1) for d in draws]
    line = {
        "metric": "aggregate node\u00b7level updates/s, ensemble", "unit": "node-level updates/s",
        "value": pack, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * t_pack / args.steps, "higher_is_better": True, "scaling": "strong",
        "dtype": "f64" if args.fp64 else "f32 (2D sub-cycle f64)", "data": "synthetic",
        "config": {"workload": f"{args.ensemble} perturbed estuary members (cfg0 generator, 300 m), "
                               f"{min(sizes)}-{max(sizes)} nodes, 11/21 sigma levels, M2 amplitude +-20 %, "
                               f"phase +-15 deg, stress 0-0.2 N/m2 in random directions, noise 0-1 m",
                   "members": args.ensemble, "nodes_total": sum(sizes), "node_levels_per_step": total_units,
                   "this_rank_members": len(mine), "parallelism": f"LPT share of members per GPU ({ws})"},
        "packed": {"value": pack, "ms_per_step": 1000.0 * t_pack / args.steps, "members_per_pack": packs},
        "concurrent": {"value": conc, "ms_per_step": 1000.0 * t_conc / args.steps},
        "one_at_a_time": {"value": seq, "ms_per_step": 1000.0 * t_seq / args.steps},
        "packed_over_one_at_a_time": pack / seq if seq > 0 else None,
        "concurrent_over_one_at_a_time": conc / seq if seq > 0 else None,
        "all_members_ok": ok,
        "notes": "value: members packed into one model per level count (one launch of every kernel per pack, "
                 "packs side by side); concurrent: members on their own streams and step graphs, one step of "
                 "every member per round; stress and wind held, tide and river runoff evaluated on the GPU "
                 "each step",
    }
    print(json.dumps(line), flush=True)


def stress_forcing(case, tau, theta):
    """Uniform stress tau (N/m2) towards angle theta and the 10 m wind that
    carries it (rho_air 1.3, C_D 1.3e-3), as the estuary cases set them."""
    import math
    import numpy as np
    m = case.mesh
    w = math.sqrt(tau / (1.3 * 1.3e-3)) if tau > 0 else 0.0
    return {"taux": np.full(m.E, tau * math.cos(theta)), "tauy": np.full(m.E, tau * math.sin(theta)),
            "windx": np.full(m.N, w * math.cos(theta)), "windy": np.full(m.N, w * math.sin(theta))}


def mixed_layer_depth(case, state, dT=0.2):
    """Depth (m) where temperature first differs from the top layer by dT
    (temperature criterion), per wet node; the column depth if nowhere."""
    import numpy as np
    m = case.mesh
    L = m.L
    H = np.maximum(m.depth + state["eta_n"], case.params.Dmin)
    zmid = 0.5 * ((1.0 - m.sigma[:-1]) + (1.0 - m.sigma[1:]))
    T = state["TF"].reshape(-1, L)
    off = np.abs(T - T[:, :1]) > dT
    first = np.where(off.any(axis=1), off.argmax(axis=1), L - 1)
    return zmid[first] * H


def run_closure(args):
    """Learned closure on the cfg1 mesh (cfg4): columns harvested from the
    plain closure under seeded forcing draws (stress 0-0.3 N/m2 in a random
    direction, surface heat flux -200..+100 W/m2), trained on the GPU, then
    one tidal day of cfg4 forcing (0.15 N/m2, -100 W/m2) with the FP32 form +
    learned closure against the plain FP64 path.  One JSON line: training,
    fallback rate, judge error, mixed-layer depth, SSH / T / S errors and time
    per simulated tidal day of both."""
    import math
    import numpy as np
    from fesomc import abi, build, cases, closure, model
    if not os.path.exists(abi.LIB_PATH):
        build.build_library()
    lib = abi.load()
    rng = np.random.default_rng(20261204)
    heat = {"qns": -100.0, "qsr": 0.0, "emp": 0.0}
    case = cases.estuary(args.config, atm=heat)
    m = case.mesh
    base = np.ascontiguousarray(case.forcing_fn(1, case.params.time_jd0 + 20.0)["runoff_rivers"], dtype=np.float64)

    def new_model(fp32, forcing):
        case.params.fp32_form = 1 if fp32 else 0
        g = model.GpuModel(case)
        f = case.forcing_fn(1, cases.advance_time(g.time_jd, case.params.dt))
        f.update(forcing)
        g.set_forcing(f)
        abi.check(lib.fesomc_gpu_set_device_forcing(g.h, abi.dptr(base), 1), "fesomc_gpu_set_device_forcing")
        return g

    c = closure.Closure(m.NS, capacity=args.lc_capacity)
    rules = [r for r in args.lc_rules.split(",") if r]
    t0 = time.perf_counter()
    draws = []
    for k in range(args.lc_draws):
        tau, th, qns = rng.uniform(0.0, 0.3), rng.uniform(0.0, 2 * math.pi), rng.uniform(-200.0, 100.0)
        draws.append({"tau": tau, "theta": th, "qns": qns})
        f = stress_forcing(case, tau, th)
        f["qns"] = np.full(m.N, qns)
        g = new_model(True, f)
        c.harvest(g, args.lc_spinup, args.lc_spinup + 1)          # spin-up, nothing harvested
        c.harvest(g, args.lc_harvest_steps, args.lc_every)
        g.close()
    harvest_s = time.perf_counter() - t0
    c.fit()
    t0 = time.perf_counter()
    losses = c.train(args.lc_epochs, batch=8192, lr=args.lc_lr, seed=3)
    train_s = time.perf_counter() - t0
    steps = args.steps
    cfg4 = stress_forcing(case, 0.15, 0.5 * math.pi)
    runs = {}
    for name, fp32, lc in (("plain_fp64", False, False), ("fp32_plain", True, False), ("fp32_learned", True, True)):
        g = new_model(fp32, cfg4)
        if lc:
            c.set_rules(unstable="unstable" in rules, boundary="boundary" in rules)
            c.attach(g, judge_every=args.lc_judge, bf16=True)
        ms = C.c_double()
        rc = lib.fesomc_gpu_time_run(g.h, steps, C.byref(ms))
        st = g.state()
        rep = closure.Closure.stats(g) if lc else None
        g.close()
        runs[name] = {"rc": rc, "ms_per_step": ms.value / steps, "state": st, "stats": rep}
    ref = runs["plain_fp64"]["state"]
    wet = ref["mask_wd_node"] > 0
    wetn = np.repeat(wet, m.L)
    mld_ref = mixed_layer_depth(case, ref)

    def errors(s):
        mld = mixed_layer_depth(case, s)
        return {"ssh_rms_m": float(np.sqrt(np.mean((s["eta_n"][wet] - ref["eta_n"][wet]) ** 2))),
                "T_rms_C": float(np.sqrt(np.mean((s["TF"][wetn] - ref["TF"][wetn]) ** 2))),
                "T_max_C": float(np.max(np.abs(s["TF"][wetn] - ref["TF"][wetn]))),
                "S_rms_psu": float(np.sqrt(np.mean((s["SF"][wetn] - ref["SF"][wetn]) ** 2))),
                "S_max_psu": float(np.max(np.abs(s["SF"][wetn] - ref["SF"][wetn]))),
                "mld_mean_m": float(np.mean(mld[wet])), "mld_rms_diff_m": float(np.sqrt(np.mean((mld[wet] - mld_ref[wet]) ** 2)))}

    day = TIDAL_DAY_S / case.params.dt
    out = {"metric": "learned closure (cfg4) vs plain FP64 per simulated tidal day", "config": workload_config(case, args.config),
           "forcing": "cfg4: uniform cross-shore stress 0.15 N/m2, non-solar surface heat flux -100 W/m2, tide and ramped river on the GPU",
           "training": {"draws": draws, "columns": c.harvested(), "harvest_s": harvest_s, "epochs": args.lc_epochs,
                        "train_s": train_s, "loss_per_epoch": [float(x) for x in losses], "parameters": c.nparams},
           "fallback_rules": rules or ["envelope only"],
           "steps": steps, "simulated_s": steps * case.params.dt, "mld_mean_plain_m": float(np.mean(mld_ref[wet]))}
    for name, r in runs.items():
        e = {"rc": r["rc"], "ms_per_step": r["ms_per_step"], "s_per_tidal_day": r["ms_per_step"] * day / 1000.0}
        if name != "plain_fp64":
            e["errors_vs_plain_fp64"] = errors(r["state"])
            e["speedup_vs_plain_fp64"] = runs["plain_fp64"]["ms_per_step"] / r["ms_per_step"]
        if r["stats"]:
            st = r["stats"]
            e["closure"] = dict(st, fallback_rate=(st["out_of_envelope"] + st["dry_columns"]) /
                                max(1, st["wet_columns"] + st["dry_columns"]),
                                envelope_fallback_rate=st["out_of_envelope"] / max(1, st["wet_columns"]))
        out[name] = e
    c.close()
    print(json.dumps(out), flush=True)


def run_lc_infer(args):
    """The learned closure's inference alone: the BF16 tensor-core kernel and
    the FP32 kernels on --lc-infer device-resident columns of the cfg1 shape
    (21 levels: 66 inputs, 21 outputs), random weights, device-timed; FLOP
    per column 2 (66*256 + 2*256*256 + 256*21)."""
    from fesomc import closure
    c = closure.Closure(21)
    n = args.lc_infer
    flop = 2.0 * (c.n_in * 256 + 2 * 256 * 256 + 256 * c.n_out) * n
    ms_tc = c.time(n, reps=max(args.steps, 1), bf16=True)
    ms_32 = c.time(n, reps=max(min(args.steps, 5), 1), bf16=False)
    c.close()
    peak = None
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    kind = "fallback"
    if os.path.exists(pk):
        with open(pk) as f:
            peak = json.load(f).get("bf16_tflops")
            kind = "measured"
    peak = peak or 1590.0
    tf = flop / (ms_tc * 1e-3) / 1e12
    print(json.dumps({"metric": "learned-closure inference", "columns": n, "flop_per_pass": flop,
                      "bf16_tcgen05": {"ms": ms_tc, "tflops": tf, "frac_of_peak": tf / peak, "peak_tflops": peak,
                                       "peak_source": kind},
                      "fp32_simt": {"ms": ms_32, "tflops": flop / (ms_32 * 1e-3) / 1e12}}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="cfg1")
    ap.add_argument("--chunk", type=int, default=0, help="--compare-forms: steps between comparisons")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ensemble", type=int, default=0, help="run the perturbed estuary ensemble of this many members")
    ap.add_argument("--fp64", action="store_true", help="--ensemble: members in the plain FP64 path")
    ap.add_argument("--compare-forms", action="store_true",
                    help="time the FP32 form against the plain FP64 path and report their differences")
    ap.add_argument("--fp32-form", action="store_true",
                    help="run the FP32 form (level fields and 3D arithmetic in FP32, 2D sub-cycle in FP64)")
    ap.add_argument("--closure", action="store_true",
                    help="learned closure report (cfg4): harvest, train, one tidal day against plain FP64")
    ap.add_argument("--lc-draws", type=int, default=6)
    ap.add_argument("--lc-spinup", type=int, default=90)
    ap.add_argument("--lc-harvest-steps", type=int, default=60)
    ap.add_argument("--lc-every", type=int, default=20)
    ap.add_argument("--lc-capacity", type=int, default=20_000_000)
    ap.add_argument("--lc-epochs", type=int, default=4)
    ap.add_argument("--lc-lr", type=float, default=1e-3)
    ap.add_argument("--lc-judge", type=int, default=100)
    ap.add_argument("--lc-rules", default="unstable,boundary",
                    help="closure fallback rules beyond the envelope: comma-separated of unstable, boundary")
    ap.add_argument("--lc-infer", type=int, default=0, help="time the closure inference on this many columns")
    ap.add_argument("--mesh-order", action="store_true",
                    help="store the mesh in its own numbering on the device (default: along a Hilbert curve)")
    ap.add_argument("--launch-shapes", default="tuned", choices=["default", "tuned", "search"],
                    help="kernel launch shapes: built-in defaults, the autotuner's (cached, searched when "
                         "absent), or a fresh search")
    ap.add_argument("--shuffle", type=int, default=None, help="number the mesh's nodes and elements at random (seed)")
    ap.add_argument("--shape", action="append", default=[],
                    help="a launch-shape knob set explicitly, NAME=VALUE (repeatable), e.g. d3end_arrays=3")
    args = ap.parse_args()
    if not args.mesh_order:
        BUILD_OPTS["sfc_order"] = 1
    if args.shuffle is not None:
        BUILD_OPTS["shuffle"] = args.shuffle
    ws, rank, local = dist_info()
    if args.lc_infer > 0:
        run_lc_infer(args)
        return
    if args.closure:
        run_closure(args)
        return
    if args.compare_forms:
        run_compare_forms(args)
        return
    if args.ensemble > 0:
        ws, rank, local = dist_info()
        run_ensemble(args, ws, rank, local)
        return
    if args.impl == "reference":
        run_reference(args, ws, rank)
    else:
        run_ours(args, ws, rank, local)


if __name__ == "__main__":
    main()
