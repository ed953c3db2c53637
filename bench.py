"""Benchmark: RK3 cell-steps/s of the compressible-LES right-hand side on a
jittered-lattice periodic Voronoi mesh (200^3 = 8M cells by default), FP64,
one replica per GPU.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cgx|reference]

Prints one JSON line (rank 0).  value = whole-job cell-steps/s from CUDA
events on the solver's stream around K graph-replayed steps (max over ranks);
e2e = the same metric through the C ABI with host buffers (pinned host state
copied in and read back every step, cgx_set_state + cgx_step_out);
roofline = the face-flux kernel pair's
algorithmic bytes per launch over its launch time, timed by CUDA events
recorded around the two kernels inside the timed steps, against the
measured HBM copy bandwidth; cpu_baseline = the CPU oracle on the host cores
on a bounded sample.  `--impl reference` times the reference's CPU path (the
oracle built on the reference's own flux header when available) instead.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RK3 cell-steps/s @8M cells FP64 vs mixed; served solves/s, p50/p99 latency"
UNIT = "cell-steps/s"
JITTER = 0.25
SEED = 1234


def bytes_model(e, f):
    """Algorithmic bytes per cell: whole RK3 step (3 stages + once-per-step
    work) and one face-flux (calcRhs) launch.  Each array element counted
    once per kernel pass, neighbour gathers assumed cached:
      per stage  504 + 56e + 96f   (state/RK 208, packed state 80,
                                    gradient 168 + 56f, extended faces 56e,
                                    compact extras 40f + 48)
      per step   320 + 8e + 32f    (SGS/properties 200, Gibbs sensor 40 + 8e,
                                    CFL 40 + 32f, totals 40)
      calcRhs    56e + 40f + 200   (extended faces 56e, compact geometry 40f,
                                    lagged properties 48, packed state 40,
                                    dudx 72, rhs write 40)
    calcRhs is two kernels: k_rhs_ext (extended faces 56e, packed state 40,
    rhs write 40) and k_rhs_comp (compact geometry 40f, lagged properties 48,
    dudx 72)."""
    step = 3 * (504 + 56 * e + 96 * f) + (320 + 8 * e + 32 * f)
    rhs = 56 * e + 40 * f + 200
    return step, rhs, {"k_rhs_ext": 56 * e + 80, "k_rhs_comp": 40 * f + 120}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.f = None

    def __enter__(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.f:
            return None
        try:
            rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        except Exception:
            return None
        finally:
            try:
                os.unlink(self.f.name)
            except Exception:
                pass
        rows = [[c.strip() for c in r] for r in rows if len(r) >= 9]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, nm in enumerate(names):
                if r[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def cpu_baseline(seconds=12.0, n=48, lib_kind="reference"):
    """The CPU oracle on a jittered n^3 box with all host threads: RK3 steps
    until `seconds` of CPU work have run.  Returns the cpu_baseline object."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Oracle, ref_available
    from nextgen_b200 import cases
    from nextgen_b200.meshgen import PeriodicBoxMesh
    cores = os.cpu_count() or 1
    m = PeriodicBoxMesh(n, jitter=JITTER, seed=SEED)
    prm = cases.tgv_params()
    rho, u, p = cases.tgv_state(m.x_cv[: m.ncv], prm)
    use_ref = lib_kind == "reference" and ref_available()
    o = Oracle(m, prm, nparts=cores, reference=use_ref)
    o.set_state_primitive(rho, u, p)
    o.init_complete()
    o.step(1)
    steps = 0
    t0 = time.perf_counter()
    while True:
        o.step(1)
        steps += 1
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    what = ("the oracle built on the reference's own IdealGasSolverFlux.hpp/States.hpp/RkWeights.hpp "
            "(compiled in place) with the reference's rank-parallel face loops restated"
            if use_ref else "the oracle (restated reference hot path)")
    return {"value": m.ncv * steps / el, "unit": UNIT, "cores": cores,
            "kind": "reference" if use_ref else "port",
            "sample": "%d RK3 steps of %s on a jittered %d^3 periodic Voronoi box (%d cells, TGV Ma 0.1), "
                      "%d OpenMP ranks over contiguous cell ranges" % (steps, what, n, m.ncv, cores)}


def served_stream(nreq=32, seed=4242, budget_gb=60):
    """The served configuration: requests arrive as a seeded Poisson process;
    each is its own jittered-lattice periodic Voronoi box (seed per request)
    with edge uniform in [16, 96], Taylor-Green or random-solenoidal (k0 = 4)
    initial state, Mach uniform in [0.1, 0.5], steps uniform in [200, 2000],
    FP64 or mixed.  Requests bring the mesher's compact mesh (made before the
    stream starts, as a mesher upstream would); admission builds the
    operators on the GPU, uploads the device mesh and prepares the case on a
    preparer thread while the GPU steps the resident cases.  The rate is twice
    the GPU's estimated service rate, so the device stays saturated.  The same
    requests also run one at a time (operator build, upload, initComplete,
    steps, state read-back) at their own precision and on the plain FP64
    path."""
    from nextgen_b200 import cases, cgx, serve
    from nextgen_b200.meshgen import PeriodicBoxMesh
    rng = np.random.default_rng(seed)
    edges = [int(e) for e in rng.integers(16, 97, size=nreq)]
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    reqs = []
    for k, n in enumerate(edges):
        compact = PeriodicBoxMesh(n, jitter=JITTER, seed=SEED + 7919 * (k + 1), nthreads=cores, compact_only=True)
        Ma = float(rng.uniform(0.1, 0.5))
        if rng.random() < 0.5:
            prm = cases.tgv_params(Ma=Ma, Re=float(rng.uniform(400, 3200)))
            rho, u, p = cases.tgv_state(compact.x_cv[: compact.ncv], prm)
            kind = "tgv"
        else:
            prm = cases.hit_params(Mt=Ma)
            rho, u, p = cases.hit_state(n, prm, Mt=Ma, k0=4.0, seed=4321 + k)
            kind = "solenoidal"
        prm.check_interval = 20
        prec = cgx.CGX_FP64 if rng.random() < 0.5 else cgx.CGX_MIXED
        r = serve.Request(k, None, prm, rho, u, p, int(rng.integers(200, 2001)), prec, compact=compact)
        r.kind = kind
        reqs.append(r)
    t_mesh = time.perf_counter() - t0
    total_cs = sum(r.cell_steps for r in reqs)
    rate = 2.0 * 2.0e8 / (total_cs / nreq)  # requests/s: twice the estimated service rate
    for r, a in zip(reqs, serve.poisson_arrivals(nreq, rate, seed=seed + 1)):
        r.arrival = float(a)
    out = serve.serve(reqs, hbm_budget=int(budget_gb * (1 << 30)), chunk=16, keep_state=False)
    # one at a time: the FP64 requests once (the same runs serve both
    # baselines), the mixed ones at their own precision and on the plain FP64
    # path
    f64 = [r for r in reqs if r.precision == cgx.CGX_FP64]
    mix = [r for r in reqs if r.precision == cgx.CGX_MIXED]
    a, _ = serve.run_sequential(f64, precision=cgx.CGX_FP64) if f64 else ({"seconds": 0.0}, None)
    b, _ = serve.run_sequential(mix, precision=cgx.CGX_MIXED) if mix else ({"seconds": 0.0}, None)
    c, _ = serve.run_sequential(mix, precision=cgx.CGX_FP64) if mix else ({"seconds": 0.0}, None)
    for r in reqs:
        r.compact.close()
    own = total_cs / (a["seconds"] + b["seconds"])
    plain = total_cs / (a["seconds"] + c["seconds"])
    out.update({"sequential_own_precision_cell_steps_per_s": own,
                "sequential_plain_fp64_cell_steps_per_s": plain,
                "sequential_runs": {"requests": len(reqs), "fp64_requests_s": a["seconds"],
                                      "mixed_requests_own_precision_s": b["seconds"],
                                      "mixed_requests_fp64_s": c["seconds"]},
                "speedup_vs_sequential_own_precision": out["cell_steps_per_s"] / own,
                "speedup_vs_sequential_plain_fp64": out["cell_steps_per_s"] / plain,
                "poisson_rate_per_s": rate, "compact_mesh_build_s": round(t_mesh, 2),
                "how": "host wall clock; admission (GPU operator build, device mesh, case set-up) inside the "
                       "served window and inside each sequential run; the mesher's compact meshes made before",
                "mix": {"fp64": sum(r.precision == cgx.CGX_FP64 for r in reqs),
                        "mixed": sum(r.precision == cgx.CGX_MIXED for r in reqs),
                        "distinct_meshes": nreq, "edges": edges,
                        "steps_total": int(sum(r.nsteps for r in reqs))}})
    return out


def workload_config(n, cells, e, f):
    """The `config` object of both arms: what the workload is, nothing about
    how it was run."""
    return {"workload": "jittered-lattice (+/-0.25h) periodic Voronoi %d^3 = %d cells per GPU, "
                        "Taylor-Green Ma 0.1 Re 1600 Pr 0.71, Vreman SGS, FP64 RK3 at CFL 0.8" % (n, cells),
            "cells": int(cells), "e_per_cell": float(e), "f_per_cell": float(f), "precision": "fp64"}


def run_reference(args):
    """The reference's CPU path on this arm's workload: the oracle built on the
    reference's own flux, state and RK headers (the reference binary stops at
    its licence check), on all host threads as contiguous cell ranges like
    MPI ranks, stepping the same 200^3 mesh and state W + K RK3 steps; K
    timed.  A 1-core leg times one step of the single-range oracle on a
    jittered 64^3 sample.  Rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Oracle, ref_available
    from nextgen_b200 import cases
    from nextgen_b200.meshgen import PeriodicBoxMesh
    cores = os.cpu_count() or 1
    n = args.n
    t0 = time.perf_counter()
    m = PeriodicBoxMesh(n, jitter=JITTER, seed=SEED, nthreads=cores)
    t_mesh = time.perf_counter() - t0
    prm = cases.tgv_params()
    rho, u, p = cases.tgv_state(m.x_cv[: m.ncv], prm)
    use_ref = ref_available()
    o = Oracle(m, prm, nparts=cores, reference=use_ref)
    o.set_state_primitive(rho, u, p)
    o.init_complete()
    config = workload_config(n, m.ncv, m.e_per_cell, m.f_per_cell)
    del rho, u, p
    if args.warmup:
        o.step(args.warmup)
    t0 = time.perf_counter()
    o.step(args.steps)
    el = time.perf_counter() - t0
    v = m.ncv * args.steps / el
    o.close()
    m.close()
    # one core, the single-range oracle (the reference's serial order)
    s1 = PeriodicBoxMesh(64, jitter=JITTER, seed=SEED, nthreads=cores)
    prm1 = cases.tgv_params()
    o1 = Oracle(s1, prm1, nparts=1, reference=use_ref)
    o1.set_state_primitive(*cases.tgv_state(s1.x_cv[: s1.ncv], prm1))
    o1.init_complete()
    try:
        os.sched_setaffinity(0, {sorted(os.sched_getaffinity(0))[0]})
    except (AttributeError, OSError):
        pass
    t1 = time.perf_counter()
    o1.step(1)
    el1 = time.perf_counter() - t1
    one_core = {"value": s1.ncv / el1, "unit": UNIT, "cores": 1,
                "sample": "1 RK3 step of the single-range oracle on a jittered 64^3 box (%d cells)" % s1.ncv}
    what = ("oracle built on the reference's own IdealGasSolverFlux.hpp/States.hpp/RkWeights.hpp compiled in place"
            if use_ref else "oracle port of the reference hot path")
    out = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic", "config": config,
           "setup": {"parallelism": "cpu %d threads (cell ranges as MPI ranks)" % cores,
                     "mesh_build_s": round(t_mesh, 2)},
           "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "reference" if use_ref else "port",
                            "sample": "%d timed RK3 steps (after %d warm-up) of the %s on the same %d-cell "
                                      "mesh and state as the GPU arm, %d OpenMP ranks"
                                      % (args.steps, args.warmup, what, config["cells"], cores)},
           "cpu_1core": one_core,
           "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)
    return 0


def run_cgx(args):
    import torch
    from nextgen_b200 import cases, cgx, dist
    from nextgen_b200.meshgen import PeriodicBoxMesh

    rank, world, local = dist.env_rank()
    if world > 1:
        torch.cuda.set_device(local)
        dist.init("nccl")
    device = local
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    if args.device_ops:
        # the mesher's compact output, operators built on this rank's GPU
        # (bit-identical to the host generator's)
        from nextgen_b200.meshgen import DeviceOperatorMesh
        compact = PeriodicBoxMesh(args.n, jitter=JITTER, seed=SEED, nthreads=max(1, cores // world),
                                  compact_only=True)
        m = DeviceOperatorMesh(compact, device=device)
        compact.close()
    else:
        m = PeriodicBoxMesh(args.n, jitter=JITTER, seed=SEED, nthreads=max(1, cores // world))
    t_mesh = time.perf_counter() - t0
    prm = cases.tgv_params()
    rho, u, p = cases.tgv_state(m.x_cv[: m.ncv], prm)
    t0 = time.perf_counter()
    gm = cgx.Mesh(m, device=device)
    t_up = time.perf_counter() - t0
    st = gm.stats()
    e, f = st.e_per_cell, st.f_per_cell
    N = m.ncv
    vol_cv = np.array(m.vol_cv)
    m.close()

    solvers = {}
    res = {}
    precs = [("fp64", cgx.CGX_FP64)] + ([("mixed", cgx.CGX_MIXED)] if not args.no_mixed else [])
    for prec_name, prec in precs:
        s = cgx.Solver(gm, prm, prec)
        s.set_state_primitive(rho, u, p)
        s.initComplete()
        if args.warmup:
            s.step(args.warmup)
        dist.barrier()
        s.synchronize()
        n0 = s.launch_count()
        with ClockSampler(device) as clk:
            # the face kernels are timed inside these steps (events in the step graph)
            ms, face = s.step_profiled(args.steps)
        s.synchronize()
        dist.barrier()
        launches = s.launch_count() - n0
        ms_max = dist.max_over_ranks(ms)
        # the other kernels' launch times from back-to-back launches after the
        # timed region; the face kernels' from inside it
        kt = s.kernel_times(reps=3)
        kt.update(face)
        res[prec_name] = {"ms": ms_max, "launches": launches, "clocks": clk.summary(),
                          "kernel_ms": kt, "tuning": s.tuning()}
        solvers[prec_name] = s

    s = solvers["fp64"]
    ktimes = res["fp64"]["kernel_ms"]
    tuning = res["fp64"]["tuning"]
    mixed = None
    if "mixed" in solvers:
        # both forms advanced W + K steps from the same initial state:
        # errors of the mixed form against the FP64 path
        r64, u64, _ = s.get_state()
        r32, u32, _ = solvers["mixed"].get_state()
        p64 = s.primitive()[0]
        p32 = solvers["mixed"].primitive()[0]
        vol = np.array(vol_cv)
        ke64 = 0.5 * (r64 * (u64 * u64).sum(1) * vol).sum()
        ke32 = 0.5 * (r32 * (u32 * u32).sum(1) * vol).sum()
        ke0 = 0.5 * (rho * (u * u).sum(1) * vol).sum()
        du = u32 - u64
        pf = p64 - p64.mean()
        ms_mixed = res["mixed"]["ms"]
        mixed = {"value": world * N * args.steps / (ms_mixed * 1e-3), "unit": UNIT,
                 "ms_per_step": ms_mixed / args.steps,
                 "speedup_vs_fp64": res["fp64"]["ms"] / ms_mixed,
                 "kernel_ms": res["mixed"]["kernel_ms"], "tuning": res["mixed"]["tuning"],
                 "gpu_launches": res["mixed"]["launches"], "clocks": res["mixed"]["clocks"],
                 "error_vs_fp64_after_steps": args.warmup + args.steps,
                 "u_l2_rel": float(np.sqrt((du ** 2).mean() / (u64 ** 2).mean())),
                 "u_linf_rel": float(np.abs(du).max() / np.abs(u64).max()),
                 "p_l2_rel_fluct": float(np.sqrt(((p32 - p64) ** 2).mean() / max((pf ** 2).mean(), 1e-300))),
                 "p_linf_rel_fluct": float(np.abs(p32 - p64).max() / max(np.abs(pf).max(), 1e-300)),
                 "ke_rel": float(abs(ke32 - ke64) / ke64),
                 "ke_decay_rel": float(abs(ke32 - ke64) / max(abs(ke0 - ke64), 1e-300))}
    step_bytes, rhs_bytes, split_bytes = bytes_model(e, f)
    peak, peak_kind = measured_peaks()
    ms_step = res["fp64"]["ms"] / args.steps
    value = world * N * args.steps / (res["fp64"]["ms"] * 1e-3)
    achieved = rhs_bytes * N / (dist.max_over_ranks(ktimes["rhs"]) * 1e-3) / 1e9

    # e2e: the C-ABI calls a host solver makes each step, with host buffers
    r_h = torch.empty(N, dtype=torch.float64, pin_memory=True)
    u_h = torch.empty(3 * N, dtype=torch.float64, pin_memory=True)
    e_h = torch.empty(N, dtype=torch.float64, pin_memory=True)
    s.get_state_ptr(r_h.data_ptr(), u_h.data_ptr(), e_h.data_ptr())
    ke = max(1, min(args.steps, args.e2e_steps))
    dist.barrier()
    t0 = time.perf_counter()
    for _ in range(ke):
        s.set_state_ptr(r_h.data_ptr(), u_h.data_ptr(), e_h.data_ptr())
        s.step_out_ptr(1, r_h.data_ptr(), u_h.data_ptr(), e_h.data_ptr())
    el = time.perf_counter() - t0
    el = dist.max_over_ranks(el)
    e2e = world * N * ke / el
    # the same loop with pageable host arrays (what a host solver's new[]
    # arrays are): the library stages them through its pinned chunks
    r_p, u_p, e_p = np.empty(N), np.empty(3 * N), np.empty(N)
    s.get_state_ptr(r_p.ctypes.data, u_p.ctypes.data, e_p.ctypes.data)
    dist.barrier()
    t0 = time.perf_counter()
    for _ in range(ke):
        s.set_state_ptr(r_p.ctypes.data, u_p.ctypes.data, e_p.ctypes.data)
        s.step_out_ptr(1, r_p.ctypes.data, u_p.ctypes.data, e_p.ctypes.data)
    el_p = dist.max_over_ranks(time.perf_counter() - t0)
    e2e_pageable = world * N * ke / el_p

    # DRAM traffic per cell of each face kernel from a committed ncu capture
    # (dram__bytes_read.sum + dram__bytes_write.sum per launch / cells),
    # scaled to this mesh's cell count
    traffic, per_kernel_dram = None, {}
    tp = os.path.join(ROOT, "profiles", "rhs_dram_bytes_per_cell.json")
    if os.path.exists(tp):
        try:
            tj = json.load(open(tp))
            traffic = float(tj["dram_bytes_per_cell"]) * N
            per_kernel_dram = {k: float(tj[k]) for k in ("k_rhs_ext", "k_rhs_comp") if k in tj}
        except Exception:
            traffic = None
    kernels = {}
    for kname, key in (("k_rhs_ext", "ext"), ("k_rhs_comp", "comp")):
        if key in ktimes and ktimes[key] > 0:
            kernels[kname] = {"launch_ms": ktimes[key], "algorithmic_bytes_per_cell": split_bytes[kname],
                              "achieved_gbs": split_bytes[kname] * N / (ktimes[key] * 1e-3) / 1e9,
                              "dram_bytes_per_cell": per_kernel_dram.get(kname)}
            if per_kernel_dram.get(kname):
                # the kernel's actual DRAM traffic over its in-step launch time
                kernels[kname]["traffic_gbs"] = per_kernel_dram[kname] * N / (ktimes[key] * 1e-3) / 1e9
                kernels[kname]["traffic_frac"] = kernels[kname]["traffic_gbs"] / peak

    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args.n, N, e, f),
        "setup": {"l2": "inputs larger than L2 (%.1f GB mesh on device)" % (st.device_bytes / 1e9),
                  "device_bytes_per_cell": st.device_bytes / N,
                  "parallelism": "replicas x%d" % world,
                  "mesh_build_s": round(t_mesh, 2), "mesh_upload_s": round(t_up, 2),
                  "mesh_operators": "gpu (cgx_operators_build)" if args.device_ops else "host generator"},
        "e2e_pageable_host_arrays": {"value": e2e_pageable, "unit": UNIT},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": 40 * N, "d2h_bytes_per_step": 40 * N,
                "steps": ke, "how": "per step: cgx_set_state (pinned host -> device), then cgx_step_out(1) "
                                    "(the step, its new state copied device -> pinned host beside the step's "
                                    "last gradient and step-end kernels); host wall clock"},
        "gpu_launches": res["fp64"]["launches"],
        "clocks": res["fp64"]["clocks"],
        "roofline": {"bound": "hbm", "kernel": "k_rhs_ext + k_rhs_comp (calcRhsBase)", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "peak_kind": peak_kind, "algorithmic_bytes_per_cell": rhs_bytes,
                     "traffic_achieved": achieved * traffic / (rhs_bytes * N) if traffic else None,
                     "traffic_frac": achieved * traffic / (rhs_bytes * N) / peak if traffic else None,
                     "launch_ms": ktimes["rhs"], "kernels": kernels},
        "step_roofline": {"bytes_per_cell_step": step_bytes, "achieved": value / world * step_bytes / 1e9,
                          "frac": value / world * step_bytes / 1e9 / peak, "unit": "GB/s"},
        "kernel_ms": ktimes,
        "tuning": tuning,
        "mixed": mixed,
    }
    for k in list(solvers):
        solvers[k].close()
    solvers = {}
    if rank == 0 and world == 1 and args.accuracy_steps > 0:
        out["accuracy"] = accuracy_block(gm, args.n, vol_cv, (rho, u, p), args.accuracy_steps)
    gm.close()
    if rank == 0 and world == 1 and args.batch_steps > 0:
        out["batch64"] = batch64_block(args.batch_steps)
    if rank == 0 and world == 1 and not args.no_served:
        out["served"] = served_stream(nreq=args.served_requests)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(seconds=args.cpu_seconds, n=args.cpu_n)
    if rank == 0:
        print(json.dumps(out), flush=True)
    dist.finalize()
    return 0


def _errors(vol, ref, got, init):
    """Velocity, pressure (fluctuation) and kinetic-energy errors of `got`
    against `ref`: (rho, u, p) triples on the same mesh."""
    r64, u64, p64 = ref
    r32, u32, p32 = got
    rho0, u0 = init
    ke = lambda r, u: 0.5 * (r * (u * u).sum(1) * vol).sum()
    ke64, ke32, ke0 = ke(r64, u64), ke(r32, u32), ke(rho0, u0)
    du = u32 - u64
    pf = p64 - p64.mean()
    return {"u_l2_rel": float(np.sqrt((du ** 2).mean() / (u64 ** 2).mean())),
            "u_linf_rel": float(np.abs(du).max() / np.abs(u64).max()),
            "p_l2_rel_fluct": float(np.sqrt(((p32 - p64) ** 2).mean() / max((pf ** 2).mean(), 1e-300))),
            "p_linf_rel_fluct": float(np.abs(p32 - p64).max() / max(np.abs(pf).max(), 1e-300)),
            "ke_rel": float(abs(ke32 - ke64) / ke64),
            "ke_decay_fp64": float((ke0 - ke64) / ke0),
            "ke_decay_rel_err": float(abs(ke32 - ke64) / max(abs(ke0 - ke64), 1e-300))}


KE_DECAY_BOUND = 1e-5  # the mixed form's kinetic-energy (decay) error bound against FP64


def accuracy_block(gm, n, vol, tgv, K):
    """The mixed-precision form against the FP64 path on the device mesh `gm`
    of the jittered n^3 lattice: the Ma 0.1 Taylor-Green state `tgv` = (rho,
    u, p) and the Mt 0.3 random-solenoidal state, each advanced K RK3 steps
    at CFL 0.8 by both precisions from the same initial state.  Returns the
    L2/L-inf errors of velocity and pressure and the kinetic-energy (decay)
    error of the mixed form, with the step times."""
    from nextgen_b200 import cases, cgx
    out = {"metric": "mixed-precision error vs FP64 after %d RK3 steps" % K, "steps": K,
           "cells": gm.ncv, "ke_decay_rel_err_bound": KE_DECAY_BOUND,
           "workload": "jittered-lattice (+/-0.25h) periodic Voronoi %d^3, CFL 0.8, Vreman" % n, "cases": {}}
    ok = True
    for kind in ("tgv", "solenoidal"):
        if kind == "tgv":
            prm = cases.tgv_params()
            rho, u, p = tgv
        else:
            prm = cases.hit_params(Mt=0.3)
            rho, u, p = cases.hit_state(n, prm, Mt=0.3, k0=4.0, seed=4321)
        prm.check_interval = 50
        res, ms = {}, {}
        for name, prec in (("fp64", cgx.CGX_FP64), ("mixed", cgx.CGX_MIXED)):
            s = cgx.Solver(gm, prm, prec)
            s.set_state_primitive(rho, u, p)
            s.initComplete()
            ms[name] = s.step_timed(K)
            r1, u1, _ = s.get_state()
            res[name] = (r1, u1, s.primitive()[0])
            s.close()
        e = _errors(vol, res["fp64"], res["mixed"], (rho, u))
        e.update({"fp64_ms_per_step": ms["fp64"] / K, "mixed_ms_per_step": ms["mixed"] / K,
                  "speedup": ms["fp64"] / ms["mixed"]})
        ok = ok and e["ke_rel"] <= KE_DECAY_BOUND and e["ke_decay_rel_err"] <= KE_DECAY_BOUND
        out["cases"][kind] = e
    out["within_bound"] = bool(ok)
    return out


def run_accuracy(args):
    """accuracy_block on the jittered n^3 mesh (200^3 = 8M cells by default)
    for `--accuracy-steps` steps (500 by default), as one JSON line."""
    from nextgen_b200 import cases, cgx
    from nextgen_b200.meshgen import PeriodicBoxMesh
    n, K = args.n, args.accuracy_steps
    m = PeriodicBoxMesh(n, jitter=JITTER, seed=SEED, nthreads=os.cpu_count() or 1)
    gm = cgx.Mesh(m)
    vol = np.array(m.vol_cv)
    prm = cases.tgv_params()
    out = accuracy_block(gm, n, vol, cases.tgv_state(m.x_cv[: m.ncv], prm), K)
    out.update({"config": {"workload": out["workload"]}, "data": "synthetic"})
    print(json.dumps(out), flush=True)
    return 0


def run_validate(args):
    """The FP64 GPU path against the CPU oracle over many steps: the Mt 0.3
    random-solenoidal state on the jittered n^3 mesh (128^3, about 2.1M cells,
    by default) advanced `--validate-steps` RK3 steps (200 by default) at CFL
    0.8 by both from the same initial state; the oracle runs on all host
    cores.  Prints one JSON line with the relative differences of the state
    and of the conserved totals, and the step counts and times reached."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Oracle
    from nextgen_b200 import cases, cgx
    from nextgen_b200.meshgen import PeriodicBoxMesh
    n, K = args.validate_n, args.validate_steps
    m = PeriodicBoxMesh(n, jitter=JITTER, seed=SEED, nthreads=os.cpu_count() or 1)
    prm = cases.hit_params(Mt=0.3)
    prm.check_interval = 50
    rho, u, p = cases.hit_state(n, prm, Mt=0.3, k0=4.0, seed=4321)
    s = cgx.Solver(cgx.Mesh(m), prm)
    s.set_state_primitive(rho, u, p)
    s.initComplete()
    o = Oracle(m, prm, nparts=os.cpu_count() or 1)
    o.set_state_primitive(rho, u, p)
    o.init_complete()
    t0 = time.perf_counter()
    assert s.step(K) == 0
    t_gpu = time.perf_counter() - t0
    t0 = time.perf_counter()
    assert o.step(K) == 0
    t_cpu = time.perf_counter() - t0
    g, r = s.get_state(), o.get_state()
    rel = lambda a, b: float(np.abs(a - b).max() / np.abs(b).max())
    tg, tr = s.totals(), o.totals()
    vol = np.array(m.vol_cv)
    scale = np.array([(r[0] * vol).sum()] + [np.abs(r[0] * r[1][:, k] * vol).sum() for k in range(3)] +
                     [(r[2] * vol).sum()])
    out = {"metric": "FP64 GPU vs CPU oracle after %d RK3 steps" % K, "cells": m.ncv,
           "config": {"workload": "jittered-lattice (+/-0.25h) periodic Voronoi %d^3, random solenoidal "
                                  "Mt 0.3, CFL 0.8, Vreman" % n},
           "rho_linf_rel": rel(g[0], r[0]), "u_linf_rel": rel(g[1], r[1]), "rhoE_linf_rel": rel(g[2], r[2]),
           "totals_rel": float((np.abs(tg - tr) / scale).max()),
           "time_gpu_vs_oracle_rel": abs(s.time()[0] - o.time()[0]) / o.time()[0],
           "steps": [s.time()[2], o.time()[2]], "gpu_s": t_gpu, "oracle_s": t_cpu,
           "oracle_threads": os.cpu_count() or 1, "data": "synthetic"}
    print(json.dumps(out), flush=True)
    return 0


def batch64_block(K, seed=64):
    """64 independent Taylor-Green cases of uneven size in one batch: edges
    log-uniform in [8, 64] (512 to 262,144 cells, +/-0.25h jitter), Mach
    uniform in [0.1, 0.5], Re uniform in [400, 3200], advanced together for K
    steps in FP64 and in mixed precision; the same cases one at a time on the
    plain FP64 path and at their own precision for comparison.  Returns the
    cell-steps/s of each."""
    from nextgen_b200 import cases, cgx
    rng = np.random.default_rng(seed)
    edges = [int(round(np.exp(x))) for x in rng.uniform(np.log(8), np.log(64), size=64)]
    from nextgen_b200.meshgen import PeriodicBoxMesh
    meshes = {}
    for e in sorted(set(edges)):
        hm = PeriodicBoxMesh(e, jitter=JITTER, seed=SEED + e)
        meshes[e] = (hm, cgx.Mesh(hm))
    cs = []
    for k, e in enumerate(edges):
        hm, gm = meshes[e]
        prm = cases.tgv_params(Ma=float(rng.uniform(0.1, 0.5)), Re=float(rng.uniform(400, 3200)))
        prm.check_interval = 50
        cs.append((gm, prm) + tuple(cases.tgv_state(hm.x_cv[: hm.ncv], prm)))
    total = float(sum(gm.ncv for gm, *_ in cs)) * K
    out = {"metric": "batched uneven instances: cell-steps/s", "unit": UNIT, "cases": len(cs),
           "cells": int(sum(gm.ncv for gm, *_ in cs)), "steps": K, "edges": edges, "data": "synthetic"}
    for name, prec in (("fp64", cgx.CGX_FP64), ("mixed", cgx.CGX_MIXED)):
        b = cgx.Batch(0, prec, max_cases=len(cs), hbm_budget=60 << 30)
        for gm, prm, rho, u, p in cs:
            assert b.add(gm, prm, rho, u, p, K + 2) is not None
        b.step(2)  # warm-up (also runs the batch autotuner)
        t0 = time.perf_counter()
        b.step(K)
        el = time.perf_counter() - t0
        out["batch_" + name] = {"cell_steps_per_s": total / el, "seconds": el}
        b.close()
    for name, prec in (("fp64", cgx.CGX_FP64), ("mixed", cgx.CGX_MIXED)):
        t0 = time.perf_counter()
        for gm, prm, rho, u, p in cs:
            s = cgx.Solver(gm, prm, prec)
            s.set_state_primitive(rho, u, p)
            s.initComplete()
            s.step(K)
            s.synchronize()
            s.close()
        el = time.perf_counter() - t0
        out["sequential_" + name] = {"cell_steps_per_s": total / el, "seconds": el}
    seq64 = out["sequential_fp64"]["cell_steps_per_s"]
    out["speedup_batch_fp64_vs_sequential_fp64"] = out["batch_fp64"]["cell_steps_per_s"] / seq64
    out["speedup_batch_mixed_vs_sequential_fp64"] = out["batch_mixed"]["cell_steps_per_s"] / seq64
    out["speedup_batch_mixed_vs_sequential_mixed"] = (out["batch_mixed"]["cell_steps_per_s"] /
                                                      out["sequential_mixed"]["cell_steps_per_s"])
    out["how"] = ("batch: host wall clock around K steps of one cgx_batch (graph replays) after a 2-step "
                  "warm-up; sequential: each case alone (solver create, initComplete, K steps) one after another")
    for hm, gm in meshes.values():
        gm.close()
        hm.close()
    return out


def run_batch64(args):
    """batch64_block for `--batch-steps` steps (300 by default), as one JSON
    line."""
    out = batch64_block(args.batch_steps)
    print(json.dumps(out), flush=True)
    return 0


def _host_phases(fn):
    """Run fn() with the host generator's phase timer on; returns (fn(),
    {phase: seconds}) parsed from what the generator writes to stderr."""
    import tempfile
    os.environ["CGX_MESHGEN_VERBOSE"] = "1"
    sys.stderr.flush()
    saved = os.dup(2)
    with tempfile.TemporaryFile(mode="w+") as tf:
        os.dup2(tf.fileno(), 2)
        try:
            res = fn()
        finally:
            os.dup2(saved, 2)
            os.close(saved)
            del os.environ["CGX_MESHGEN_VERBOSE"]
        tf.seek(0)
        phases = {}
        for line in tf.read().splitlines():
            if line.startswith("meshgen "):
                name, sec = line[len("meshgen "):].rsplit(None, 2)[0].strip(), float(line.split()[-2])
                phases[name] = phases.get(name, 0.0) + sec
    return res, phases


def run_opbuild(args):
    """The operator build (gradient coefficients, extended faces, level-2
    ghosts, per-cell factors) of the jittered n^3 periodic Voronoi mesh
    (128^3, about 2.1M cells, by default): the host generator's operator
    phases on all host cores against cgx_operators_build on the GPU from the
    mesher's compact output of the same mesh.  Checks that every array is
    bit-identical and prints one JSON line with the times, including the
    whole admission of a new mesh both ways (generator or mesher + device
    operators, then cgx_mesh_create)."""
    from nextgen_b200 import cgx
    from nextgen_b200.meshgen import DeviceOperatorMesh, PeriodicBoxMesh
    n = args.opbuild_n
    threads = os.cpu_count() or 1
    DeviceOperatorMesh(PeriodicBoxMesh(8, jitter=JITTER, seed=SEED)).close()  # context + module load
    t0 = time.perf_counter()
    host, ph = _host_phases(lambda: PeriodicBoxMesh(n, jitter=JITTER, seed=SEED, nthreads=threads))
    host_total = time.perf_counter() - t0
    mesher = ("seeds", "voronoi", "compact faces")
    host_ops = sum(v for k, v in ph.items() if k not in mesher)
    t0 = time.perf_counter()
    compact = PeriodicBoxMesh(n, jitter=JITTER, seed=SEED, nthreads=threads, compact_only=True)
    mesher_s = time.perf_counter() - t0
    runs = []
    for _ in range(3):
        t0 = time.perf_counter()
        dev = DeviceOperatorMesh(compact)
        runs.append((time.perf_counter() - t0, dev.device_ms))
        if len(runs) < 3:
            dev.close()
    fields = ["cvocv_i", "cvocv_v", "cvocv_grad_coeff", "cvoef", "n_ef", "c_ef", "area_over_delta_fa", "cmag_cv",
              "dcmag_hat_cv", "sa_to_vol_ratio", "x_cv", "icv_owner_g", "shift_g"]
    same = all(np.array_equal(getattr(dev, f), getattr(host, f)) for f in fields) and dev.nef == host.nef
    t0 = time.perf_counter()
    gm = cgx.Mesh(dev)
    mesh_create = time.perf_counter() - t0
    gm.close()
    wall = min(r[0] for r in runs)
    dms = min(r[1] for r in runs)
    out = {"metric": "operator build time", "unit": "s", "cells": host.ncv, "extended_faces": host.nef,
           "config": {"workload": "jittered-lattice (+/-0.25h) periodic Voronoi %d^3, EF_OPS DEFAULT "
                                  "(interp 1/3), SIGMA_THRESH 0.45" % n},
           "host_operator_s": host_ops, "host_threads": threads,
           "host_phases_s": {k: round(v, 4) for k, v in ph.items()},
           "host_mesher_s": sum(v for k, v in ph.items() if k in mesher), "host_generator_total_s": host_total,
           "device_build_s": dms / 1e3, "device_build_with_copies_s": wall,
           "speedup_device_vs_host": host_ops / (dms / 1e3),
           "speedup_with_copies_vs_host": host_ops / wall,
           "cgx_mesh_create_s": mesh_create, "bit_identical": bool(same),
           "admission_s": {"host_generator_then_mesh_create": host_total + mesh_create,
                           "mesher_then_device_ops_then_mesh_create": mesher_s + wall + mesh_create,
                           "mesher_compact_only_s": mesher_s},
           "data": "synthetic"}
    print(json.dumps(out), flush=True)
    dev.close()
    return 0 if same else 1


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cgx", choices=["cgx", "reference"])
    ap.add_argument("--n", type=int, default=200, help="lattice edge (cells = n^3)")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--cpu-n", type=int, default=48)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-served", action="store_true")
    ap.add_argument("--served-requests", type=int, default=32)
    ap.add_argument("--served-only", action="store_true",
                    help="instead of the throughput bench: only the served stream, as one JSON line")
    ap.add_argument("--accuracy", action="store_true",
                    help="instead of the throughput bench: mixed vs FP64 errors (TGV and solenoidal)")
    ap.add_argument("--accuracy-steps", type=int, default=500,
                    help="steps of the mixed-vs-FP64 accuracy block of the default run (0: skip it)")
    ap.add_argument("--batch64", action="store_true",
                    help="instead of the throughput bench: 64 uneven cases in one batch vs one at a time")
    ap.add_argument("--batch-steps", type=int, default=300,
                    help="steps of the 64-case batch block of the default run (0: skip it)")
    ap.add_argument("--validate", action="store_true",
                    help="instead of the throughput bench: FP64 GPU vs CPU oracle over many steps")
    ap.add_argument("--validate-n", type=int, default=128)
    ap.add_argument("--validate-steps", type=int, default=200)
    ap.add_argument("--device-ops", dest="device_ops", action="store_true", default=True,
                    help="build the bench mesh's operators on the GPU from the mesher's compact mesh "
                         "(the default; bit-identical to the host generator's)")
    ap.add_argument("--host-ops", dest="device_ops", action="store_false",
                    help="build the bench mesh with the host generator's operators instead")
    ap.add_argument("--opbuild", action="store_true",
                    help="instead of the throughput bench: operator build on the GPU vs the host generator")
    ap.add_argument("--opbuild-n", type=int, default=128)
    args = ap.parse_args()
    if args.warmup < 0 or args.steps < 1:
        sys.exit("steps >= 1, warmup >= 0")
    if args.impl == "reference":
        return run_reference(args)
    if args.accuracy:
        return run_accuracy(args)
    if args.batch64:
        return run_batch64(args)
    if args.validate:
        return run_validate(args)
    if args.opbuild:
        return run_opbuild(args)
    if args.served_only:
        print(json.dumps(served_stream(nreq=args.served_requests)), flush=True)
        return 0
    return run_cgx(args)


if __name__ == "__main__":
    sys.exit(main())
