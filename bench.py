"""Benchmark of the OpenTM homogenization hot path on B200.

Workload (the configuration the headline metric is quoted on): the OC optimisation loop on a
128^3 periodic cell -- rho0 = 0.3 + 0.05 U(-1,1) (seed 1), Linear density filter of radius 2
(periodic), SIMP p = 3 (k0 = 1, kmin = 1e-3), maximise trace(K^H) at volume fraction 0.3,
OC move limit 0.2, warm-started load cases, V(2,2)-preconditioned CG to ||r||/||f|| <= 1e-6.
One step = one OC iteration = one homogenization solve (3 load cases, K^H, sensitivity,
filter adjoint, OC update). The metric is solves/s with p50/p99 step latency.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Ours: every rank runs an independent replica on its own GPU (weak scaling, no data-path
collective); the timed region is bracketed by barrier + synchronize, the per-rank device
time is max-reduced, rank 0 prints one JSON line. The L2 cache (126 MB) is flushed by writing
a 256 MB buffer before every timed step, outside the timed events.

With N = 1 the line also carries the other configurations measured in the same run (--extra 1,
the default): `solve32` (configuration 1), `solve256` (configuration 3, the FP32 and both 16-bit
forms with their K^H and sensitivity errors against the FP64 oracle) and `serve`
(configuration 5 at 1000 requests/s offered); `mixed` is the same OC loop in the BF16 form with
its own K^H error.

Reference arm (--impl reference): the reference cannot be built offline, so the FP64 CPU
restatement of its algorithm (oracle/) runs the same OC loop on the host cores with all
threads, step for step: each step is one OC iteration whose 3 load cases are solved from the
previous iteration's solutions, as our arm's are. Both arms report the same `config`.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_CELL = 128
TOL = 1e-6
VOLFRAC = 0.3
MOVE = 0.2
DAMP = 0.5
FILTER_R = 2.0
P_SIMP, K0, KMIN = 3.0, 1.0, 1e-3
METRIC = "solves/s & p50/p99 latency, mixed vs FP32 MG on one B200 at K^H err<=1e-5"
UNIT = "solves/s"


def oc_config(n):
    """The workload of the headline line, shared by both arms (so their configs compare equal)."""
    return {"workload": f"OC loop, {n}^3 periodic cell, 3 load cases, V(2,2)-PCG to rel.res {TOL}, "
                        "warm-started load cases", "reso": n, "tol": TOL,
            "l2": "GPU arm: L2 flushed (256 MB write) before every timed step"}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = [l.split(",") for l in open(self.path).read().strip().splitlines() if l.strip()]
        os.unlink(self.path)
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax = max(smax, float(r[2]))
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def job_seconds(lat_ms, world, device):
    """Seconds of this rank's device-timed steps, max-reduced over the ranks: the job takes as
    long as its slowest replica."""
    import torch
    t = torch.tensor([sum(lat_ms) / 1e3], dtype=torch.float64, device=device)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------------------
# Our arm
# ---------------------------------------------------------------------------------------
def run_ours(args, rank, world, local_rank):
    import torch

    from opentm_b200 import (DensityFilter, HomoConfig, Homogenization_H, OCOptimizer, copy_to_device, copy_to_host,
                             launch_count, pinned_empty)
    from opentm_b200 import workloads as wl

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    n = args.n
    ne = n ** 3
    rho0 = wl.config2_density(n, seed=1)

    def make(precision, profile=False):
        H = Homogenization_H(HomoConfig(reso=n, femRelThres=TOL, pre_smooth=2, post_smooth=2, max_iter=200,
                                        precision=precision, profile=profile, smoother=args.smoother,
                                        cluster_cycle=int(args.cluster_cycle)))
        df = DensityFilter((n, n, n), FILTER_R, 1, True, P_SIMP, K0, KMIN)
        oc = OCOptimizer(ne, 0.001, MOVE, DAMP)
        return H, df, oc

    dC = -np.eye(3)  # objective -trace(K^H)
    g_k = torch.empty((n, n, n), dtype=torch.float32, device=dev)
    g_rho = torch.empty_like(g_k)

    def step(H, df, oc, rho):
        H.update_density(df, rho)  # filter + SIMP map straight into the handle's conductivities
        C = H.heatMatrixSensitivity(dC, g_k)  # dC is constant: K^H and the sensitivity in one pass
        df.backward(g_k, g_rho)
        oc.update(g_rho, rho, VOLFRAC)
        return C

    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > L2

    def timed_loop(precision, steps, warmup, e2e=False, profile=False):
        H, df, oc = make(precision, profile)
        rho = torch.from_numpy(rho0).to(dev)
        # the caller's per-step host arrays in page-locked memory from the library's allocator
        rho_np, out_np = pinned_empty(rho0.shape), pinned_empty(rho0.shape)
        rho_np[...] = rho0
        for _ in range(warmup):
            step(H, df, oc, rho)
        H.profile(reset=True)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        lat, Cs = [], []
        l0 = launch_count()
        for _ in range(steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            if e2e:
                copy_to_device(rho, rho_np)
            C = step(H, df, oc, rho)
            if e2e:
                copy_to_host(out_np, rho)
            e1.record()
            e1.synchronize()
            if e2e:
                rho_np[...] = out_np
            lat.append(e0.elapsed_time(e1))
            Cs.append(C)
        torch.cuda.synchronize()
        launches = launch_count() - l0
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        prof = H.profile(reset=True)
        iters = H.stats().iterations
        # one more (untimed) step for the error check: the step writes the conductivities straight
        # into the handle, so the field it used is formed again from the density it started from
        rho_chk = rho.clone()
        C_chk = step(H, df, oc, rho)
        k_last = df.forward(rho_chk).detach().cpu().numpy()
        return {"lat_ms": lat, "C": Cs, "launches": launches, "prof": prof, "k_last": k_last, "C_chk": C_chk,
                "iters": iters}

    clocks = ClockSampler(local_rank)
    clocks.start()
    main = timed_loop("fp32", args.steps, args.warmup)
    clk = clocks.stop()
    e2e = timed_loop("fp32", args.steps, args.warmup, e2e=True)
    # the same loop again with CUDA events around the first fine-level post-smoothing sweep of every iteration
    # (the event nodes need the chunked iteration graphs instead of the device-side loop)
    prof = timed_loop("fp32", args.steps, args.warmup, profile=True)
    mixed = None
    if args.mixed:
        try:
            mixed = timed_loop("bf16", args.steps, args.warmup)
        except Exception as ex:  # precision form not available
            mixed = {"error": str(ex)}

    def total_s(res):
        return job_seconds(res["lat_ms"], world, dev)

    t_main = total_s(main)
    t_e2e = total_s(e2e)
    t_prof = total_s(prof)
    t_mixed = total_s(mixed) if mixed and "lat_ms" in mixed else None
    if rank != 0:
        return None

    value = args.steps * world / t_main
    lat = np.array(main["lat_ms"])
    hbm, peak_kind = load_peaks()
    pr = prof["prof"]
    roofline = None
    if pr.sweeps > 0:
        launch_ms = pr.sweep_ms / pr.sweeps / pr.launches_per_sweep
        bytes_launch = pr.sweep_bytes / pr.launches_per_sweep
        achieved = bytes_launch / (launch_ms * 1e-3) / 1e9
        kname = ("k_tile_sweep (tiled post-smoothing leg: prolongation + 2 Gauss-Seidel sweeps, one launch each, "
                 "3 load cases)" if pr.kernel_kind == 1
                 else "k_gs_fine_pair (one colour-pair pass, 3 load cases)")
        tkey = "k_tile_sweep" if pr.kernel_kind == 1 else "k_gs_fine_pair"
        traffic = None
        tp = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tp):
            traffic = json.load(open(tp)).get(f"{tkey}_dram_bytes_per_launch_n{n}")
        roofline = {"bound": "hbm", "kernel": kname,
                    "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                    "frac": round(achieved / hbm, 4), "traffic": traffic,
                    "peak_kind": f"{peak_kind} hbm_gbs", "launch_us": round(launch_ms * 1e3, 3),
                    "algorithmic_bytes_per_launch": bytes_launch, "launches_timed": pr.sweeps * pr.launches_per_sweep,
                    "measured_in": "second timed pass of the same loop with per-sweep CUDA events "
                                   f"({args.steps * world / t_prof:.1f} solves/s with the events)"}

    line = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(t_main * 1e3 / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": oc_config(n), "replicas": world, "precision": "fp32", "smoother": args.smoother,
        "p50_ms": round(float(np.percentile(lat, 50)), 4), "p99_ms": round(float(np.percentile(lat, 99)), 4),
        "pcg_iterations_last_step": main["iters"],
        "e2e": {"value": round(args.steps * world / t_e2e, 3), "unit": UNIT, "h2d_bytes_per_step": 4 * ne,
                "d2h_bytes_per_step": 4 * ne + 72},
        "gpu_launches": int(main["launches"]),
        "roofline": roofline,
    }
    if mixed is not None:
        line["mixed"] = ({"value": round(args.steps * world / t_mixed, 3), "unit": UNIT, "precision": "bf16",
                          "pcg_iterations_last_step": mixed["iters"]} if t_mixed else mixed)
    if clk:
        line["clocks"] = clk
    if world == 1 and not args.no_cpu:
        line["cpu_baseline"], err = cpu_baseline(main["k_last"], main["C_chk"])
        line["kh_err"], line["kh_err_entries"] = err
        if mixed is not None and "lat_ms" in mixed:
            _, (e, ee) = cpu_baseline(mixed["k_last"], mixed["C_chk"], timed=False)
            line["mixed"]["kh_err"], line["mixed"]["kh_err_entries"] = e, ee
    if world == 1 and args.extra:
        # the other configurations on the same GPU, measured in the same run
        line["solve32"] = run_solve32(args, emit=False)
        line["solve256"] = run_solve256(args, emit=False)
        line["serve"] = serve_summary(args)
    print(json.dumps(line), flush=True)
    return line


def kh_errors(C_gpu, C_ref):
    """Largest K^H error relative to max |K|, and every entry's error on its own scale
    |dK_ij| / sqrt(|K_ii K_jj|)."""
    C_gpu, C_ref = np.asarray(C_gpu, dtype=np.float64), np.asarray(C_ref, dtype=np.float64)
    scale = np.sqrt(np.abs(np.outer(np.diag(C_ref), np.diag(C_ref))))
    ent = np.abs(C_gpu - C_ref) / scale
    return float(np.abs(C_gpu - C_ref).max() / np.abs(C_ref).max()), [[float(f"{v:.3e}") for v in row] for row in ent]


def cpu_baseline(k_last, C_gpu, timed=True):
    """FP64 oracle (the reference algorithm restated) timed on the host cores for one solve of the
    same workload (the field of one more step after the timed ones), and the K^H errors of the GPU
    result against it (the oracle converged to 1e-10)."""
    import oracle as ora
    ora.build()
    k = k_last.astype(np.float64)
    base = None
    if timed:
        t = time.perf_counter()
        r = ora.homogenize(k, tol=TOL, want_energy=True)
        s = ora.sensitivity(r["energy"], k, -np.eye(3))
        t_solve = time.perf_counter() - t
        base = {"value": round(1.0 / t_solve, 5), "unit": UNIT, "cores": ora.num_threads(), "kind": "port",
                "sample": f"one {k.shape[0]}^3 homogenization solve from a zero initial guess (3 load cases to "
                          f"{TOL}, K^H, sensitivity) in FP64 with the multigrid-PCG restatement, {t_solve:.2f} s"}
        del s
    ref = ora.homogenize(k, tol=1e-10)
    return base, kh_errors(C_gpu, ref["C"])


# ---------------------------------------------------------------------------------------
# Reference arm: the FP64 CPU restatement of the reference algorithm
# ---------------------------------------------------------------------------------------
def run_reference(args, rank, world):
    """The same OC loop as our arm, step for step, in the FP64 restatement on the host cores: each
    step is one OC iteration (density filter, conductivity, the 3 load cases solved from the
    previous iteration's solutions with the hierarchy built once, K^H, sensitivity, filter
    adjoint, OC update)."""
    if rank != 0:
        return None
    import oracle as ora
    from opentm_b200 import workloads as wl

    ora.build()
    ora.set_num_threads(os.cpu_count() or 1)
    n = args.n
    rho = wl.config2_density(n, seed=1).astype(np.float64)
    chi = np.zeros((3, n, n, n))
    iters = []

    def step():
        rho_f, ws = ora.conv_forward(rho, 1, FILTER_R, True)
        k = KMIN + rho_f ** P_SIMP * (K0 - KMIN)
        r = ora.homogenize_warm(k, chi, tol=TOL, want_energy=True)
        iters.append(max(r["iters"]))
        sk = ora.sensitivity(r["energy"], k, -np.eye(3))
        g = ora.conv_backward(sk * P_SIMP * rho_f ** (P_SIMP - 1) * (K0 - KMIN), ws, 1, FILTER_R, True)
        new, _ = ora.oc_update(g, rho, VOLFRAC, 0.001, MOVE, DAMP)
        rho[...] = new

    for _ in range(args.warmup):
        step()
    lat = []
    for _ in range(args.steps):
        t = time.perf_counter()
        step()
        lat.append(time.perf_counter() - t)
    total = sum(lat)
    value = args.steps / total
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 5), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(total * 1e3 / args.steps, 3),
            "p50_ms": round(float(np.percentile(np.array(lat) * 1e3, 50)), 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": oc_config(n), "pcg_iterations_last_step": iters[-1] if iters else None,
            "cpu_baseline": {"value": round(value, 5), "unit": UNIT, "cores": ora.num_threads(), "kind": "port",
                             "sample": "each step is one OC iteration of the FP64 multigrid-PCG restatement: filter, "
                                       "3 load cases solved from the previous solutions (hierarchy built once per "
                                       "iteration), K^H, sensitivity, filter adjoint, OC update"},
            "e2e": {"value": round(value, 5), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return line


# ---------------------------------------------------------------------------------------
# Serving workload (configuration 5): Poisson arrivals of mixed-resolution requests
# ---------------------------------------------------------------------------------------
def serve_fields(seed=4, per_reso=4):
    """A few seeded density fields per resolution (i.i.d. U(0.001,1) smoothed by a periodic
    3x3x3 box mean, SIMP p = 3), reused cyclically by the request stream."""
    from opentm_b200 import workloads as wl
    out = {}
    for n in wl.SERVE_RESOS:
        fl = []
        for j in range(per_reso):
            rho = (0.001 + 0.999 * wl.uniform(seed * 1000 + n * 10 + j, n ** 3)).reshape(n, n, n)
            for ax in range(3):  # separable periodic box mean
                rho = (np.roll(rho, 1, ax) + rho + np.roll(rho, -1, ax)) / 3.0
            fl.append(wl.simp(rho.astype(np.float32)))
        out[n] = fl
    return out


def run_serve(args, emit=True):
    import torch

    from opentm_b200 import HomoConfig, Homogenization_H, copy_to_device, pinned_empty
    from opentm_b200 import workloads as wl
    torch.cuda.set_device(0)
    fields = serve_fields()
    # serial plain-FP32 baseline: one resident handle per resolution, requests solved one after
    # another from a zero initial guess (H2D of the field, update, 3 load cases, K^H)
    handles = {n: Homogenization_H(HomoConfig(reso=n, femRelThres=TOL, pre_smooth=2, post_smooth=2,
                                              warm_start=False)) for n in wl.SERVE_RESOS}
    kdev = {n: torch.empty((n, n, n), dtype=torch.float32, device="cuda") for n in wl.SERVE_RESOS}
    # the field goes through a page-locked staging array, as the server's own ring does
    stage = {n: pinned_empty((n, n, n)) for n in wl.SERVE_RESOS}

    def upload(n, field):
        stage[n][...] = field
        copy_to_device(kdev[n], stage[n])

    for n in wl.SERVE_RESOS:  # warm-up (graph capture)
        upload(n, fields[n][0])
        handles[n].update(kdev[n])
        handles[n].heatMatrix()
    reqs0 = wl.serving_requests(200, seed=4, rate=500.0)  # arrival times unused: back to back
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for (t, n, i) in reqs0:
        upload(n, fields[n][i % len(fields[n])])
        handles[n].update(kdev[n])
        handles[n].heatMatrix()
    torch.cuda.synchronize()
    serial_rate = len(reqs0) / (time.perf_counter() - t0)
    for h in handles.values():
        h.close()
    rates = [args.rate] if args.rate > 0 else [50.0, 200.0, 500.0, 1000.0, 2000.0]
    results = []
    for rate in rates:
        results.append(serve_once(args, fields, rate, serial_rate))
    line = dict(results[-1])
    if len(results) > 1:
        line["sweep"] = [{k: r[k] for k in ("rate", "value", "p50_ms", "p99_ms")} for r in results]
        best = max(results, key=lambda r: r["value"])
        line.update({k: best[k] for k in ("value", "p50_ms", "p99_ms", "ms_per_step", "steps", "gpu_launches")})
        line["config"]["rate"] = best["rate"]
    line.pop("rate", None)
    if emit:
        print(json.dumps(line), flush=True)
    return line


def serve_summary(args, rate=1000.0, requests=2000):
    """Configuration 5 at one offered rate for the default line: solves/s, p50/p99 latency and the
    speed-up over serial single-request solves."""
    a = argparse.Namespace(**vars(args))
    a.rate, a.requests = rate, requests
    line = run_serve(a, emit=False)
    keep = ("value", "unit", "p50_ms", "p99_ms", "serial_fp32_solves_per_s", "speedup_vs_serial", "steps",
            "gpu_launches")
    out = {k: line[k] for k in keep if k in line}
    out["config"] = line["config"]
    out["config"]["rate"] = rate
    return out


def serve_once(args, fields, rate, serial_rate):
    from opentm_b200 import Server, launch_count
    from opentm_b200 import workloads as wl
    # about 4 s of arrivals per rate (at least 100 requests, at most --requests)
    reqs = wl.serving_requests(min(args.requests, max(100, int(4 * rate))), seed=4, rate=rate)
    srv = Server(hbm_budget_bytes=150 * 10 ** 9, max_active=args.max_active, fem_rel_thres=TOL,
                 iters_per_step=args.iters_per_step, batched=args.batched, streams=args.streams)
    # warm-up: every size once per concurrently running request, so that the handle form has a
    # resident handle (and its captured solve graph) of every size on every stream
    n_warm = 1 if args.batched else min(args.streams, args.max_active)
    for n in wl.SERVE_RESOS:
        for _ in range(n_warm):
            srv.submit(fields[n][0])
        srv.run_until_idle()
    l0 = launch_count()
    t_start = time.perf_counter()
    pending, arrival, done_at = list(reqs), {}, {}
    active = []
    while pending or active:
        now = time.perf_counter() - t_start
        while pending and pending[0][0] <= now:
            t, n, i = pending.pop(0)
            rid = srv.submit(fields[n][i % len(fields[n])])
            arrival[rid] = t
            active.append(rid)
        if not active:
            time.sleep(max(0.0, pending[0][0] - now))
            continue
        srv.step()
        now = time.perf_counter() - t_start
        still = []
        for j, rid in enumerate(active):
            st = srv.state(rid)
            if st == 0:  # admission is first come, first served: the rest is queued too
                still.extend(active[j:])
                break
            if st == 1:
                still.append(rid)
            else:
                srv.poll(rid)  # raises for a failed request
                done_at[rid] = now
        active = still
    makespan = max(done_at.values()) - min(arrival.values())
    lat = np.array([done_at[r] - arrival[r] for r in done_at]) * 1e3
    value = len(done_at) / makespan
    srv.close()
    return {"metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": 1, "steps": len(done_at),
            "warmup": n_warm * len(wl.SERVE_RESOS), "ms_per_step": round(1e3 / value, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"serving stream, {len(reqs)} requests, Poisson arrivals, "
                                   f"resolutions {wl.SERVE_RESOS} weights {wl.SERVE_WEIGHTS}",
                       "form": "batched" if args.batched else "handles on streams",
                       "streams": None if args.batched else min(args.streams, args.max_active),
                       "max_active": args.max_active, "iters_per_step": args.iters_per_step, "tol": TOL,
                       "budget_bytes": 150 * 10 ** 9},
            "rate": rate, "p50_ms": round(float(np.percentile(lat, 50)), 3),
            "p99_ms": round(float(np.percentile(lat, 99)), 3),
            "serial_fp32_solves_per_s": round(serial_rate, 3), "speedup_vs_serial": round(value / serial_rate, 3),
            "gpu_launches": int(launch_count() - l0)}


# ---------------------------------------------------------------------------------------
# Configuration 3: one 256^3 solve in FP32 and in the two 16-bit forms, against the FP64 oracle
# ---------------------------------------------------------------------------------------
def run_solve256(args, emit=True):
    from opentm_b200 import workloads as wl
    n = 256 if (args.n == N_CELL or not emit) else args.n
    return run_solve(args, n, wl.simp(wl.config3_density(n, seed=2)), "configuration 3",
                     f"{n}^3 thresholded smoothed Gaussian field (seed 2), SIMP p=3", headline="bf16", emit=emit)


def fine_sweep_roofline(args, n, kd):
    """HBM roofline of the fine-level sweep kernel at a cell whose working set exceeds L2: CUDA
    events around the first fine-level post-smoothing leg of every PCG iteration of a few FP32
    solves (the profiled solve runs the iterations as chunked graphs with event nodes)."""
    import torch
    from opentm_b200 import HomoConfig, Homogenization_H
    H = Homogenization_H(HomoConfig(reso=n, femRelThres=TOL, pre_smooth=2, post_smooth=2, warm_start=False,
                                    max_iter=200, smoother=args.smoother, profile=True))
    H.update(kd)
    H.heatMatrix()
    H.profile(reset=True)
    for _ in range(2):
        H.update(kd)
        H.heatMatrix()
    torch.cuda.synchronize()
    pr = H.profile(reset=True)
    del H
    if pr.sweeps <= 0:
        return None
    hbm, peak_kind = load_peaks()
    launch_ms = pr.sweep_ms / pr.sweeps / pr.launches_per_sweep
    bytes_launch = pr.sweep_bytes / pr.launches_per_sweep
    achieved = bytes_launch / (launch_ms * 1e-3) / 1e9
    return {"bound": "hbm", "kernel": "k_tile_sweep (post-smoothing leg)" if pr.kernel_kind == 1 else "k_gs_fine_pair",
            "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s", "frac": round(achieved / hbm, 4),
            "peak_kind": f"{peak_kind} hbm_gbs", "launch_us": round(launch_ms * 1e3, 3),
            "algorithmic_bytes_per_launch": bytes_launch, "launches_timed": pr.sweeps * pr.launches_per_sweep}


def run_solve32(args, emit=True):
    """Configuration 1: one plain solve of a 32^3 cell with rho ~ U(0.001, 1) (seed 0)."""
    from opentm_b200 import workloads as wl
    n = 32 if (args.n == N_CELL or not emit) else args.n
    return run_solve(args, n, wl.simp(wl.config1_density(n, seed=0)), "configuration 1",
                     f"{n}^3 rho ~ U(0.001, 1) i.i.d. (seed 0), SIMP p=3", headline="fp32", emit=emit)


def run_solve(args, n, k, label, field, headline, emit=True):
    """One cold solve (update, 3 load cases from zero, K^H, sensitivity) per step in the FP32 and
    both 16-bit forms, with their K^H (per entry) and sensitivity errors against the FP64 oracle.
    The oracle reference is converged to 1e-10 from the FP32 solution (the FP64 solution does not
    depend on the initial guess); run as its own workload, the oracle is also timed cold on the
    host cores as the CPU baseline."""
    import torch

    import oracle as ora
    from opentm_b200 import HomoConfig, Homogenization_H

    torch.cuda.set_device(0)
    kd = torch.from_numpy(k).cuda()
    dC = -np.eye(3)
    res = {}
    chi32 = None
    for prec in ("fp32", "bf16", "fp16"):
        H = Homogenization_H(HomoConfig(reso=n, femRelThres=TOL, pre_smooth=2, post_smooth=2, precision=prec,
                                        warm_start=False, max_iter=200, smoother=args.smoother))
        sens = torch.empty_like(kd)
        H.update(kd)
        H.heatMatrix()  # builds the solve graph
        lat = []
        for _ in range(max(1, args.steps)):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            H.update(kd)
            C = H.heatMatrixSensitivity(dC, sens)
            e1.record()
            e1.synchronize()
            lat.append(e0.elapsed_time(e1))
        st = H.stats()
        res[prec] = {"ms": float(np.median(lat)), "C": C, "sens": sens.cpu().numpy(), "iterations": st.iterations,
                     "refinements": st.refinements, "rel_res": max(st.rel_res)}
        if prec == "fp32":
            chi32 = np.stack([H.solution(c).cpu().numpy() for c in range(3)]).astype(np.float64)
        del H
    sweep_roofline = fine_sweep_roofline(args, n, kd) if n * n * n * 40 > 126 * 2 ** 20 else None
    # the sensitivity's error is set by the solve tolerance: the same FP32 solve to 1e-7 beside it
    tight = None
    if n * n * n * 40 > 126 * 2 ** 20:
        H = Homogenization_H(HomoConfig(reso=n, femRelThres=TOL / 10, pre_smooth=2, post_smooth=2, warm_start=False,
                                        max_iter=200, smoother=args.smoother))
        sens_t = torch.empty_like(kd)
        H.update(kd)
        C_t = H.heatMatrixSensitivity(dC, sens_t)
        tight = {"tol": TOL / 10, "C": C_t, "sens": sens_t.cpu().numpy(), "iterations": H.stats().iterations}
        del H
    ora.build()
    k64 = k.astype(np.float64)
    base = None
    if emit:
        t = time.perf_counter()
        r0 = ora.homogenize(k64, tol=TOL, want_energy=True)
        ora.sensitivity(r0["energy"], k64, dC)
        t_ora = time.perf_counter() - t
        base = {"value": round(1.0 / t_ora, 4), "unit": "solves/s", "cores": ora.num_threads(), "kind": "port",
                "sample": f"one {n}^3 cold solve (3 load cases to {TOL}) + sensitivity of the FP64 restatement, "
                          f"{t_ora:.1f} s"}
    ref = ora.homogenize_warm(k64, np.ascontiguousarray(chi32), tol=1e-10, want_energy=True)
    s_ref = ora.sensitivity(ref["energy"], k64, dC)
    out = {}
    for prec, r in res.items():
        kh, kh_ent = kh_errors(r["C"], ref["C"])
        se = float(np.abs(r["sens"] - s_ref).max() / np.abs(s_ref).max())
        se2 = float(np.linalg.norm(r["sens"] - s_ref) / np.linalg.norm(s_ref))
        out[prec] = {"solve_ms": round(r["ms"], 3), "solves_per_s": round(1e3 / r["ms"], 3), "kh_err": kh,
                     "kh_err_entries": kh_ent, "sens_err": se, "sens_err_l2": se2, "iterations": r["iterations"],
                     "refinements": r["refinements"], "rel_res": r["rel_res"]}
    if sweep_roofline:
        out["fp32"]["roofline"] = sweep_roofline
    if tight:
        kh, kh_ent = kh_errors(tight["C"], ref["C"])
        out["fp32_tol_1e-7"] = {"kh_err": kh, "sens_err": float(np.abs(tight["sens"] - s_ref).max() / np.abs(s_ref).max()),
                                "sens_err_l2": float(np.linalg.norm(tight["sens"] - s_ref) / np.linalg.norm(s_ref)),
                                "iterations": tight["iterations"]}
    line = {"metric": f"{n}^3 solve: solves/s (update + 3 load cases from zero + K^H + sensitivity), error vs "
                      "FP64 oracle",
            "value": out[headline]["solves_per_s"], "unit": "solves/s", "n_gpus": 1, "steps": args.steps,
            "higher_is_better": True, "dtype": "f32" if headline == "fp32" else f"{headline}+f64 refinement",
            "data": "synthetic",
            "config": {"workload": f"{label}: {field}, cold solve to rel.res {TOL}, V(2,2), coarsest FP64 direct",
                       "reso": n},
            "forms": out}
    if base:
        line["cpu_baseline"] = base
    if emit:
        print(json.dumps(line), flush=True)
    return line


# ---------------------------------------------------------------------------------------
# Configuration 4: MMA loop on a 384^3 cell (16-bit fine levels, FP64 MMA on the device)
# ---------------------------------------------------------------------------------------
def run_mma384(args):
    import torch

    from opentm_b200 import DensityFilter, HomoConfig, Homogenization_H, MMAOptimizer
    from opentm_b200 import workloads as wl

    torch.cuda.set_device(0)
    n = 384 if args.n == N_CELL else args.n
    ne = n ** 3
    rho = torch.from_numpy(wl.config4_density(n, seed=3)).cuda()
    H = Homogenization_H(HomoConfig(reso=n, femRelThres=TOL, pre_smooth=2, post_smooth=2, precision="bf16"))
    df = DensityFilter((n, n, n), FILTER_R, 1, True, P_SIMP, K0, KMIN)
    mma = MMAOptimizer(2, ne, 1.0, 0.0, 1000.0, 0.0)
    mma.setBound(0.001, 1.0)
    g_k = torch.empty_like(rho)
    dfdx, dg0, dg1 = torch.empty_like(rho), torch.full_like(rho, 1.0 / (0.25 * ne)), torch.empty_like(rho)
    e = [np.zeros((3, 3)) for _ in range(3)]
    for i in range(3):
        e[i][i, i] = 1.0
    iso_eps = 1e-3
    lat, C = [], None
    iters = max(args.steps, 1)
    for it in range(args.warmup + iters):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        k = df.forward(rho)
        H.update(k)
        C = H.heatMatrixSensitivity(-e[0], g_k)  # objective -K_xx (constant dC: one pass)
        df.backward(g_k, dfdx)
        a, b = C[0, 0] - C[1, 1], C[1, 1] - C[2, 2]
        dC = (np.sign(a) * (e[0] - e[1]) + np.sign(b) * (e[1] - e[2])) / iso_eps
        H.Sensitivity(dC, g_k)
        df.backward(g_k, dg1)
        g = [float(rho.mean().item()) / 0.25 - 1.0, (abs(a) + abs(b)) / iso_eps - 1.0]
        mma.update(it + 1, rho, dfdx, g, [dg0, dg1])
        e1.record()
        e1.synchronize()
        if it >= args.warmup:
            lat.append(e0.elapsed_time(e1))
    ms = float(np.mean(lat))
    line = {"metric": "384^3 MMA loop: iterations/s (filter, bf16 solve of 3 load cases, K^H, 2 sensitivities, "
                      "filter adjoints, FP64 MMA update)",
            "value": round(1e3 / ms, 4), "unit": "iterations/s", "n_gpus": 1, "steps": iters, "warmup": args.warmup,
            "ms_per_step": round(ms, 3), "p50_ms": round(float(np.percentile(lat, 50)), 3),
            "p99_ms": round(float(np.percentile(lat, 99)), 3), "higher_is_better": True, "dtype": "bf16+f64",
            "data": "synthetic",
            "config": {"workload": f"configuration 4: {n}^3, max K_xx s.t. volume 0.25 and isotropy "
                                   f"|Kxx-Kyy|+|Kyy-Kzz| <= {iso_eps}, rho0 = 0.25 + 0.02 U(-1,1) seed 3", "reso": n},
            "final_KH_diag": [float(C[i, i]) for i in range(3)], "final_volume": float(rho.mean().item()),
            "solve_iterations_last": H.stats().iterations}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------
# The design driver: runCustom as the reference's main() runs it
# ---------------------------------------------------------------------------------------
def run_design(args):
    """runInstance(128, {1, 1e-4}, {0.3, 0.2, 0.1, 0.1, 0.05, 0.05}, IWP, oc) (main.cpp:85): the
    tensor-matching design loop through the C driver. Iterations/s from the driver's own loop
    clock, as the difference of a run of warmup + steps iterations and one of warmup iterations
    (both build the solver and capture its graph once)."""
    import torch

    from opentm_b200 import launch_count
    from opentm_b200.driver import DesignConfig, InitWay, Model, run_custom
    torch.cuda.set_device(0)
    n = N_CELL if args.n == N_CELL else args.n
    steps, warm = max(args.steps, 1), max(args.warmup, 1)
    tt = (0.3, 0.2, 0.1, 0.1, 0.05, 0.05)
    out = {}
    for model in (Model.oc, Model.mma):
        base = dict(reso=n, heatRatio=(1.0, 1e-4), target_tensor=tt, winit=InitWay.IWP, model=model)
        _, a = run_custom(DesignConfig(max_iter=warm, **base))
        l0 = launch_count()
        _, b = run_custom(DesignConfig(max_iter=warm + steps, **base))
        launches = launch_count() - l0
        k = b["iterations"] - a["iterations"]
        dt = b["loop_seconds"] - a["loop_seconds"]
        out[model.name] = {"iterations_per_s": round(k / dt, 3) if k > 0 and dt > 0 else None,
                           "ms_per_iteration": round(1e3 * dt / k, 3) if k > 0 else None, "timed_iterations": k,
                           "objective_last": b["objective"], "volume_last": b["volume"],
                           "init_ms": round(1e3 * b["init_seconds"], 2), "gpu_launches": int(launches)}
    cpu = None
    if not args.no_cpu:
        import oracle as ora
        from oracle import driver as od
        ora.set_num_threads(os.cpu_count() or 1)
        rho0 = od.init_density(od.INIT_IWP, n)
        t0 = time.perf_counter()
        od.run_custom(rho0, "oc", heat_ratio=(1.0, 1e-4), target=tt, iters=1, tol=0.01)
        cpu = {"value": round(1.0 / (time.perf_counter() - t0), 5), "unit": "iterations/s",
               "cores": ora.num_threads(), "kind": "port",
               "sample": f"one OC design iteration at {n}^3 of the FP64 restatement (solve tolerance 0.01)"}
    line = {"metric": f"design iterations/s of runCustom (OC and MMA) at {n}^3",
            "value": out["oc"]["iterations_per_s"], "unit": "iterations/s", "n_gpus": 1, "steps": steps,
            "warmup": warm, "ms_per_step": out["oc"]["ms_per_iteration"], "higher_is_better": True,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"runInstance({n}, {{1, 1e-4}}, {list(tt)}, IWP, oc|mma), solve tolerance 0.01"},
            "models": out, "cpu_baseline": cpu, "gpu_launches": out["oc"]["gpu_launches"]}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_CELL)
    ap.add_argument("--mixed", type=int, default=1)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--workload", default="oc", choices=["oc", "serve", "solve32", "solve256", "mma384", "design"])
    ap.add_argument("--requests", type=int, default=2000)
    ap.add_argument("--rate", type=float, default=0.0, help="Poisson rate; 0 sweeps 50..2000 req/s")
    ap.add_argument("--max-active", type=int, default=64)
    ap.add_argument("--iters-per-step", type=int, default=2)
    ap.add_argument("--batched", action="store_true", help="serve: batched form instead of handles on streams")
    ap.add_argument("--streams", type=int, default=8, help="serve: requests running at once in the handle form")
    ap.add_argument("--extra", type=int, default=1,
                    help="add the 32^3 and 256^3 solves and one serving rate to the default line (N = 1 only)")
    ap.add_argument("--cluster-cycle", type=int, default=1,
                    help="lower levels as one thread-block-cluster launch: automatic (1), from 16^3 (2), from 32^3 (3), off (0)")
    ap.add_argument("--smoother", default="tiled", choices=["tiled", "color"],
                    help="fine-level smoother: shared-memory tiles (default) or global colour-pair passes")
    args = ap.parse_args()
    if args.workload == "serve":
        run_serve(args)
        return
    if args.workload == "solve256":
        run_solve256(args)
        return
    if args.workload == "solve32":
        run_solve32(args)
        return
    if args.workload == "mma384":
        run_mma384(args)
        return
    if args.workload == "design":
        run_design(args)
        return

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                             device_id=torch.device("cuda", local_rank))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
