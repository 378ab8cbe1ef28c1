#!/usr/bin/env python
"""Benchmark of the B200 update-and-measure path of the 3D layered-disorder XY model.

Metric: site-updates/s (one site-update = one Metropolis proposal at one site;
Wolff and measurement time are included).  Workload (per GPU): 256 disorder
realisations x 16 temperatures uniformly spaced in [1.1, 1.5], L = 32 cubes,
J_xy = 1.2, J_z(z) ~ U[0.5, 1.5] per realisation from its disorder seed, one
Wolff update per sweep, every sweep after thermalization measured into 32
bins (FP64 reductions).  A step is one persistent launch of S sweeps over all
4096 replicas, replayed from a CUDA graph; the default W + K = 3 + 17 steps of S = 100 sweeps is the
whole 2000-sweep job.  The state (512 MiB FP32) is larger than L2.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun (N > 1) every rank runs its own 4096 replicas (weak scaling,
no data-path collective); the time is the max over ranks of the CUDA-event
time.  `--impl reference` times the CPU restatement of the reference path
(its vectorised Metropolis batches on glibc's vector math library) on the
host cores instead (rank 0 only).
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BASE_SEED = 20260710  # the reference's benchmark base_seed (examples/theta_l64_s1000_benchmark.toml:11)
BYTES_PER_UPDATE = 12  # FP32 theta: read twice and half written per sweep


def parse():
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=17)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["b200", "reference"], default="b200")
    p.add_argument("--sweeps-per-step", type=int, default=100)
    p.add_argument("--samples", type=int, default=256, help="disorder realisations per GPU")
    p.add_argument("--temperatures", type=int, default=16)
    p.add_argument("--L", type=int, default=32)
    p.add_argument("--no-plain", action="store_true", help="skip the single-task L=64 comparison")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    p.add_argument("--cpu-seconds", type=float, default=15.0, help="target length of the CPU baseline sample")
    p.add_argument("--no-serve", action="store_true", help="skip the served-stream side figure")
    p.add_argument("--no-large", action="store_true", help="skip the L=256 large-lattice side figure")
    p.add_argument("--no-job", action="store_true", help="skip the job-file side figure")
    p.add_argument("--no-tune", action="store_true",
                   help="use the default kernel choice instead of the autotuner (profiling runs)")
    p.add_argument("--serve-tasks", type=int, default=4096, help="tasks of the served stream")
    p.add_argument("--serve-epoch", type=int, default=100, help="sweeps per server epoch")
    p.add_argument("--serve-only", action="store_true", help="run only the served stream (prints its own line)")
    return p.parse_args()


def load_pkg():
    import importlib.util

    pkg_dir = os.path.join(ROOT, "slsf-rs_b200")
    if "slsf_rs_b200" in sys.modules:
        return sys.modules["slsf_rs_b200"]
    spec = importlib.util.spec_from_file_location("slsf_rs_b200", os.path.join(pkg_dir, "__init__.py"),
                                                  submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["slsf_rs_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def workload(pkg, samples, n_temps, L, rank):
    """(disorder seed, T, run seed, J_xy, J_z) per replica of one rank: samples
    rank*samples + 1 .. (rank+1)*samples, so ranks hold disjoint replicas."""
    temps = np.linspace(1.1, 1.5, n_temps)
    out = []
    for s in range(1, samples + 1):
        sample = s + rank * samples
        dseed = BASE_SEED + sample - 1  # src/model.rs:741
        jz = pkg.uniform_layer_disorder(L, 0.5, 1.5, dseed)
        jxy = np.full(L, 1.2)
        for T in temps:
            out.append((dseed, float(T), pkg.task_seed(BASE_SEED, L, sample, float(T)), jxy, jz))
    return out


def max_over_ranks(value, dist, device):
    """The job time of a multi-rank run: the max of the ranks' times (one
    all_reduce of a scalar; no data-path collective)."""
    if dist is None:
        return value
    import torch

    t = torch.tensor([value], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def resident_profile():
    """Per-site figures of the committed k_resident ncu capture (DRAM bytes per replica site per
    launch, warp instructions per site-update), or {}."""
    path = os.path.join(ROOT, "profiles", "k_resident_c2_traffic.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


def traffic_per_site():
    v = resident_profile().get("dram_bytes_per_site_per_launch")
    return float(v) if v is not None else None


def issue_roofline(value, sm_mhz, sms=148):
    """The bound that does bind the one-CTA kernel: instruction issue.  Achieved warp
    instructions per second (site-updates/s x the committed ncu count of warp instructions per
    site-update) against 4 schedulers x SMs x the SM clock sampled in the timed region."""
    ipsu = resident_profile().get("warp_instructions_per_site_update")
    if ipsu is None or not sm_mhz:
        return None
    achieved = value * ipsu
    peak = 4 * sms * sm_mhz * 1e6
    return {"bound": "issue", "warp_instructions_per_site_update": ipsu, "achieved": achieved, "peak": peak,
            "unit": "warp instructions/s", "frac": achieved / peak,
            "source": "instructions per site-update from profiles/k_resident_c2_traffic.json (ncu), peak = "
                      "4 issue slots x 148 SMs x median SM clock of the timed region"}


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons every 200 ms."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) == 7:
                self.rows.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=5)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        sm, mx, reasons = [], None, set()
        for r in self.rows:
            try:
                sm.append(float(r[0]))
                mx = float(r[1])
            except ValueError:
                continue
            for k, name in enumerate(names):
                if r[3 + k].lower() == "active":
                    reasons.add(name)
        loaded = [v for v in sm if mx and v > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def host_description():
    """CPU model, logical CPUs, physical cores and the baseline build in use."""
    import oracle

    cpu = oracle.host_cpu()
    return {"cpu_model": cpu["model"], "logical_cpus": cpu["logical_cpus"], "physical_cores": cpu["physical_cores"],
            "build": oracle.baseline_lib().name + (" (8-lane AVX-512 batches)" if cpu["avx512f"] else
                                                   " (4-lane AVX2 batches)")}


BASELINE_LABEL = ("FP64 C++ restatement of SLSF-rs in the reference's order, Metropolis batches on glibc's vector "
                  "sincos/exp as the reference's on sleef's (not the Rust binary)")


def cpu_baseline(L, temps, sweeps_hint, seconds, threads=None):
    """Time the reference-order CPU path with the reference's vectorised
    Metropolis batches (oracle/baseline_simd.cpp) on all host threads on a
    bounded sample of the workload: one L^3 replica per thread (rank-per-task,
    src/model.rs:680-685), sized to run about `seconds`."""
    import oracle

    threads = threads or os.cpu_count() or 1
    jxy = np.full(L, 1.2)
    jz = oracle.uniform_disorder(L, 0.5, 1.5, BASE_SEED)
    # calibrate with one replica x 2 sweeps on one thread
    t1, _ = oracle.bench_tasks((L, L, L), jxy, jz, [temps[0]], math.pi, 1, [1], 2, 1, simd=True)
    per_sweep = t1 / 2
    sweeps = max(2, min(sweeps_hint, int(seconds / max(per_sweep, 1e-9))))
    n = threads
    tt = [temps[i % len(temps)] for i in range(n)]
    sec, chk = oracle.bench_tasks((L, L, L), np.tile(jxy, n), np.tile(jz, n), tt, math.pi, 1,
                                  [BASE_SEED + i for i in range(n)], sweeps, threads, simd=True)
    updates = n * sweeps * L ** 3
    out = {"value": updates / sec, "unit": "site-updates/s", "cores": threads, "kind": "port",
           "sample": f"{n} replicas of L={L} x {sweeps} sweeps (Metropolis + 1 Wolff + measure each), "
                     f"{threads} threads, {BASELINE_LABEL}",
           "seconds": sec}
    out.update(host_description())
    return out


def cpu_plain(L=64, T=1.3, sweeps_hint=1000, seconds=8.0):
    """c1 on the CPU: the oracle's reference-order path driving one L^3 task on
    one thread (the reference runs one task per process), on a bounded sample
    of the 1000-sweep run sized to about `seconds`."""
    import oracle

    jxy = np.full(L, 1.2)
    jz = oracle.uniform_disorder(L, 0.5, 1.5, BASE_SEED)
    t1, _ = oracle.bench_tasks((L, L, L), jxy, jz, [T], math.pi, 1, [BASE_SEED], 2, 1, simd=True)
    sweeps = max(2, min(sweeps_hint, int(seconds / max(t1 / 2, 1e-9))))
    sec, _ = oracle.bench_tasks((L, L, L), jxy, jz, [T], math.pi, 1, [BASE_SEED], sweeps, 1, simd=True)
    return {"value": sweeps * L ** 3 / sec, "unit": "site-updates/s", "cores": 1, "kind": "port",
            "sample": f"c1 single replica L={L}, T={T}, {sweeps} of its {sweeps_hint} sweeps (Metropolis + 1 Wolff + "
                      f"measure each), 1 thread, {BASELINE_LABEL}",
            "seconds": sec}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    L = args.L
    temps = list(np.linspace(1.1, 1.5, args.temperatures))
    threads = os.cpu_count() or 1
    step_seconds = max(1.0, min(10.0, 150.0 / max(1, args.steps + args.warmup)))
    times, updates = [], []
    for k in range(args.warmup + args.steps):
        r = cpu_baseline(L, temps, args.sweeps_per_step, step_seconds, threads)
        if k >= args.warmup:
            times.append(r["seconds"])
            updates.append(r["value"] * r["seconds"])
    value = sum(updates) / sum(times)
    line = {
        "impl": "reference", "metric": "site-updates/s", "value": value, "unit": "site-updates/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"c2 batched replicas: L={L}, J_xy=1.2, J_z~U[0.5,1.5], T in [1.1,1.5], "
                               "Metropolis + 1 Wolff + measure per sweep", "L": L},
        "cpu_baseline": dict({"value": value, "unit": "site-updates/s", "cores": threads, "kind": "port",
                              "sample": r["sample"]}, **host_description()),
        "e2e": {"value": value, "unit": "site-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def plain_rate(pkg, ctx, L=64, T=1.3, sweeps=1000):
    """Single-task GPU path, as ThetaModel is driven (src/model.rs:379-442): per
    sweep one slsf_task_sweep + one slsf_task_measure, each returning to the host."""
    jz = pkg.uniform_layer_disorder(L, 0.5, 1.5, BASE_SEED)
    t = pkg.Task(ctx, (L, L, L), np.full(L, 1.2), jz, T, wolff_steps=1, seed=pkg.task_seed(BASE_SEED, L, 1, T))
    t.init_random()
    for _ in range(20):
        t.sweep(1)
        t.measure()
    t0 = time.perf_counter()
    for _ in range(sweeps):
        t.sweep(1)
        t.measure()
    dt = time.perf_counter() - t0
    t.close()
    return {"value": sweeps * L ** 3 / dt, "unit": "site-updates/s",
            "config": f"c1 single replica L={L}, T={T}, {sweeps} sweeps, Metropolis + 1 Wolff + measure per sweep"}


def large_lattice(pkg, ctx, stream, L=256, T=1.22, sweeps=50, warmup=5):
    """Large lattice near the transition: one L^3 replica (J_xy = 1.2, J_z ~
    U[0.5, 1.5]); every sweep is Metropolis + one Wolff update, then the
    observables (energy, m^2, helicity sums) and C_z(r) for r = 1..L/2, as
    ThetaModel::sweep + ThetaModel::measure with z correlations.

    The figure runs the task through the batched entry point (grid-wide
    kernels; the observables and C_z of every sweep go into device bins, the
    correlation launches queued after each sweep by slsf_task_corr_fuse), so
    the whole run is one call with no host round trip per sweep; CUDA events on
    the context's stream.  `per_call` drives the same replica one call at a
    time (slsf_task_sweep, slsf_task_measure, slsf_task_correlations per sweep,
    each returning to the host), with the device time of each part."""
    import torch

    jz = pkg.uniform_layer_disorder(L, 0.5, 1.5, BASE_SEED)
    seed = pkg.task_seed(BASE_SEED, L, 1, T)
    t = pkg.Task(ctx, (L, L, L), np.full(L, 1.2), jz, T, wolff_steps=1, seed=seed, thermalization=0, binsize=1,
                 n_bins=warmup + sweeps)
    t.init_random()
    t.corr_setup(0, L // 2, 1, warmup + sweeps)
    t.corr_fuse(1)
    ctx.batch_run([t], warmup)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        st = ctx.batch_run([t], sweeps)
        e1.record(stream)
    torch.cuda.synchronize()
    total_ms = e0.elapsed_time(e1)
    _, n_corr = t.corr_bins()
    cluster = st[0]["wolff_cluster_sites"]
    t.close()
    out = {"value": sweeps * L ** 3 / (total_ms / 1e3), "unit": "site-updates/s",
           "config": f"c4 large lattice: L={L} (V={L ** 3}), T={T}, J_xy=1.2, J_z~U[0.5,1.5], Metropolis + 1 Wolff, "
                     f"observables and C_z(r<={L // 2}) every sweep into device bins; {sweeps} timed sweeps after "
                     f"{warmup}, one batched call",
           "ms_per_sweep": total_ms / sweeps, "mean_cluster_fraction": cluster / (sweeps * L ** 3),
           "correlation_measurements": n_corr}
    # the same replica one call at a time, as ThetaModel is driven
    t = pkg.Task(ctx, (L, L, L), np.full(L, 1.2), jz, T, wolff_steps=1, seed=seed)
    t.init_random()
    for _ in range(warmup):
        t.sweep(1)
        t.measure()
        t.correlations(0, L // 2)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    parts = {"sweep_ms": 0.0, "measure_ms": 0.0, "correlations_ms": 0.0}
    n_call = min(sweeps, 20)
    with torch.cuda.stream(stream):
        for _ in range(n_call):
            ev[0].record(stream)
            t.sweep(1)
            ev[1].record(stream)
            t.measure()
            ev[2].record(stream)
            t.correlations(0, L // 2)
            ev[3].record(stream)
            torch.cuda.synchronize()
            parts["sweep_ms"] += ev[0].elapsed_time(ev[1])
            parts["measure_ms"] += ev[1].elapsed_time(ev[2])
            parts["correlations_ms"] += ev[2].elapsed_time(ev[3])
    t.close()
    per_call = {k: v / n_call for k, v in parts.items()}
    per_call["ms_per_sweep"] = sum(per_call.values())
    per_call["value"] = L ** 3 / (per_call["ms_per_sweep"] / 1e3)
    per_call["note"] = "each part's events include the host's enqueue latency after the previous call returned"
    out["per_call"] = per_call
    return out


SERVE_L = (8, 16, 24, 32, 48, 64)


def serve_requests(pkg, n_tasks, seed=BASE_SEED):
    """Served-stream tasks: L ~ U{8,16,24,32,48,64}, T ~ U[1.0,1.6], sweeps ~
    U{200..2000}, disorder seed per task (J_xy = 1.2, J_z ~ U[0.5,1.5]); the
    first 20% of sweeps thermalize, the rest go into 32 bins."""
    rng = np.random.default_rng(seed)
    Ls = rng.choice(SERVE_L, n_tasks)
    Ts = rng.uniform(1.0, 1.6, n_tasks)
    sweeps = rng.integers(200, 2001, n_tasks)
    out = []
    jz_cache = {}
    for i in range(n_tasks):
        L, T, sw = int(Ls[i]), float(Ts[i]), int(sweeps[i])
        dseed = BASE_SEED + i
        key = (L, dseed)
        if key not in jz_cache:
            jz_cache[key] = pkg.uniform_layer_disorder(L, 0.5, 1.5, dseed)
        out.append(dict(tag=i + 1, dims=(L, L, L), T=T, seed=pkg.task_seed(BASE_SEED, L, i + 1, T),
                        jxy=np.full(L, 1.2), jz=jz_cache[key], sweeps=sw, therm=sw // 5, n_bins=32))
    return out


def serve_run(pkg, ctx, reqs, rate, epoch_sweeps):
    """Submits `reqs` as a Poisson stream of `rate` tasks/s (all at once when
    rate is None) to a continuous-batching server running on its worker
    thread; returns throughput and latency figures from the server's clock."""
    srv = pkg.Server(ctx, epoch_sweeps=epoch_sweeps)
    rng = np.random.default_rng(BASE_SEED + 1)
    gaps = rng.exponential(1.0 / rate, len(reqs)) if rate else np.zeros(len(reqs))
    arrivals = np.cumsum(gaps)
    results = []
    srv.start()
    t0 = time.perf_counter()
    for r, at in zip(reqs, arrivals):
        delay = at - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        srv.submit(r["tag"], r["dims"], r["T"], r["seed"], r["jxy"], r["jz"], r["sweeps"],
                   thermalization=r["therm"], n_bins=r["n_bins"])
        if len(results) < len(reqs):
            results.extend(srv.poll(256))
    srv.wait_idle(3600)
    srv.stop()
    results.extend(srv.poll(len(reqs)))
    st = srv.stats()
    srv.close()
    ok = [r for r in results if r["status"] == pkg.OK]
    lat = np.array([r["finish_s"] - r["submit_s"] for r in ok])
    wait = np.array([r["admit_s"] - r["submit_s"] for r in ok])
    first = min(r["submit_s"] for r in results)
    last = max(r["finish_s"] for r in results)
    updates = sum(r["dims"][0] ** 3 * r["sweeps"] for r in reqs)
    return {"tasks": len(reqs), "completed": len(ok), "failed": len(results) - len(ok),
            "offered_tasks_per_s": rate, "makespan_s": last - first,
            "throughput": updates / (last - first), "unit": "site-updates/s",
            "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
            "p50_queue_s": float(np.percentile(wait, 50)), "p99_queue_s": float(np.percentile(wait, 99)),
            "epochs": st["epochs"], "launch_groups": st["launches"], "peak_active": st["peak_active"],
            "peak_bytes": st["peak_bytes"], "busy_s": st["busy_s"]}


def served_stream(pkg, ctx, n_tasks, epoch_sweeps):
    """Served stream: capacity with every task queued at t = 0, then Poisson
    arrivals offering 0.8x and 1.5x that capacity."""
    reqs = serve_requests(pkg, n_tasks)
    mean_work = float(np.mean([r["dims"][0] ** 3 * r["sweeps"] for r in reqs]))
    # kernel choice per request size from the autotuner (the server's launches use the context's table)
    tuned = {str(L): ctx.autotune((L, L, L)) for L in SERVE_L}
    warm = serve_requests(pkg, 64, seed=BASE_SEED + 7)
    serve_run(pkg, ctx, warm, None, epoch_sweeps)
    sat = serve_run(pkg, ctx, reqs, None, epoch_sweeps)
    capacity = sat["throughput"]
    out = {"workload": f"c3 served stream: {n_tasks} tasks, L~U{{8..64}}, T~U[1.0,1.6], sweeps~U{{200..2000}}, "
                       f"J_xy=1.2, J_z~U[0.5,1.5] per task, 20% thermalization, 32 bins, epoch {epoch_sweeps} sweeps",
           "mean_site_updates_per_task": mean_work, "saturation": sat, "capacity": capacity, "kernel_choice": tuned}
    for load in (0.8, 1.5):
        rate = load * capacity / mean_work
        r = serve_run(pkg, ctx, reqs, rate, epoch_sweeps)
        r["offered_load"] = load
        out[f"load_{load}"] = r
    return out


def job_figure(pkg):
    """Job files end to end (slsf-rs_b200/jobs.py): a bounded sample of the
    reference's production job shape (L in {8, 16, 24, 32}, ten temperatures in
    [1.1, 1.5], two-point J_xy = 1.5 +- 0.5, J_z = 0.1, no correlations: the
    served path) and a default-correlation job (r_max = L/2 measured every
    sweep, measured inside the one-CTA kernel's sweeps).
    Wall clock around run_job (task expansion, device set-up, runs, estimates);
    synthetic tasks from the job schema, no files written."""
    import time
    import importlib

    jobs = importlib.import_module("slsf_rs_b200.jobs")
    out = {}
    specs = {
        "served": """
name = "bench_served"
[model]
L = [8, 16, 24, 32]
T = [1.1, 1.1444444444444444, 1.1888888888888889, 1.2333333333333334, 1.2777777777777777, 1.3222222222222222,
     1.3666666666666667, 1.4111111111111112, 1.4555555555555555, 1.5]
samples = 8
base_seed = 20260710
j_xy = 1.5
delta_j_xy = [0.5]
j_z = 0.1
[run]
sweeps = 2000
thermalization = 500
binsize = 100
[measure]
corr_rmax_xy = [0, 0, 0, 0]
corr_rmax_z = [0, 0, 0, 0]
""",
        "correlated": """
name = "bench_correlated"
[model]
L = [8, 16]
T = [1.1, 1.15, 1.2, 1.25, 1.3, 1.35, 1.4, 1.45, 1.5, 1.55]
samples = 16
base_seed = 20260710
j_xy = 1.5
delta_j_xy = [0.5]
j_z = 0.1
[run]
sweeps = 1000
thermalization = 200
binsize = 50
""",
    }
    with pkg.Context() as ctx:
        for key, text in specs.items():
            cfg = jobs.config_from_toml(text)
            tasks = jobs.make_tasks(cfg)
            t0 = time.perf_counter()
            res = jobs.run_job(ctx, cfg, tasks=tasks)
            wall = time.perf_counter() - t0
            updates = sum(t["l_x"] * t["l_y"] * t["l_z"] * (t["thermalization"] + t["sweeps"]) for t in tasks)
            out[key] = {"tasks": len(tasks), "wall_s": wall, "value": updates / wall, "unit": "site-updates/s",
                        "completed": len(res["tasks"]),
                        "job": f"L={cfg.l}, {len(cfg.temperatures)} T, {cfg.samples} samples, "
                               f"{cfg.thermalization}+{cfg.sweeps} sweeps, "
                               + ("no correlations" if key == "served" else
                                  f"C_x, C_y, C_xy(z), C_z with r_max = L/2 every {cfg.correlation_interval} sweep")}
    return out


def serve_only(args):
    import torch

    torch.cuda.set_device(0)
    pkg = load_pkg()
    pkg.load()
    ctx = pkg.Context(0)
    res = served_stream(pkg, ctx, args.serve_tasks, args.serve_epoch)
    ctx.close()
    print(json.dumps(res))
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.serve_only:
        return serve_only(args)

    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)

    pkg = load_pkg()
    pkg.load()
    ctx = pkg.Context(local_rank)
    stream = torch.cuda.Stream(device=dev)
    ctx.set_stream(stream.cuda_stream)

    L, S = args.L, args.sweeps_per_step
    # kernel, cluster and CTA size for this shape
    choice = ctx.tune_get((L, L, L)) if args.no_tune else ctx.autotune((L, L, L))
    wl = workload(pkg, args.samples, args.temperatures, L, rank)
    n = len(wl)
    total_sweeps = (args.warmup + args.steps) * S
    therm = args.warmup * S
    n_bins = 32
    binsize = max(1, (args.steps * S + n_bins - 1) // n_bins)
    tasks = []
    for dseed, T, seed, jxy, jz in wl:
        t = pkg.Task(ctx, (L, L, L), jxy, jz, T, proposal_width=math.pi, wolff_steps=1, seed=seed,
                     thermalization=therm, binsize=binsize, n_bins=n_bins)
        t.init_random()
        tasks.append(t)
    handles = ctx.handle_array(tasks)
    # one step = one replay of a CUDA graph holding the persistent launch
    session = ctx.session(tasks, S)

    # warm-up steps = thermalization sweeps
    for _ in range(args.warmup):
        session.step()
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()

    clocks = ClockSampler(local_rank)
    clocks.start()
    launches0 = ctx.launches
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    with torch.cuda.stream(stream):
        ev[0].record(stream)
        for k in range(args.steps):
            session.step()
            ev[k + 1].record(stream)
    torch.cuda.synchronize(dev)
    launches = ctx.launches - launches0
    clk = clocks.stop()
    session.close()
    step_ms = [ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)]
    elapsed = sum(step_ms) / 1e3
    elapsed = max_over_ranks(elapsed, dist, dev)
    updates_rank = n * S * args.steps * L ** 3
    value = updates_rank * world / elapsed

    # end-to-end through the public API: every step uploads its task table
    # (pinned) and reads back every task's counters and bins
    e2e_steps = max(1, min(args.steps, 5))
    bins_out = np.zeros((n, n_bins, pkg.BIN_COLS))
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        ctx.batch_run(tasks, S, handles=handles)
        ctx.batch_bins(tasks, n_bins, out=bins_out, handles=handles)
    e2e_dt = time.perf_counter() - t0
    e2e_dt = max_over_ranks(e2e_dt, dist, dev)
    e2e_value = n * S * e2e_steps * L ** 3 * world / e2e_dt
    view_bytes = 112  # sizeof(slsf::TaskView) uploaded per task per batch launch
    h2d = n * view_bytes + 8 * n  # task table + handle table of the gather
    d2h = n * 32 + n * n_bins * pkg.BIN_COLS * 8  # per-task counters + bins

    peak, peak_kind = peaks()
    avg_launch_s = elapsed / args.steps
    alg_bytes = BYTES_PER_UPDATE * n * S * L ** 3
    achieved = alg_bytes / avg_launch_s / 1e9
    tps = traffic_per_site()
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": (tps * n * L ** 3) if tps is not None else None,
                "peak_kind": peak_kind,
                "kernel": "k_resident (one launch = S sweeps of every replica, each replica resident in one CTA's shared memory)"
                if choice["kind"] == "resident" else f"k_cluster ({choice['cluster']} CTAs per replica)",
                "algorithmic_bytes_per_launch": alg_bytes}

    extra = {}
    if rank == 0 and world == 1:
        if not args.no_plain:
            extra["plain"] = plain_rate(pkg, ctx)
            extra["plain"]["batched_over_plain"] = value / extra["plain"]["value"]
            # the same single-task path on the headline's replica size, for context
            same = plain_rate(pkg, ctx, L=L, T=1.3, sweeps=500)
            extra["plain"]["same_L"] = {"value": same["value"], "L": L, "batched_over_plain": value / same["value"]}
        if not args.no_large:
            extra["large"] = large_lattice(pkg, ctx, stream)
        if not args.no_serve:
            extra["served"] = served_stream(pkg, ctx, args.serve_tasks, args.serve_epoch)
        if not args.no_job:
            extra["job"] = job_figure(pkg)
        if not args.no_cpu:
            extra["cpu_baseline"] = cpu_baseline(L, list(np.linspace(1.1, 1.5, args.temperatures)), 2000,
                                                 args.cpu_seconds)
            extra["cpu_baseline"]["gpu_over_cpu"] = value / extra["cpu_baseline"]["value"]
            c1 = cpu_plain()
            if "plain" in extra:
                c1["plain_gpu_over_cpu"] = extra["plain"]["value"] / c1["value"]
            extra["cpu_baseline"]["c1"] = c1

    if rank == 0:
        line = {
            "metric": "site-updates/s", "value": value, "unit": "site-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": f"c2 batched replicas per GPU: {args.samples} disorder x {args.temperatures} T "
                                   f"in [1.1,1.5], L={L}, J_xy=1.2, J_z~U[0.5,1.5], Metropolis (width pi) + 1 Wolff "
                                   f"+ measure per sweep, {total_sweeps} sweeps total, {S} sweeps per step",
                       "replicas_per_gpu": n, "L": L, "sweeps_per_step": S, "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (state 512 MiB per GPU)", "reductions": "fp64",
                       "kernel_choice": choice},
            "clocks": clk, "gpu_launches": launches,
            "e2e": {"value": e2e_value, "unit": "site-updates/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps": e2e_steps},
            "roofline": roofline,
            "issue_roofline": issue_roofline(value / world, clk.get("sm_mhz")) if choice["kind"] == "resident" else None,
            "step_ms": step_ms,
        }
        line.update(extra)
        print(json.dumps(line))
    for t in tasks:
        t.close()
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
