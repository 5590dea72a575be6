"""Benchmark of the adaptive cubature hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload oscillatory_cornerpeak_8d | gaussian_5d | productpeak_6d_batch]

A step integrates one batch of the workload to its epsrel through the
library's public C ABI (cub_integrate / cub_integrate_batch).  The default
workload is the 8-D Genz pair: oscillatory cos(2 pi 0.3 + sum 1.1 x_i) and
corner peak (1 + sum 0.5 x_i)^-9 on [0,1]^8, FP64, epsrel 1e-6, epsabs 1e-12
(synthetic parameters as specified; the analytic integral checks every
result).  Metric: integrals/s (whole job, all GPUs), with Geval/s beside it.

--impl reference times the reference algorithm's CPU implementation (the
oracle port of the two-phase engine, oracle/cuhre_oracle.c) on the host
cores with all threads, on the same workload.

Under torchrun (weak scaling, no collective on the data path): for the
single-integral workloads each rank integrates its own copy of the step's
integrals; for batch workloads the job's world x count integrals are dealt
to the ranks by a greedy split of probe costs (cubature.parallel), other
sharded workloads cut contiguously (cubature.parallel.shard_bounds).
Steps are bracketed by a barrier and device synchronisation, and the max
time over ranks is used.
"""
from __future__ import annotations

import argparse
import faulthandler
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "old-gpuintegration_b200"))
sys.path.insert(0, str(ROOT / "oracle"))

WORKLOADS = {
    # name: (family list, ndim, a, u, epsrel, epsabs, batch)
    "oscillatory_cornerpeak_8d": {
        "items": [("oscillatory", 8, 1.1, 0.3), ("corner_peak", 8, 0.5, 0.0)],
        "epsrel": 1e-6, "epsabs": 1e-12,
    },
    "gaussian_5d": {
        "items": [("gaussian", 5, 5.0, 0.5)], "epsrel": 1e-3, "epsabs": 1e-12,
    },
    # 4096 product peaks, a_i log-uniform in [1,50], u_i uniform in [0.1,0.9],
    # per-integral seed; breadth-first refinement with the reference's region
    # test (every integral converges; the two-phase policy leaves ~5% of
    # these with boxes at the 2048-bisection cap)
    "productpeak_6d_batch": {
        "batch": ("product_peak", 6, 4096), "epsrel": 1e-5, "epsabs": 1e-12,
        "policy": "breadth",
    },
    "productpeak_6d_batch_refpolicy": {
        "batch": ("product_peak", 6, 4096), "epsrel": 1e-5, "epsabs": 1e-12,
        "policy": "reference",
    },
    # 256 x the 7-D table integrand: 512-knot spline x 128 x 128 bilinear x
    # Gaussian kernel (sigma 0.25), mu offsets uniform in [-1, 1]; FP64
    # tables (seeded synthetic data, cubature.tables); breadth-first
    "table7_7d_batch": {
        "tables": ("table7", 7, 256), "epsrel": 1e-6, "epsabs": 1e-12, "policy": "breadth",
    },
    # learned control variate on 7-D product peaks (the batch generator at
    # n = 7): network trained on the tensor cores, integral of f - g plus
    # integral of g, plain method as fallback and check; the plain method's
    # rate on the same integrands is measured in the same run
    "cv_productpeak_7d_batch": {
        "cv": ("product_peak", 7, 256), "epsrel": 1e-6, "epsabs": 1e-12, "policy": "breadth",
    },
}

# Algorithmic FP64 flops per integrand evaluation, FMA = 2 (transcendental
# calls counted separately): map 2n + 5 rule FMAs 10 + Jacobian 1 + f.
F_FAMILY = {
    "gaussian": lambda n: 4 * n + 1,
    "oscillatory": lambda n: 2 * n + 2,
    "corner_peak": lambda n: 2 * n + 1 + 4 + 1,
    "product_peak": lambda n: 5 * n + (n - 1) + 1,
    # spline 12 + bilinear 10 + kernel 6 (+1 exp); cell searches are integer
    "table7": lambda n: 12 + 10 + 6,
}


def flops_per_region(family: str, n: int) -> float:
    from cubature import npoints

    per_eval = 2 * n + 10 + 1 + F_FAMILY[family](n)
    return npoints(n) * per_eval + 5 * n + 3 * 9 * 3 + 8


def product_peak_params(n: int, count: int):
    import numpy as np

    out = []
    for k in range(count):
        rng = np.random.default_rng(k)
        a = np.exp(rng.uniform(math.log(1.0), math.log(50.0), n))
        u = rng.uniform(0.1, 0.9, n)
        out.append((list(a), list(u)))
    return out


class ClockSampler:
    """nvidia-smi clocks/throttle sampling (every 10 ms) during the timed
    region, plus one query right after it for regions shorter than the
    sampling period.  Read-only: no GPU setting is touched."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.idx = device_index
        self.proc = None
        self.lines: list[str] = []

    def _cmd(self, loop: bool):
        cmd = ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
               "--format=csv,noheader,nounits"]
        return cmd + (["-lms", "10"] if loop else [])

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(self._cmd(True), stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        try:
            out = subprocess.run(self._cmd(False), capture_output=True, text=True, timeout=10)
            self.lines.extend(l.strip() for l in out.stdout.splitlines() if l.strip())
        except (OSError, subprocess.TimeoutExpired):
            pass

    def summary(self) -> dict:
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def profiled_traffic(kernel: str, workload: str):
    """DRAM bytes (read + write) per launch of `kernel` on `workload` from
    the committed ncu summary profiles/<kernel>_<workload>.md (the line
    'traffic_bytes_per_launch: N'); None when there is no such capture."""
    import re

    path = ROOT / "profiles" / f"{kernel}_{workload}.md"
    if not path.exists():
        return None
    m = re.search(r"^traffic_bytes_per_launch:\s*(\d+)", path.read_text(), re.M)
    return int(m.group(1)) if m else None


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def measure_fp64_peak(torch) -> float:
    """FP64 dense throughput of cuBLAS DGEMM on this GPU (TFLOP/s), the
    denominator for the FP64-bound rule kernel."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2 * n ** 3 / best / 1e12


def cpu_reference_rate(workload: dict, seconds: float, threads: int = 0,
                       regions_per_integral: float | None = None):
    """Integrals/s of the oracle's two-phase engine on the host cores over a
    bounded sample of the workload (whole integrals, repeated)."""
    import oracle as O

    jobs = []
    if "tables" in workload:
        return cpu_table7_rate(workload, seconds, threads, regions_per_integral)
    if "items" in workload:
        for fam, n, a, u in workload["items"]:
            jobs.append((fam, n, a, u))
    else:
        fam, n, count = workload["batch"] if "batch" in workload else workload["cv"]
        for a, u in product_peak_params(n, count):
            jobs.append((fam, n, a, u))
    rules = {}
    t0 = time.perf_counter()
    done = 0
    evals = 0
    i = 0
    while True:
        fam, n, a, u = jobs[i % len(jobs)]
        R = rules.setdefault(n, O.Rule(n))
        cap = (1 << 30) if workload.get("policy") == "breadth" else 0
        r = R.integrate_reference(O.make_integrand(fam, n, a, u), workload["epsrel"],
                                  workload["epsabs"], phase1_cap=cap, nthreads=threads)
        done += 1
        evals += r["neval"]
        i += 1
        el = time.perf_counter() - t0
        if el >= seconds and done >= len(jobs) if "items" in workload else el >= seconds:
            break
    cores = threads if threads > 0 else O.max_threads()
    return done / el, evals / el, cores, done, el


# Regions per integral of the 7-D table workload at epsrel 1e-6 (breadth
# policy): the mean over its first 16 offsets, measured on the GPU (the
# engine's own count, the same algorithm as the oracle).  One such integral
# takes the oracle minutes, so the CPU rate is measured at epsrel 1e-4 in
# regions/s and divided by the regions per integral -- the GPU run's own
# figure for the same integrands when there is one, else this mean.
TABLE7_REGIONS_PER_INTEGRAL = 17_000_000


def cpu_table7_rate(workload: dict, seconds: float, threads: int = 0,
                    regions_per_integral: float | None = None):
    import oracle as O
    from cubature import tables as T

    d = T.table7_data(0)
    offs = T.table7_offsets(workload["tables"][2])
    R = O.Rule(7)
    t0 = time.perf_counter()
    regions = evals = done = 0
    while True:
        f = O.make_table7(d["spline_x"], d["spline_y"], d["grid_x"], d["grid_y"], d["grid_z"],
                          d["sigma"], offs[done % len(offs)])
        r = R.integrate_reference(f, 1e-4, workload["epsabs"], phase1_cap=1 << 30,
                                  nthreads=threads)
        regions += r["nregions"]
        evals += r["neval"]
        done += 1
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    cores = threads if threads > 0 else O.max_threads()
    per = regions_per_integral or TABLE7_REGIONS_PER_INTEGRAL
    rate = regions / el / per
    return rate, evals / el, cores, done, el


def cpu_model() -> str:
    """The host CPU's model name (/proc/cpuinfo), or the platform string."""
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform

    return platform.processor() or platform.machine()


REF_DRIVER = ROOT / "oracle" / "_ref" / "ref_driver"
FAMILY_IDS = {"gaussian": 1, "oscillatory": 2, "corner_peak": 3, "product_peak": 4,
              "continuous": 5, "discontinuous": 6, "cossum": 7}


def reference_gpu_rate(workload: dict, warmup: int, reps: int, device: int):
    """The unmodified reference engine (quad::GPUcuhre compiled from its own
    sources by oracle/ref_driver/Makefile) on the same integrands, one
    process on this GPU: warm median ms per integrate() call, summed over
    the step's integrands.  None when the driver was not built or fails."""
    if "items" not in workload or not REF_DRIVER.exists():
        return None
    env = dict(os.environ, CUDA_VISIBLE_DEVICES=os.environ.get("CUDA_VISIBLE_DEVICES",
                                                                 str(device)).split(",")[0])
    per, total_ms = [], 0.0
    for fam, n, a, u in workload["items"]:
        av = a if isinstance(a, (list, tuple)) else [a] * n
        uv = u if isinstance(u, (list, tuple)) else [u] * n
        cmd = [str(REF_DRIVER), "bench", str(FAMILY_IDS[fam]), str(n), repr(workload["epsrel"]),
               repr(workload["epsabs"]), str(warmup), str(reps)] + [repr(float(x)) for x in av]
        cmd += [repr(float(x)) for x in uv]
        try:
            out = subprocess.run(cmd, capture_output=True, text=True, timeout=300, env=env)
        except (OSError, subprocess.TimeoutExpired):
            return None
        rec = None
        for line in out.stdout.splitlines():
            if line.startswith("BENCH "):
                rec = json.loads(line[6:])
        if out.returncode != 0 or rec is None:
            return None
        per.append({"family": fam, "ndim": n, "median_ms": rec["median_ms"],
                    "min_ms": rec["min_ms"], "nregions": rec["nregions"],
                    "errorFlag": rec["errorFlag"], "integral": rec["integral"]})
        total_ms += rec["median_ms"]
    return {"value": len(per) / (total_ms / 1e3), "unit": "integrals/s",
            "ms_per_step": total_ms, "per_integrand": per, "reps": reps, "warmup": warmup,
            "source": "unmodified reference engine (quad::GPUcuhre) built from its sources by "
                      "oracle/ref_driver/Makefile; warm median of steady-clock times around "
                      "integrate(), device synchronised on both sides"}


def cv_side_block(ctx, cub, count: int, epsrel: float = 1e-6, epsabs: float = 1e-12) -> dict:
    """The learned control variate against the plain method on the same
    integrands (the 7-D product-peak batch, seeds 0..count-1): one pass of
    each, timed with the device synchronised on both sides; an integral
    counts when it converged and lies within epsrel of the analytic value."""
    import torch
    import oracle as O

    n = 7
    cases = product_peak_params(n, count)
    plist = [cub.make_params(n, a, u) for a, u in cases]
    exact = [O.exact(O.make_integrand("product_peak", n, a, u)) for a, u in cases]

    def verified(res):
        return sum(1 for r, ex in zip(res, exact)
                   if r.status == 0 and abs(r.integral - ex) <= epsrel * abs(ex))

    out = {"workload": "cv_productpeak_7d_batch", "integrals": count, "epsrel": epsrel,
           "epsabs": epsabs, "target_ratio": 3.0}
    try:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res_cv, st = ctx.cv_integrate_batch("product_peak", plist, epsrel, epsabs)
        torch.cuda.synchronize()
        t_cv = time.perf_counter() - t0
        t0 = time.perf_counter()
        res_pl = ctx.integrate_batch("product_peak", n, plist, epsrel, epsabs,
                                     cub.options(policy=cub.POLICY_BREADTH))
        torch.cuda.synchronize()
        t_pl = time.perf_counter() - t0
    except Exception as e:  # reported, the headline line still prints
        out["error"] = f"{type(e).__name__}: {e}"
        return out
    g_cv, g_pl = verified(res_cv), verified(res_pl)
    out["cv"] = {"value": g_cv / t_cv, "unit": "integrals/s", "seconds": t_cv, "verified": g_cv,
                 "regions": int(sum(r.nregions for r in res_cv)),
                 "fallbacks": int(st["fallbacks"]), "rejected": int(st["rejected"]),
                 "mean_residual_ratio": st["mean_residual_ratio"],
                 "ms_coarse": st["ms_coarse"], "ms_train": st["ms_train"],
                 "ms_integrate": st["ms_integrate"],
                 "regions_residual": int(st["regions_residual"]),
                 "regions_network": int(st["regions_network"])}
    out["plain"] = {"value": g_pl / t_pl, "unit": "integrals/s", "seconds": t_pl,
                    "verified": g_pl, "regions": int(sum(r.nregions for r in res_pl))}
    out["ratio"] = out["cv"]["value"] / out["plain"]["value"] if out["plain"]["value"] else None
    return out


def cpu_sample_text(workload: dict, done: int, el: float,
                    regions_per_integral: float | None = None) -> str:
    if "tables" in workload:
        per = regions_per_integral or TABLE7_REGIONS_PER_INTEGRAL
        return (f"{done} integrals at epsrel 1e-4 in {el:.1f} s; their regions/s divided by "
                f"{per:.4g} regions per integral at epsrel 1e-6 "
                "(oracle engine, OpenMP over regions)")
    return (f"{done} whole integrals of the workload in {el:.1f} s "
            "(oracle two-phase engine, OpenMP over regions)")


def run_reference(args, workload, world, rank):
    """The reference arm: CPU implementation of the path on the host cores."""
    if rank != 0:
        return 0
    per_step = max(1.0, 30.0 / max(1, args.steps + args.warmup))
    for _ in range(args.warmup):
        cpu_reference_rate(workload, per_step * 0.25)
    rates, evr = [], []
    for _ in range(args.steps):
        r, e, cores, done, el = cpu_reference_rate(workload, per_step)
        rates.append(r)
        evr.append(e)
    value = statistics.median(rates)
    line = {
        "impl": "reference", "metric": "integrals/s", "value": value, "unit": "integrals/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 / value, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "epsrel": workload["epsrel"]},
        "geval_per_s": statistics.median(evr) / 1e9,
        "cpu_baseline": {"value": value, "unit": "integrals/s", "cores": cores, "kind": "port",
                         "sample": cpu_sample_text(workload, done, el)},
        "e2e": {"value": value, "unit": "integrals/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main() -> int:
    faulthandler.enable()
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="oscillatory_cornerpeak_8d")
    ap.add_argument("--cpu-seconds", type=float, default=8.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="skip timing the reference engine on the GPU beside the run")
    ap.add_argument("--no-device-loop", action="store_true",
                    help="long lists: the host launches every iteration (cub_options."
                         "no_device_loop) instead of one graph launch per stretch")
    ap.add_argument("--no-check-exit", action="store_true",
                    help="exit 0 even when integrals miss the check (profiling runs of "
                         "workloads whose misses are the algorithm's own)")
    ap.add_argument("--no-cv", action="store_true",
                    help="skip the learned-control-variate side block of the default workload")
    ap.add_argument("--cv-count", type=int, default=64,
                    help="integrals of the control-variate side block (the first of the "
                         "256-integral configuration; --cv-count 256 runs all of it)")
    ap.add_argument("--count", type=int, default=0,
                    help="batch workloads: integrals per step (default: the workload's)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    workload = dict(WORKLOADS[args.workload])
    for key in ("batch", "tables", "cv"):
        if args.count and key in workload:
            fam, n, _ = workload[key]
            workload[key] = (fam, n, args.count)
    world, rank, local = dist_setup()

    if args.impl == "reference":
        return run_reference(args, workload, world, rank)

    import torch
    import cubature as cub

    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
        pg = dist

    ctx = cub.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream, device=f"cuda:{local}")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    # the step: integrate the workload through the public C ABI
    opts = cub.options(policy=cub.POLICY_BREADTH if workload.get("policy") == "breadth"
                       else cub.POLICY_REFERENCE, device_loop=not args.no_device_loop)
    if "items" in workload:
        items = [cub.Integrand(f, n, a, u) for f, n, a, u in workload["items"]]

        same_dim = len({f.ndim for f in items}) == 1

        def single_calls():
            return [ctx.integrate(f, workload["epsrel"], workload["epsabs"], opts) for f in items]

        def step():
            # one public-API call per integrand, the reference's calling
            # pattern (one mixed-family call, cub_integrate_mixed_batch, is
            # measured beside it)
            return single_calls()

        def mixed_call():
            return ctx.integrate_mixed(items, workload["epsrel"], workload["epsabs"], opts)

        fams = [(f.family, f.ndim) for f in items]
        exact = []
        import oracle as O

        for f in items:
            exact.append(O.exact(O.make_integrand(f.family, f.ndim, f.a, f.u)))
    elif "cv" in workload:
        from cubature.parallel import shard_bounds

        fam, n, count = workload["cv"]
        a0, b0 = shard_bounds(world * count, world, rank)
        cases = product_peak_params(n, world * count)[a0:b0]
        plist = [cub.make_params(n, a, u) for a, u in cases]
        cv_stats = {}

        def step():
            res, st_cv = ctx.cv_integrate_batch(fam, plist, workload["epsrel"], workload["epsabs"])
            cv_stats.update(st_cv)
            return res

        def plain_step():
            return ctx.integrate_batch(fam, n, plist, workload["epsrel"], workload["epsabs"], opts)

        fams = [(fam, n)] * len(plist)
        import oracle as O

        exact = [O.exact(O.make_integrand(fam, n, a, u)) for a, u in cases]
    elif "tables" in workload:
        from cubature import tables as T
        from cubature.parallel import shard_bounds

        fam, n, count = workload["tables"]
        a0, b0 = shard_bounds(world * count, world, rank)
        offs = list(T.table7_offsets(world * count)[a0:b0])
        tab = T.Table7(T.table7_data(0), local)

        def step():
            return ctx.integrate_table7_batch(tab, offs, workload["epsrel"], workload["epsabs"],
                                              opts)

        fams = [(fam, n)] * len(offs)
        import oracle as O

        d7 = T.table7_data(0)
        exact = [O.table7_exact(d7["spline_x"], d7["spline_y"], d7["grid_x"], d7["grid_y"],
                                d7["grid_z"], d7["sigma"], o) for o in offs]
    else:
        # weak scaling: `count` integrals per rank; the job's world * count
        # integrals (seed = global index) are dealt to the ranks by a greedy
        # split of their probe costs (region counts at a 100x looser
        # tolerance, probed once before the timed steps)
        from cubature.parallel import balanced_assignment, probe_costs

        fam, n, count = workload["batch"]
        all_cases = product_peak_params(n, world * count)
        if world > 1:
            all_params = [cub.make_params(n, a, u) for a, u in all_cases]
            costs = probe_costs(ctx, fam, n, all_params, workload["epsrel"], workload["epsabs"],
                                opts)
            mine = balanced_assignment(costs, world)[rank]
        else:
            mine = list(range(count))
        cases = [all_cases[i] for i in mine]
        plist = [cub.make_params(n, a, u) for a, u in cases]

        def step():
            return ctx.integrate_batch(fam, n, plist, workload["epsrel"], workload["epsabs"], opts)

        fams = [(fam, n)] * len(plist)
        import oracle as O

        exact = [O.exact(O.make_integrand(fam, n, a, u)) for a, u in cases]

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    # regions per (family, ndim) in the persistent kernels and in the
    # multi-launch rule kernel, from one untimed step with the counters read
    # after each call
    split = {}

    def add_split(key, total, s0):
        pk, ml = s0["persistent_regions"], s0["regions_evaluated"]
        a, b, c = split.get(key, (0, 0, 0))
        split[key] = (a + pk, b + ml, c + max(0, total - pk - ml))

    if "items" in workload:
        for f, key in zip(items, fams):
            ctx.reset_stats()
            r = ctx.integrate(f, workload["epsrel"], workload["epsabs"], opts)
            add_split(key, r.nregions, ctx.stats())
    else:
        ctx.reset_stats()
        res0 = step()
        add_split(fams[0], sum(r.nregions for r in res0), ctx.stats())
    torch.cuda.synchronize()

    ctx.reset_stats()
    step_ms, wall_ms = [], []
    results = None
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            if pg:
                pg.barrier()
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            t0 = time.perf_counter()
            results = step()
            t1 = time.perf_counter()
            ev1.record(stream)
            torch.cuda.synchronize()
            step_ms.append(ev0.elapsed_time(ev1))
            wall_ms.append((t1 - t0) * 1e3)
    st = ctx.stats()
    # Kernel durations for the roofline: the same steps again with the
    # library's CUDA events around every launch (counters reset).  Timing
    # makes the library wait for each launch with a stream synchronisation
    # instead of its completion word, so `value` and `e2e` come from the
    # untimed pass above.
    ctx.reset_stats()
    ctx.set_timing(True)
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        step()
        torch.cuda.synchronize()
    ctx.set_timing(False)
    st_timed = ctx.stats()
    for key in ("ms_persistent", "ms_eval", "ms_phase2"):
        st[key] = st_timed[key]
    plain_cmp = None
    single_cmp = None
    if "items" in workload and len(workload["items"]) > 1 and same_dim:
        # the same integrals in one mixed-family call, timed the same way
        ms = []
        for _ in range(max(3, args.steps)):
            flush.zero_()
            torch.cuda.synchronize()
            s0 = torch.cuda.Event(enable_timing=True)
            s1 = torch.cuda.Event(enable_timing=True)
            s0.record(stream)
            mixed_call()
            s1.record(stream)
            torch.cuda.synchronize()
            ms.append(s0.elapsed_time(s1))
        single_cmp = {"value": len(items) * len(ms) / (sum(ms) / 1e3), "unit": "integrals/s",
                      "ms_per_step": sum(ms) / len(ms),
                      "call": "cub_integrate_mixed_batch, all integrands in one call"}
    graph_cmp = None
    if "items" in workload:
        # the same integrals as one replayed CUDA graph (cub_graph_launch:
        # one graph launch and one wait per step), timed the same way
        g = ctx.graph([(f.family, f.ndim, 1) for f in items], opts)
        for _ in range(3):
            g.launch(items, workload["epsrel"], workload["epsabs"])
        ms, wms = [], []
        for _ in range(max(3, args.steps)):
            flush.zero_()
            torch.cuda.synchronize()
            s0 = torch.cuda.Event(enable_timing=True)
            s1 = torch.cuda.Event(enable_timing=True)
            s0.record(stream)
            t0 = time.perf_counter()
            g.launch(items, workload["epsrel"], workload["epsabs"])
            t1 = time.perf_counter()
            s1.record(stream)
            torch.cuda.synchronize()
            ms.append(s0.elapsed_time(s1))
            wms.append((t1 - t0) * 1e3)
        replays, reruns = g.info()
        g.close()
        graph_cmp = {"value": len(items) * len(ms) / (sum(ms) / 1e3), "unit": "integrals/s",
                     "e2e": len(items) * len(wms) / (sum(wms) / 1e3),
                     "ms_per_step": sum(ms) / len(ms), "replays": replays, "reruns": reruns,
                     "call": "cub_graph_launch, every integrand in one replayed CUDA graph"}
    if "cv" in workload:
        # the plain method on the same integrands, same tolerance, one pass
        torch.cuda.synchronize()
        p0 = time.perf_counter()
        plain_res = plain_step()
        torch.cuda.synchronize()
        p_s = time.perf_counter() - p0
        plain_cmp = {"value": len(plain_res) / p_s, "unit": "integrals/s",
                     "regions": int(sum(r.nregions for r in plain_res)),
                     "cv_stats": dict(cv_stats)}

    # correctness of the last step against the analytic (or closed-form)
    # integrals: an integral counts when it converged (status 0) and lies
    # within epsrel of the true value; the looser 2 epsrel count is reported
    # beside it
    nint = len(results)
    bad = bad2 = 0
    for r, ex in zip(results, exact):
        ok1 = r.status == 0 and (ex is None or abs(r.integral - ex) <= workload["epsrel"] * abs(ex))
        ok2 = r.status == 0 and (ex is None or
                                 abs(r.integral - ex) <= 2 * workload["epsrel"] * abs(ex))
        bad += 0 if ok1 else 1
        bad2 += 0 if ok2 else 1
    neval = sum(r.neval for r in results)
    nreg = {}
    for (fam, n), r in zip(fams, results):
        nreg[(fam, n)] = nreg.get((fam, n), 0) + r.nregions

    dev_ms = sum(step_ms)
    wall = sum(wall_ms)
    if pg:
        t = torch.tensor([dev_ms, wall], dtype=torch.float64, device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        dev_ms, wall = float(t[0]), float(t[1])
        # ranks may hold different numbers of integrals (balanced shares)
        fb = torch.tensor([float(bad), float(bad2), float(nint), float(neval)],
                          dtype=torch.float64, device="cuda")
        pg.all_reduce(fb, op=pg.ReduceOp.SUM)
        bad, bad2, n_all, neval_all = int(fb[0]), int(fb[1]), int(fb[2]), int(fb[3])
    else:
        n_all, neval_all = nint, neval
    good = n_all - bad
    value = good * args.steps / (dev_ms / 1e3)
    e2e_value = good * args.steps / (wall / 1e3)

    # roofline of the dominant kernel (FP64-bound rule evaluation).  The
    # regions are split between the persistent kernel (short lists) and the
    # multi-launch rule kernel (long lists); each gets its own share of the
    # algorithmic flops (per-region flops x regions it evaluated).
    # Roofline of the dominant kernel (FP64-bound rule evaluation).  Each
    # kernel gets the algorithmic flops of the regions it evaluated, per
    # (family, ndim): the split of every integrand's regions between the
    # persistent kernels and the multi-launch rule kernel is taken from one
    # untimed pass with the counters read after each call (the split is the
    # same every step).
    persist_flops = ml_flops = p2_flops = 0.0
    for (fam, n), (pk_r, ml_r, p2_r) in split.items():
        persist_flops += pk_r * flops_per_region(fam, n) * args.steps
        ml_flops += ml_r * flops_per_region(fam, n) * args.steps
        p2_flops += p2_r * flops_per_region(fam, n) * args.steps
    pk_name = "k_replicated" if st.get("replicated_launches", 0) >= max(
        1, st["persistent_launches"] - st.get("replicated_launches", 0)) else "k_persistent"
    kernels = {
        pk_name: (persist_flops, st["ms_persistent"]),
        "k_eval": (ml_flops, st["ms_eval"]),
        "k_phase2": (p2_flops, st["ms_phase2"]),
    }
    dom = max(kernels, key=lambda k: kernels[k][1])
    dom_flops, dom_ms = kernels[dom]
    achieved = dom_flops / (dom_ms / 1e3) / 1e12 if dom_ms > 0 else None
    peak = cub.fp64_peak(local) if rank == 0 else None
    peak_dgemm = measure_fp64_peak(torch) if rank == 0 else None

    cpu = None
    if rank == 0 and not args.no_cpu:
        per = sum(nreg.values()) / max(1, nint) if "tables" in workload else None
        rate, evr, cores, done, el = cpu_reference_rate(workload, args.cpu_seconds,
                                                        regions_per_integral=per)
        rate1, _, _, done1, el1 = cpu_reference_rate(workload, args.cpu_seconds / 2, threads=1,
                                                     regions_per_integral=per)
        cpu = {"value": rate, "unit": "integrals/s", "cores": cores, "kind": "port",
               "sample": cpu_sample_text(workload, done, el, per), "cpu_model": cpu_model(),
               "one_thread": {"value": rate1, "unit": "integrals/s", "cores": 1,
                              "sample": cpu_sample_text(workload, done1, el1, per)}}
    cv_side = None
    if rank == 0 and "items" in workload and not args.no_cv and args.cv_count > 0:
        cv_side = cv_side_block(ctx, cub, args.cv_count)
    ref_gpu = None
    if rank == 0 and not args.no_ref_gpu:
        ref_gpu = reference_gpu_rate(workload, 3, max(5, args.steps), local)

    if rank == 0:
        line = {
            "metric": "integrals/s", "value": value, "unit": "integrals/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": args.workload, "integrals_per_step": nint,
                       "policy": workload.get("policy", "reference"),
                       "epsrel": workload["epsrel"], "epsabs": workload["epsabs"],
                       "parallelism": ("replicas" if "items" in workload else
                                       (f"balanced_shards{world}" if "batch" in workload
                                        else f"shards{world}")) if world > 1 else "single",
                       "l2": "flushed between steps (256 MB write)",
                       "device_loop": not args.no_device_loop,
                       "regions_per_step": int(sum(nreg.values())),
                       "timing": "value: CUDA events on the library's stream around each "
                                 "step's public-API calls (inputs are parameter blocks; the "
                                 "host drives the launches); e2e: host wall clock around "
                                 "the same calls; roofline kernel times: a second pass of "
                                 "the same steps with the library's per-launch events on"},
            "geval_per_s": neval_all * args.steps / (dev_ms / 1e3) / 1e9,
            "e2e": {"value": e2e_value, "unit": "integrals/s",
                    "h2d_bytes_per_step": st.get("h2d_bytes", 0) // max(1, args.steps),
                    "d2h_bytes_per_step": st.get("d2h_bytes", 0) // max(1, args.steps)},
            "gpu_launches": st["launches"],
            "roofline": {"kernel": dom, "bound": "fp64", "pipe": "fp64 (CUDA cores)",
                         "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": (achieved / peak) if achieved and peak else None,
                         "traffic": profiled_traffic(dom, args.workload),
                         "peak_source": "in-run DFMA throughput loop on the FP64 CUDA cores "
                                        "(cub_fp64_peak); MEASURED_PEAKS.json has no FP64 figure",
                         "peak_dgemm": peak_dgemm,
                         "peak_dgemm_source": "in-run cuBLAS DGEMM 8192^3 (FP64 tensor path)",
                         "kernel_ms_per_step": {k: v[1] / args.steps for k, v in kernels.items()},
                         "algorithmic_flops_per_step": {k: v[0] / args.steps
                                                        for k, v in kernels.items()},
                         "regions_per_step": {pk_name: sum(v[0] for v in split.values()),
                                              "k_eval": sum(v[1] for v in split.values()),
                                              "k_phase2": sum(v[2] for v in split.values())},
                         "persistent_iterations_per_step": st["persistent_iterations"] / args.steps,
                         "eval_launches_per_step": st["eval_launches"] / args.steps},
            "cpu_baseline": cpu,
            "clocks": clocks.summary(),
            "check": {"integrals": n_all, "failed": bad, "failed_2epsrel": bad2,
                      "rule": "status 0 and |I - I*| <= epsrel |I*| against the analytic or "
                              "closed-form I*; value and e2e count only the integrals that "
                              "pass (failed_2epsrel: the same test at 2 epsrel)"},
        }
        if ref_gpu is not None:
            line["reference_gpu"] = ref_gpu
        if cv_side is not None:
            line["cv_vs_plain"] = cv_side
        if plain_cmp is not None:
            line["plain_same_integrands"] = plain_cmp
        if single_cmp is not None:
            line["config"]["call"] = "cub_integrate, one call per integrand"
            line["mixed_call"] = single_cmp
        if graph_cmp is not None:
            line["graph_call"] = graph_cmp
        print(json.dumps(line), flush=True)
    ctx.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    # integrals that miss the analytic value by more than 2 epsrel (or do not
    # converge) are counted in "check" and fail the run
    return 1 if bad and not args.no_check_exit else 0


if __name__ == "__main__":
    sys.exit(main())
