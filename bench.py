#!/usr/bin/env python
"""bench.py — k-point·steps/s of the EDUS k-space propagation on B200.

Workload (N=1): config 1 — hBN-type Haldane_CoreBN_Nedge model (3 bands, core band
decoupled), 120x120 Monkhorst–Pack grid, Rytova–Keldysh Coulomb mean field from
the shipped Ncut=20 coefficient files, Adams–Bashforth 4 with RK4 start-up,
dt = 0.005 fs, 30 fs sin^2 pulse at 0.4 eV and 0.5 V/A, FP64. One bench step is
one complete solve (6043 time steps of 14400 k points). Inputs are synthetic
(generated by edus_b200.workloads); nothing is read from the reference.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
  python bench.py --workload wannier|sweep|serve [--requests R]

--workload selects the batched / served measurements of edus_b200.suite
(8-band Wannier solves, the 256-instance pulse sweep, the request stream),
each against the plain FP64 single-solve path and with the J(t) error of the
mixed-precision path.

N > 1 runs one independent solve per GPU (replicas, weak scaling); the time is
the max over ranks. --impl reference times the CPU restatement of the reference
(the oracle; the reference itself needs MPI/Armadillo and is not built here) on
the host cores, rank 0 only.
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "hbn_coulomb_120x120_ab4_rk4start_dt0.005fs_30fs_fp64"
METRIC = "k-point·steps/s"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="budget of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", choices=["coulomb", "wannier", "sweep", "serve"], default="coulomb")
    ap.add_argument("--requests", type=int, default=2000, help="serve: requests in the stream")
    ap.add_argument("--rate", type=float, default=None, help="serve: Poisson arrival rate (1/s); default all at once")
    return ap.parse_args()


def dist_env():
    from edus_b200.replicas import dist_env as env

    return env()


def make_workload(workdir):
    from edus_b200 import workloads as W

    return W.hbn_coulomb(workdir)


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (of measured)"
    except Exception:
        return 6650.0, "fallback 6.65 TB/s (of fallback)"


def ncu_traffic(kernel):
    """Per-launch DRAM bytes of `kernel` recorded from an ncu capture in profiles/."""
    path = os.path.join(ROOT, "profiles", "roofline_traffic.txt")
    try:
        for line in open(path):
            s = line.split()
            if len(s) >= 2 and s[0] == kernel:
                return float(s[1])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1].split()[0]))
                mx = max(mx, float(parts[2].split()[0]))
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.f.name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline_oracle(path, workdir, budget_s, threads):
    """Time the oracle on a bounded sample (the first S time steps) of the workload."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    import edus_b200 as E
    from oracle_lib import Oracle

    p = E.parse_input(path)
    o = Oracle(p, workdir)
    t0 = time.perf_counter()
    o.run(2)
    per = max((time.perf_counter() - t0) / 2, 1e-6)
    o.close()
    S = int(max(2, min(o.info.nsteps, budget_s / per)))
    o = Oracle(p, workdir)
    t0 = time.perf_counter()
    o.run(S)
    dt = time.perf_counter() - t0
    nk = o.info.nk
    o.close()
    return {"value": nk * S / dt, "unit": METRIC, "cores": threads, "kind": "port",
            "sample": f"{WORKLOAD}: first {S} of {o.info.nsteps} time steps on {nk} k points, {dt:.1f} s"}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    d = tempfile.mkdtemp(prefix="edus_ref_")
    path = make_workload(d)
    budget = max(2.0, min(20.0, 150.0 / max(1, args.steps + args.warmup)))
    for _ in range(args.warmup):
        cpu_baseline_oracle(path, d, budget / 4, threads)
    vals = []
    for _ in range(args.steps):
        vals.append(cpu_baseline_oracle(path, d, budget, threads))
    v = statistics.mean(x["value"] for x in vals)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": WORKLOAD, "nk": 14400, "bands": 3},
            "cpu_baseline": {"value": v, "unit": METRIC, "cores": threads, "kind": "port", "sample": vals[-1]["sample"]},
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch

    from edus_b200.replicas import ReplicaGroup, whole_job_rate

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    group = ReplicaGroup("nccl", device=f"cuda:{local}")
    import edus_b200 as E

    d = tempfile.mkdtemp(prefix="edus_bench_")
    path = make_workload(d)
    p = E.parse_input(path)
    pb = E.Problem(p, d)
    ctx = E.Context(pb, device=local)
    nk, nsteps, n = pb.info.nk, pb.info.nsteps, pb.info.ncv
    units = nk * nsteps  # k-point·steps per solve
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")  # > 126 MB L2

    barrier = group.barrier

    for _ in range(max(args.warmup, 1)):  # the first run captures the CUDA graph
        ctx.reset()
        ctx.run()
    sampler = ClockSampler(local)
    sampler.start()
    barrier()
    dev_ms = []
    launches = 0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        ctx.reset()
        ctx.run()
        ms, l = ctx.last_timing()
        dev_ms.append(ms)
        launches += l
    barrier()
    clocks = sampler.stop()
    max_ms = group.max(sum(dev_ms))
    value = whole_job_rate(world, units, args.steps, max_ms * 1e-3)

    # end to end through the C ABI with host buffers: H2D of the initial state,
    # the solve, D2H of the observable log and of the final state
    rho0 = pb.get("P0")
    host_rho = np.empty_like(rho0)
    barrier()
    t0 = time.perf_counter()
    nobs = 0
    for _ in range(args.steps):
        ctx.reset()
        ctx.set_state(rho0)
        ctx.run()
        obs = ctx.obs()
        host_rho[...] = ctx.get_state()
        nobs = len(obs)
    torch.cuda.synchronize()
    e2e_value = whole_job_rate(world, units, args.steps, group.max(time.perf_counter() - t0))
    obs_bytes = nobs * C.sizeof(E.abi.Obs)

    # live roofline of the dominant kernel (fused RHS + AB update), CUDA events on its stream
    # (each AB launch of the profiled steps runs 8 times back to back between its
    # events: the kernel's duration in a pipeline, not one event pair's overhead)
    ctx.reset()
    prof = ctx.profile(min(600, nsteps), reps=8)
    per_launch_ms = prof["rhs_ms"] / max(prof["rhs_launches"], 1)
    # algorithmic bytes per k point for one RHS + AB4 update (full n x n matrices, complex128):
    # rho read + write 32 n^2, H and D_xyz 64 n^2, AB history (3 reads + 1 write) 64 n^2
    bytes_per_k = 32 * n * n + 64 * n * n + 16 * n * n * 4
    alg_bytes = bytes_per_k * nk
    achieved = alg_bytes / (per_launch_ms * 1e-3) / 1e9
    peak, peak_src = measured_peaks()
    kern = f"k_rhs_ep<{n},32>"
    traffic = ncu_traffic(kern)

    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            try:
                cpu = cpu_baseline_oracle(path, d, args.cpu_seconds, os.cpu_count() or 1)
            except Exception as ex:  # the baseline is reported, not required
                cpu = {"error": str(ex)}
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "nk": nk, "bands": n, "time_steps_per_solve": nsteps,
                       "step": "one full solve", "l2": "flushed between timed solves (256 MiB write)",
                       "parallelism": f"replicas x{world}", "graph": "whole time loop captured in one CUDA graph"},
            "roofline": {"bound": "hbm", "kernel": kern, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "algorithmic_bytes_per_launch": alg_bytes,
                         "launch_ms": per_launch_ms, "peak_source": peak_src,
                         "launch_timing": "CUDA events on the context stream around 8 back-to-back repeats of each "
                                          "AB launch of the profiled steps, averaged over launches",
                         "coulomb_pair_ms": prof["coulomb_ms"] / max(prof["coulomb_launches"], 1)},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": int(rho0.nbytes),
                    "d2h_bytes_per_step": int(obs_bytes + host_rho.nbytes)},
            "gpu_launches": launches,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    group.close()
    return 0


def run_suite(args):
    import torch

    from edus_b200 import suite

    torch.cuda.set_device(0)
    sampler = ClockSampler(0)
    sampler.start()
    if args.workload == "wannier":
        line = suite.wannier_line()
    elif args.workload == "sweep":
        line = suite.sweep_line()
    else:
        line = suite.serve_line(count=args.requests, rate=args.rate)
    line.update({"n_gpus": 1, "clocks": sampler.stop()})
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload != "coulomb":
        return run_suite(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
