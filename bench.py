#!/usr/bin/env python
"""bench.py — k-point·steps/s of the EDUS k-space propagation on B200.

Default workload (configuration 3, the batched pulse sweep): the seeded
256-instance sweep — half the hBN two-band model (Haldane_CoreBN_Nedge with
its decoupled core band dropped), half the synthetic 8-band Wannier model
(11x11 R vectors); grids N x N, N even in 48..144; peak field log-uniform in
0.05-0.8 V/A; CEP uniform; 10-60 fs sin^2 pulses at 0.4 / 0.3 eV; RK4,
dt 0.01 fs — in one mixed-precision batch (FP32 H, D and commutator, FP64
state and observables), run as a continuous sweep: one bench step advances
every live instance by 128 time steps (graph-replayed chunks of persistent
kernels), then retires each instance whose time grid has ended (its
observable log copied to the host) and admits it again from its input file
(parse, host set-up, upload), so 256 instances stay live.

  value  k-point·steps of the K timed steps / their CUDA-event device time
  e2e    the same k-point·steps / the wall time of the timed steps, which
         includes every retirement (D2H of the logs) and re-admission
         (input parse, host set-up, H2D of tables, state and field)

Beside it, on the same instances: the plain FP64 single-solve path run
request by request on a stratified sample (per-model rates weighted by the
sweep's mix of k-point·steps), the FP64 batch, the speed-ups (batching and
precision separately), the mixed path's J1 / population / rho errors against
the FP64 path, the live roofline of the dominant batch kernel, and
configuration 1 (hBN + Rytova-Keldysh mean field, 120x120, AB4 with RK4
start-up, dt 0.005 fs, 30 fs, FP64 single solve) as a second workload.
Inputs are synthetic (edus_b200.workloads, seeded).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
  python bench.py --workload coulomb|wannier|serve [--requests R] [--rate r]

--impl reference times the reference program itself on the host cores
(oracle/_ref/EDUS.x: anpicon/EDUS compiled from its sources with one MPI rank,
`make -C oracle ref`; the oracle's C restatement if that binary is absent) on
a bounded sample of the same sweep, rank 0 only. N > 1 runs one independent
sweep per GPU (replicas, weak scaling); the time is the max over ranks.
"""
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
# requests with the Coulomb mean field run as contexts on streams of their own:
# more hardware queues than the default 8 let those streams overlap
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

SWEEP = "pulse_sweep_256_hbn2+wannier8_48-144_10-60fs_rk4_dt0.01fs_mixed"
COULOMB = "hbn_coulomb_120x120_ab4_rk4start_dt0.005fs_30fs_fp64"
METRIC = "k-point·steps/s"
STEP_TIME_STEPS = 128
TIME_AU_FS = 0.02418884326505
REF_EXE = os.path.join(ROOT, "oracle", "_ref", "EDUS.x")


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-seconds", type=float, default=20.0, help="budget of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", choices=["sweep", "coulomb", "wannier", "serve"], default="sweep")
    ap.add_argument("--requests", type=int, default=2000, help="serve: requests in the stream")
    ap.add_argument("--rate", type=float, default=None, help="serve: Poisson arrival rate (1/s)")
    return ap.parse_args()


def dist_env():
    from edus_b200.replicas import dist_env as env

    return env()


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (of measured)"
    except Exception:
        return 6650.0, "fallback 6.65 TB/s (of fallback)"


def ncu_traffic(kernel, kpoints=None):
    """Per-launch DRAM bytes of `kernel` from an ncu capture recorded in
    profiles/roofline_traffic.txt: `<kernel> <bytes per launch>`, or
    `<kernel> per_kpoint <bytes>` for a capture of a smaller launch of the same
    kernel, scaled here by the k points of this launch."""
    path = os.path.join(ROOT, "profiles", "roofline_traffic.txt")
    try:
        for line in open(path):
            s = line.split()
            if len(s) >= 3 and s[0] == kernel and s[1] == "per_kpoint":
                return float(s[2]) * kpoints if kpoints else None
            if len(s) >= 2 and s[0] == kernel and s[1] != "per_kpoint":
                return float(s[1])
    except OSError:
        pass
    return None


def host_cores():
    """(CPUs this process may run on, physical cores of the host from lscpu)."""
    try:
        logical = len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        logical = os.cpu_count() or 1
    try:
        out = subprocess.run(["lscpu", "-p=CORE,SOCKET"], capture_output=True, text=True, timeout=10).stdout
        phys = len({ln for ln in out.splitlines() if ln and not ln.startswith("#")})
    except Exception:
        phys = None
    return logical, phys or logical


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


# ------------------------------------------------------------------ sweep inputs (no GPU, no product library)

def sweep_specs():
    from edus_b200 import workloads as W

    return W.sweep(256)


def spec_units(spec):
    """k-point·steps of one sweep instance: N^2 x the reference loop's step count
    (t from -0.21 fs to the pulse end, dt 0.01 fs, it = 0..itfi)."""
    dt = spec["dt_fs"] / TIME_AU_FS
    t0 = -0.21 / TIME_AU_FS
    itfi = int((spec["duration"] / TIME_AU_FS - t0) / dt)
    return spec["n"] * spec["n"] * (itfi + 1)


def kind_weights(specs):
    """Share of the sweep's k-point·steps per model."""
    tot = {}
    for s in specs:
        tot[s["kind"]] = tot.get(s["kind"], 0.0) + spec_units(s)
    return tot


def mix_rate(rates, units):
    """Rate of the whole mix from per-model rates: total work / sum of per-model times."""
    return sum(units.values()) / sum(units[k] / rates[k] for k in units)


def write_sweep_instance(root, i, spec, t_fin_fs=None):
    from edus_b200 import workloads as W

    d = os.path.join(root, f"i{i}" + ("" if t_fin_fs is None else f"_t{t_fin_fs:.4f}"))
    os.makedirs(d, exist_ok=True)
    if spec["kind"] == "hbn":
        path = W.hbn_rk4(d, n=spec["n"], field=spec["field"], duration=spec["duration"], it_res=spec["it_res"],
                         dt_fs=spec["dt_fs"], phase=spec["phase"], t_fin_fs=t_fin_fs)
    else:
        model = os.path.join(root, "W8_tb.dat")
        if not os.path.exists(model):
            W.write_wannier_tb(model)
        link = os.path.join(d, "W8_tb.dat")
        if not os.path.exists(link):
            os.symlink(model, link)
        path = W.wannier(d, n=spec["n"], field=spec["field"], duration=spec["duration"], it_res=spec["it_res"],
                         dt_fs=spec["dt_fs"], phase=spec["phase"], t_fin_fs=t_fin_fs, write_model=False)
    return path, d


def median_instance(specs, kind):
    ks = sorted((s["n"], i) for i, s in enumerate(specs) if s["kind"] == kind)
    return ks[len(ks) // 2][1]


# ------------------------------------------------------------------ CPU: the reference program on a sweep sample

class ReferenceSample:
    """The reference program (oracle/_ref/EDUS.x, all host threads) on one
    median-grid instance per model of the sweep. Each measurement runs the
    instance to step S0 + dS and subtracts a calibrated run to step S0 (the
    pulse starts at step 21, so every timed step is inside the pulse and the
    process start and set-up cancel): rate = N^2 dS / (wall(S0 + dS) - wall(S0))."""

    S0 = 40

    def __init__(self, root, threads, budget_s):
        self.specs = sweep_specs()
        self.root = root
        self.threads = threads
        self.units = kind_weights(self.specs)
        self.pick = {k: median_instance(self.specs, k) for k in ("hbn", "wannier")}
        self.base = {}
        self.dS = {}
        per_kind = max(1.0, budget_s / 2.0)
        for k, i in self.pick.items():
            w0 = self._wall(i, self.S0)
            w1 = self._wall(i, self.S0 + 20)
            per_step = max((w1 - w0) / 20.0, 1e-5)
            self.base[k] = w0
            self.dS[k] = int(min(4000, max(20, per_kind / per_step)))

    def _wall(self, i, steps):
        spec = self.specs[i]
        t_fin = -0.21 + (steps + 0.5) * spec["dt_fs"]
        path, d = write_sweep_instance(self.root, i, spec, t_fin_fs=t_fin)
        os.makedirs(os.path.join(d, "Output"), exist_ok=True)
        env = dict(os.environ, OMP_NUM_THREADS=str(self.threads))
        t0 = time.perf_counter()
        r = subprocess.run([REF_EXE, os.path.basename(path)], cwd=d, env=env, capture_output=True, text=True)
        w = time.perf_counter() - t0
        if r.returncode != 0:
            raise RuntimeError(f"reference exited {r.returncode}: {r.stderr[-500:]}")
        return w

    def measure(self):
        rates, detail = {}, {}
        for k, i in self.pick.items():
            n = self.specs[i]["n"]
            w = self._wall(i, self.S0 + self.dS[k])
            rates[k] = n * n * self.dS[k] / max(w - self.base[k], 1e-6)
            detail[k] = {"instance": i, "grid": f"{n}x{n}", "timed_steps": self.dS[k], "kpoint_steps_per_s": rates[k]}
        return mix_rate(rates, self.units), detail


class OracleSample:
    """Fallback when the reference binary is absent: the oracle's C restatement
    (test infrastructure) on the same instances and steps, timed in process."""

    S0 = 40

    def __init__(self, root, threads, budget_s):
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        os.environ["OMP_NUM_THREADS"] = str(threads)
        self.specs = sweep_specs()
        self.root = root
        self.units = kind_weights(self.specs)
        self.pick = {k: median_instance(self.specs, k) for k in ("hbn", "wannier")}
        self.budget = budget_s

    def measure(self):
        import edus_b200 as E
        from oracle_lib import Oracle

        rates, detail = {}, {}
        for k, i in self.pick.items():
            spec = self.specs[i]
            path, d = write_sweep_instance(self.root, i, spec)
            o = Oracle(E.parse_input(path), d)
            o.run(self.S0)
            t0 = time.perf_counter()
            o.run(10)
            per = (time.perf_counter() - t0) / 10
            dS = int(min(2000, max(10, self.budget / 2 / max(per, 1e-6))))
            t0 = time.perf_counter()
            o.run(dS)
            w = time.perf_counter() - t0
            o.close()
            rates[k] = spec["n"] ** 2 * dS / w
            detail[k] = {"instance": i, "grid": f"{spec['n']}x{spec['n']}", "timed_steps": dS, "kpoint_steps_per_s": rates[k]}
        return mix_rate(rates, self.units), detail


def cpu_sample(root, budget_s):
    logical, phys = host_cores()
    threads = max(4, logical)  # the reference's Coulomb path needs >= 4 OpenMP threads
    if os.path.exists(REF_EXE):
        s, kind = ReferenceSample(root, threads, budget_s), "reference"
    else:
        s, kind = OracleSample(root, threads, budget_s), "port"
    return s, kind, threads, logical, phys


def cpu_line(s, kind, threads, logical, phys, value, detail):
    what = "oracle/_ref/EDUS.x (the reference compiled from its sources)" if kind == "reference" else "the oracle's C restatement"
    return {"value": value, "unit": METRIC, "cores": threads, "kind": kind,
            "host": {"cpus_available": logical, "physical_cores_lscpu": phys},
            "sample": f"{what} on the median-grid hBN and Wannier instances of the sweep, steps {s.S0}..{s.S0}+dS "
                      f"(all inside the pulse), rates weighted by the sweep's k-point·steps per model",
            "per_model": detail}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    root = tempfile.mkdtemp(prefix="edus_ref_")
    steps = max(1, args.steps)
    budget = max(2.0, min(8.0, 150.0 / (steps + args.warmup)))
    s, kind, threads, logical, phys = cpu_sample(root, budget)
    for _ in range(args.warmup):
        s.measure()
    vals, detail = [], None
    for _ in range(steps):
        v, detail = s.measure()
        vals.append(v)
    v = statistics.mean(vals)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": args.gpus, "steps": steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": SWEEP, "instances": 256, "parallelism": "host threads"},
            "cpu_baseline": cpu_line(s, kind, threads, logical, phys, v, detail),
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ GPU: the continuous sweep

class SweepBatch:
    """The 256 sweep instances live in one batch; finished ones are re-admitted
    from their input files."""

    def __init__(self, root, precision, E, abi, specs):
        self.E, self.abi = E, abi
        self.specs = specs
        self.paths = [write_sweep_instance(root, i, s) for i, s in enumerate(specs)]
        self.b = E.Batch(precision=precision)
        self.live = {}
        self.problems = {}
        self.retired = 0
        for i in range(len(specs)):
            self._admit(i)

    def _admit(self, i):
        E = self.E
        path, d = self.paths[i]
        pb = E.Problem(E.parse_input(path), d, defer_model=self.specs[i]["kind"] == "wannier")
        if self.specs[i]["kind"] == "hbn":
            pb.drop_decoupled_core()
        s = self.b.add(pb)
        pb.close()
        self.live[s] = i

    def step(self, time_steps=STEP_TIME_STEPS, readmit=True):
        self.b.advance(time_steps)
        for s, i in list(self.live.items()):
            if self.b.poll(s)[0] == self.abi.EDUS_INST_DONE:
                self.b.obs(s)
                self.b.release(s)
                del self.live[s]
                self.retired += 1
                if readmit:
                    self._admit(i)

    def close(self):
        self.b.close()


def stratified(specs, kind, count):
    ks = sorted((s["n"], i) for i, s in enumerate(specs) if s["kind"] == kind)
    return [ks[round(j * (len(ks) - 1) / max(1, count - 1))][1] for j in range(count)]


def single_fp64(E, path, d, kind):
    pb = E.Problem(E.parse_input(path), d)
    if kind == "hbn":
        pb.drop_decoupled_core()
    ctx = E.Context(pb)
    ctx.run()
    ms, _ = ctx.last_timing()
    out = (pb.info.nk * pb.info.nsteps, ms * 1e-3, ctx.obs(), ctx.get_state())
    ctx.close()
    pb.close()
    return out


def rel_l2(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def fp64_comparison(E, abi, root, specs, per_kind=6):
    """The plain FP64 single-solve path, request by request, on per_kind
    instances per model spread over the grid sizes; the same instances in one
    mixed batch to completion; errors of the mixed path against FP64."""
    sample = {k: stratified(specs, k, per_kind) for k in ("hbn", "wannier")}
    rates, refs, units_run = {}, {}, 0.0
    for k, idx in sample.items():
        u = t = 0.0
        for i in idx:
            path, d = write_sweep_instance(root, i, specs[i])
            uu, tt, log, rho = single_fp64(E, path, d, k)
            u += uu
            t += tt
            refs[i] = (log, rho)
        rates[k] = u / t
        units_run += u
    b = E.Batch(precision=abi.EDUS_PREC_MIXED)
    slots = {}
    for k, idx in sample.items():
        for i in idx:
            path, d = write_sweep_instance(root, i, specs[i])
            pb = E.Problem(E.parse_input(path), d, defer_model=k == "wannier")
            if k == "hbn":
                pb.drop_decoupled_core()
            slots[i] = b.add(pb)
            pb.close()
    while not all(b.poll(s)[0] == abi.EDUS_INST_DONE for s in slots.values()):
        b.advance(256)
    errs = {}
    for k, idx in sample.items():
        j1, pop, rho = [], [], []
        for i in idx:
            lb, st = b.obs(slots[i]), b.get_state(slots[i])
            log, r = refs[i]
            j1.append(rel_l2([x["J1"] for x in lb], [x["J1"] for x in log]))
            pop.append(float(np.abs(np.array([x["pop"] for x in lb]) - np.array([x["pop"] for x in log])).max()))
            rho.append(float(np.abs(st - r).max()))
        errs[k] = {"instances": idx, "j1_rel_l2_max": max(j1), "j1_rel_l2_median": float(np.median(j1)),
                   "pop_abs_max": max(pop), "rho_abs_max": max(rho)}
    b.close()
    return rates, errs


def roofline_of_batch(b, n_of_kind, tuned):
    """Dominant kernel of a profiled advance (CUDA events around every launch).
    Algorithmic bytes per RK4 stage launch: 16 n^2 per k point (the
    mixed-precision k-point·step moves 64 n^2: FP64 state read + write 32 n^2,
    FP32 H and D_x,y,z 32 n^2; a step is four stage launches)."""
    prof = b.profile(64)
    top = max(prof, key=lambda e: e["total_ms"])
    total = sum(e["total_ms"] for e in prof)
    n = top["nbands"]
    per_ms = top["total_ms"] / top["launches"]
    alg = 16 * n * n * top["kpoints"]
    tile, regs = tuned
    kt = tile.get(n, 0) if tile else 0
    form = regs.get(n, 0) if regs else 0
    if top["kind"] == 0:
        kern = f"k_bobs<{n},1>"
    elif form in (3, 4, 5):
        kern = f"k_bpipe<{n},{kt},{top['kind'] - 1},{form - 3}>"
    else:
        kern = f"k_bstage<{n},{kt}> stage {top['kind'] - 1}"
    achieved = alg / (per_ms * 1e-3) / 1e9
    peak, src = measured_peaks()
    return {"bound": "hbm", "kernel": kern, "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": ncu_traffic(kern, top["kpoints"]), "algorithmic_bytes_per_launch": alg, "launch_ms": per_ms,
            "share": top["total_ms"] / total,
            "peak_source": src,
            "launch_timing": "CUDA-event pair around every launch of 64 eagerly launched sweep time steps on the batch stream",
            "kernels": [{"nbands": e["nbands"], "kind": ["observables", "stage0", "stage1", "stage2", "stage3"][e["kind"]],
                         "launches": e["launches"], "ms": e["total_ms"]} for e in sorted(prof, key=lambda e: -e["total_ms"])]}


def config1_line(E, local, steps):
    """Configuration 1 (FP64 single solve), one full solve per step, L2 flushed between."""
    import torch

    from edus_b200 import workloads as W

    d = tempfile.mkdtemp(prefix="edus_c1_")
    path = W.hbn_coulomb(d)
    p = E.parse_input(path)
    pb = E.Problem(p, d)
    ctx = E.Context(pb, device=local)
    nk, nsteps, n = pb.info.nk, pb.info.nsteps, pb.info.ncv
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    for _ in range(3):
        ctx.reset()
        ctx.run()
    dev = []
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        ctx.reset()
        ctx.run()
        dev.append(ctx.last_timing()[0])
    value = nk * nsteps * steps / (sum(dev) * 1e-3)
    rho0 = pb.get("P0")
    t0 = time.perf_counter()
    for _ in range(steps):
        ctx.reset()
        ctx.set_state(rho0)
        ctx.run()
        ctx.obs()
        ctx.get_state()
    e2e = nk * nsteps * steps / (time.perf_counter() - t0)
    ctx.reset()
    prof = ctx.profile(min(600, nsteps), reps=8)
    per_launch_ms = prof["rhs_ms"] / max(prof["rhs_launches"], 1)
    # rho read + write 32 n^2, H and D_xyz 64 n^2, AB4 history (3 reads + 1 write) 64 n^2
    alg = (32 * n * n + 64 * n * n + 64 * n * n) * nk
    achieved = alg / (per_launch_ms * 1e-3) / 1e9
    peak, src = measured_peaks()
    kern = f"k_rhs_ep<{n},32>"
    ctx.close()
    # AB4 with RK4 start-up: one RHS per step, four in each of the first three steps
    rhs_per_solve = nsteps + 3 * (4 - 1)
    return {"workload": COULOMB, "value": value, "unit": METRIC, "ms_per_solve": sum(dev) / steps, "solves": steps,
            "time_steps_per_solve": nsteps, "nk": nk, "e2e": e2e, "dtype": "f64",
            "rhs_evals_per_s": {"value": value * rhs_per_solve / nsteps, "unit": "k-point RHS evaluations/s"},
            "roofline": {"bound": "hbm", "kernel": kern, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": ncu_traffic(kern), "algorithmic_bytes_per_launch": alg,
                         "launch_ms": per_launch_ms, "peak_source": src,
                         "coulomb_pair_ms": prof["coulomb_ms"] / max(prof["coulomb_launches"], 1)}}


def run_ours(args):
    import torch

    from edus_b200.replicas import ReplicaGroup, whole_job_rate

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    group = ReplicaGroup("nccl", device=f"cuda:{local}")
    import edus_b200 as E
    from edus_b200 import abi

    root = tempfile.mkdtemp(prefix="edus_bench_")
    specs = sweep_specs()
    t_setup = time.perf_counter()
    sw = SweepBatch(root, abi.EDUS_PREC_MIXED, E, abi, specs)
    setup_s = time.perf_counter() - t_setup
    for _ in range(max(args.warmup, 1)):
        sw.step()
    sampler = ClockSampler(local)
    sampler.start()
    group.barrier()
    s0 = sw.b.stats()
    w0 = time.perf_counter()
    r0 = sw.retired
    for _ in range(args.steps):
        sw.step()
    torch.cuda.synchronize()
    wall = time.perf_counter() - w0
    s1 = sw.b.stats()
    group.barrier()
    clocks = sampler.stop()
    units = s1["kpoint_steps"] - s0["kpoint_steps"]
    dev_s = (s1["device_ms"] - s0["device_ms"]) * 1e-3
    max_dev = group.max(dev_s)
    max_wall = group.max(wall)
    value = whole_job_rate(world, units / args.steps, args.steps, max_dev)
    e2e = whole_job_rate(world, units / args.steps, args.steps, max_wall)
    launches = s1["launches"] - s0["launches"]
    h2d = (s1["h2d_bytes"] - s0["h2d_bytes"]) / args.steps
    d2h = (s1["d2h_bytes"] - s0["d2h_bytes"]) / args.steps
    group.close()
    if rank != 0:
        sw.close()
        return 0

    from edus_b200 import autotune

    tuned = autotune.tuned_options(abi.EDUS_PREC_MIXED)
    roof = roofline_of_batch(sw.b, None, tuned)
    live = len(sw.live)
    sw.close()

    # the same sweep in an FP64 batch (batching without the precision change)
    sw64 = SweepBatch(root, abi.EDUS_PREC_FP64, E, abi, specs)
    sw64.step()
    a0 = sw64.b.stats()
    for _ in range(3):
        sw64.step()
    a1 = sw64.b.stats()
    fp64_batch = (a1["kpoint_steps"] - a0["kpoint_steps"]) / ((a1["device_ms"] - a0["device_ms"]) * 1e-3)
    sw64.close()

    rates, errs = fp64_comparison(E, abi, root, specs)
    fp64_single = mix_rate(rates, kind_weights(specs))

    c1 = config1_line(E, local, min(args.steps, 5))

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        try:
            s, kind, threads, logical, phys = cpu_sample(tempfile.mkdtemp(prefix="edus_cpu_"), args.cpu_seconds)
            v, detail = s.measure()
            cpu = cpu_line(s, kind, threads, logical, phys, v, detail)
        except Exception as ex:  # the baseline is reported, not required
            cpu = {"error": str(ex)}

    j1_max = max(e["j1_rel_l2_max"] for e in errs.values())
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": max_dev / args.steps * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "mixed (fp32 H, D, commutator; fp64 state, observables)", "data": "synthetic",
        "config": {"workload": SWEEP, "instances": 256, "live_instances": live,
                   "step": f"every live instance advanced {STEP_TIME_STEPS} RK4 time steps; finished instances retired "
                           "and re-admitted from their input files",
                   "l2": "inputs larger than L2 (the live instances' state and tables are ~10 GB)",
                   "parallelism": f"replicas x{world}", "graph": "chunks of 16 time steps replayed from CUDA graphs",
                   "host_setup_s": setup_s, "retired_in_timed_steps": sw.retired - r0},
        "fp64_single_solve": {"value": fp64_single, "per_model": rates,
                              "how": "plain FP64 single-solve path, request by request, 6 instances per model spread over "
                                     "the grid sizes; per-model rates weighted by the sweep's k-point·steps"},
        "fp64_batch": {"value": fp64_batch, "how": "the same continuous sweep in an FP64 batch, 3 steps"},
        # RK4: four RHS evaluations per k-point·step
        "rhs_evals_per_s": {"value": 4 * value, "unit": "k-point RHS evaluations/s"},
        "speedup_vs_fp64_single": value / fp64_single,
        "speedup_batching_fp64": fp64_batch / fp64_single,
        "speedup_precision_batched": value / fp64_batch,
        "target_3x_at_1e-6": {"speedup": value / fp64_single, "j1_rel_l2_max": j1_max,
                              "met": bool(value / fp64_single >= 3.0 and j1_max <= 1e-6)},
        "errors_vs_fp64": errs,
        "roofline": roof,
        "cpu_baseline": cpu,
        "e2e": {"value": e2e, "unit": METRIC, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "how": "wall time of the timed steps: advance, retirement (D2H of observable logs), re-admission "
                       "(input parse, host set-up, H2D of tables, state and field)"},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "config1_fp64": c1,
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ other workloads

def run_coulomb(args):
    """Configuration 1 as the primary line (FP64 single solve)."""
    import torch

    import edus_b200 as E

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    sampler = ClockSampler(local)
    sampler.start()
    c1 = config1_line(E, local, args.steps)
    clocks = sampler.stop()
    line = {"metric": METRIC, "value": c1["value"], "unit": METRIC, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": c1["ms_per_solve"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": COULOMB, "nk": c1["nk"], "step": "one full solve",
                       "l2": "flushed between timed solves (256 MiB write)"},
            "roofline": c1["roofline"], "e2e": {"value": c1["e2e"], "unit": METRIC}, "clocks": clocks}
    print(json.dumps(line), flush=True)
    return 0


def run_suite(args):
    import torch

    from edus_b200 import suite

    torch.cuda.set_device(0)
    sampler = ClockSampler(0)
    sampler.start()
    if args.workload == "wannier":
        line = suite.wannier_line()
    else:
        line = suite.serve_line(count=args.requests, rate=args.rate)
    line.update({"n_gpus": 1, "clocks": sampler.stop()})
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "coulomb":
        return run_coulomb(args)
    if args.workload in ("wannier", "serve"):
        return run_suite(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
