"""Measurements of the batched and served forms on the configuration workloads.

Each function returns one JSON-ready dict in the bench line format. They run on
one GPU; inputs are synthetic (edus_b200.workloads).

  wannier_line  8-band Wannier model, 96x96, 40 fs, RK4 (one solve): the plain
                FP64 single-solve path against M copies of the same solve (CEP
                varied) run concurrently in the mixed-precision batch.
  sweep_line    seeded 256-instance pulse sweep (half hBN, half 8-band Wannier,
                grids 48^2-144^2, 10-60 fs) in one mixed-precision batch, against
                the plain FP64 single-solve path run request by request on a
                sample of the same instances.
  serve_line    Poisson stream of requests (2, 8 or 16 bands, grids 32^2-192^2,
                10-100 fs) through the served engine (continuous batching),
                against the plain FP64 single-solve path run request by request
                on the first requests of the stream.

The error of the mixed path is the relative L2 norm over t of J1(t) against
the FP64 single-solve path (which matches the reference's CPU output to 1e-12).
"""
import math
import os
import tempfile
import time

import numpy as np

import edus_b200 as E
from edus_b200 import abi
from edus_b200 import workloads as W

METRIC = "k-point·steps/s"


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _J1(log):
    return np.array([x["J1"] for x in log])


class _Dirs:
    def __init__(self):
        self.root = tempfile.mkdtemp(prefix="edus_suite_")
        self.models = {}

    def instance(self, spec, i):
        d = os.path.join(self.root, f"i{i}")
        os.makedirs(d, exist_ok=True)
        if spec["kind"] == "wannier":
            name = spec.get("name", "W8")
            key = (name, spec.get("nw", 8), spec.get("nside", 11))
            if key not in self.models:
                self.models[key] = W.write_wannier_tb(os.path.join(self.root, f"{name}_{key[1]}_{key[2]}_tb.dat"), nw=key[1],
                                                      nside=key[2])
            link = os.path.join(d, f"{name}_tb.dat")
            if not os.path.exists(link):
                os.symlink(self.models[key], link)
        return W.write_instance(d, spec), d


def _single_fp64(path, d, graphs=True):
    """Plain FP64 single-solve path: (k-point steps / s, observable log)."""
    p = E.parse_input(path)
    pb = E.Problem(p, d)
    ctx = E.Context(pb, use_graphs=graphs)
    ctx.run()
    ms, _ = ctx.last_timing()
    log = ctx.obs()
    units = pb.info.nk * pb.info.nsteps
    ctx.close()
    pb.close()
    return units, ms * 1e-3, log


def _batch_run(problems, precision, chunk=16, **kw):
    b = E.Batch(precision=precision, chunk_steps=chunk, **kw)
    slots = [b.add(p) for p in problems]
    while not all(b.poll(s)[0] == abi.EDUS_INST_DONE for s in slots):
        b.advance(chunk * 8)
    st = b.stats()
    logs = [b.obs(s) for s in slots]
    b.close()
    return st, logs


def wannier_line(copies=16, n=96, duration=40.0):
    D = _Dirs()
    spec = dict(kind="wannier", n=n, field=0.4, phase=0.0, duration=duration, it_res=10, dt_fs=0.01)
    path, d = D.instance(spec, 0)
    units, secs, ref_log = _single_fp64(path, d)
    fp64_rate = units / secs
    problems = []
    for c in range(copies):
        pth, dd = D.instance(dict(spec, phase=2 * math.pi * c / copies), c)
        problems.append(E.Problem(E.parse_input(pth), dd, defer_model=True))
    st, logs = _batch_run(problems, abi.EDUS_PREC_MIXED)
    mixed_rate = st["kpoint_steps"] / (st["device_ms"] * 1e-3)
    err = _rel(_J1(logs[0]), _J1(ref_log))
    st64, logs64 = _batch_run(problems[:1], abi.EDUS_PREC_FP64)
    return {
        "metric": METRIC, "value": mixed_rate, "unit": METRIC, "higher_is_better": True, "dtype": "mixed (fp32 commutator, fp64 rho)",
        "data": "synthetic",
        "config": {"workload": f"wannier8_{n}x{n}_rk4_dt0.01fs_{duration:g}fs", "form": f"{copies} concurrent solves, mixed batch"},
        "fp64_single_solve": fp64_rate, "speedup_vs_fp64_single": mixed_rate / fp64_rate,
        "fp64_batch_one_solve": st64["kpoint_steps"] / (st64["device_ms"] * 1e-3),
        "j1_rel_l2_vs_fp64": err,
    }


def sweep_line(count=256, fp64_sample_every=16, err_sample=16):
    D = _Dirs()
    specs = W.sweep(count)
    problems, paths = [], []
    t0 = time.perf_counter()
    for i, s in enumerate(specs):
        pth, d = D.instance(s, i)
        paths.append((pth, d))
        pb = E.Problem(E.parse_input(pth), d, defer_model=(s["kind"] == "wannier"))
        if s["kind"] == "hbn":
            pb.drop_decoupled_core()
        problems.append(pb)
    setup_s = time.perf_counter() - t0
    st, logs = _batch_run(problems, abi.EDUS_PREC_MIXED)
    mixed_rate = st["kpoint_steps"] / (st["device_ms"] * 1e-3)
    for p in problems:
        p.close()
    # plain FP64 single-solve path, request by request, on every fp64_sample_every-th instance
    units = secs = 0.0
    errs = []
    sample = [i for i in range(count) if i % fp64_sample_every in (0, 1)]  # both kinds alternate
    for i in sample:
        u, s, ref = _single_fp64(*paths[i])
        units += u
        secs += s
        if len(errs) < err_sample:
            errs.append(_rel(_J1(logs[i]), _J1(ref)))
    fp64_rate = units / secs
    return {
        "metric": METRIC, "value": mixed_rate, "unit": METRIC, "higher_is_better": True, "dtype": "mixed (fp32 commutator, fp64 rho)",
        "data": "synthetic",
        "config": {"workload": f"pulse_sweep_{count}_hbn+wannier8_48-144_10-60fs", "form": "one batch, chunked graph replay",
                   "kpoint_steps": st["kpoint_steps"], "device_s": st["device_ms"] * 1e-3, "host_setup_s": setup_s},
        "fp64_single_solve_sample": {"value": fp64_rate, "instances": len(sample)},
        "speedup_vs_fp64_single": mixed_rate / fp64_rate,
        "j1_rel_l2_vs_fp64": {"max": max(errs), "median": float(np.median(errs)), "instances": len(errs)},
    }


def serve_requests(count, seed=7, nmin=32, nmax=192, dmin=10.0, dmax=100.0, coulomb_frac=0.5):
    """Request stream of the serving workload. Each request carries the
    Rytova-Keldysh mean field with probability coulomb_frac: those use the hBN
    tight-binding model (the reference's Coulomb path is built for its
    tight-binding models), 3 bands, r0 uniform over the whole angstroms 5..20,
    integrated as configuration 1 (Adams-Bashforth 4 with RK4 start-up, dt
    0.005 fs, output every 0.1 fs); the others draw 2 bands (hBN, core band
    dropped), 8 or 16 (Wannier, 11x11 / 13x13 R), RK4 at dt 0.01 fs. Grid
    N x N, N even in [nmin, nmax]; duration uniform in [dmin, dmax] fs; peak
    field log-uniform 0.05-0.8 V/A; CEP uniform."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(count):
        coul = bool(rng.random() < coulomb_frac)
        nb = 3 if coul else int(rng.choice([2, 8, 16]))
        n = 2 * int(rng.integers(nmin // 2, nmax // 2 + 1))
        spec = dict(n=n, field=float(math.exp(rng.uniform(math.log(0.05), math.log(0.8)))),
                    phase=float(rng.uniform(0, 2 * math.pi)), duration=float(rng.uniform(dmin, dmax)), it_res=10, dt_fs=0.01)
        if coul:
            spec.update(kind="hbn_coulomb", r0=int(rng.integers(5, 21)), dt_fs=0.005, it_res=20)
        elif nb == 2:
            spec["kind"] = "hbn"
        else:
            spec.update(kind="wannier", nw=nb, nside=11 if nb == 8 else 13, name=f"W{nb}")
        out.append(spec)
    return out


def _class(spec):
    return "coulomb" if spec["kind"] == "hbn_coulomb" else str(spec.get("nw", 2))


def _units(spec):
    dt = spec["dt_fs"] / 0.02418884326505
    itfi = int((spec["duration"] + 0.21) / 0.02418884326505 / dt)
    return spec["n"] ** 2 * (itfi + 1)


def serve_line(count=2000, rate=None, per_class=30, seed=7, max_s=None, load=1.25, **kw):
    """Served mixed-precision stream (configuration 4) against the plain FP64
    single-solve path on the same requests.

    Arrivals: Poisson at `rate`, by default `load` x the service capacity
    estimated from measured per-class rates (the autotuner's batch rates of the
    2-, 8- and 16-band classes, and the FP64 context rate of one Coulomb
    request): a saturating stream. Coulomb tables are generated on the GPU
    once per r0 before the stream starts. The FP64 path runs, request by
    request, the first per_class requests of each class in stream order; its
    per-class rates give the FP64 time of the whole stream, and the speed-up is
    that over the served span."""
    from edus_b200 import autotune

    D = _Dirs()
    specs = serve_requests(count, seed=seed, **kw)
    t0 = time.perf_counter()
    tables = {r0: W.coulomb_tables_for(os.path.join(D.root, "coulomb"), r0)
              for r0 in sorted({x["r0"] for x in specs if x["kind"] == "hbn_coulomb"})}
    tables_s = time.perf_counter() - t0

    def write(q):
        sp = specs[q]
        if sp["kind"] != "hbn_coulomb":
            return D.instance(sp, q)
        d = os.path.join(D.root, f"i{q}")
        cdir, label = tables[sp["r0"]]
        return W.hbn_coulomb(d, n=sp["n"], field=sp["field"], duration=sp["duration"], dt_fs=sp["dt_fs"],
                             it_res=sp["it_res"], phase=sp["phase"], r0_ang=sp["r0"], label=label, tables=cdir), d

    paths = [write(q) for q in range(count)]
    reqs = [(E.parse_input(p), d) for p, d in paths]
    units = {}
    for sp in specs:
        units[_class(sp)] = units.get(_class(sp), 0.0) + _units(sp)
    # service capacity from measured per-class rates
    # mixed batches run the 2-band class in FP64 (its k-gradient needs FP64 stage inputs)
    tuned = autotune.load().get(autotune.gpu_name(), {})
    cap_rates = {c: float(tuned.get("fp64" if c == "2" else "mixed", {}).get(c, {}).get("kpoint_steps_per_s", 0))
                 for c in ("2", "8", "16")}
    cap_rates = {c: r for c, r in cap_rates.items() if r > 0}
    qc = next(q for q, sp in enumerate(specs) if sp["kind"] == "hbn_coulomb")
    u, sec, _ = _single_fp64(*paths[qc])
    cap_rates["coulomb"] = u / sec
    capacity = count / sum(units[c] / cap_rates[c] for c in units if c in cap_rates)
    if rate is None:
        rate = load * capacity
    gaps = np.random.Generator(np.random.PCG64(seed + 1)).exponential(1.0 / rate, size=count)
    s = E.Server(precision=abi.EDUS_PREC_MIXED)
    t_start = s.clock()
    ids = []
    for (p, d), g in zip(reqs, gaps):
        target = (s.clock() - t_start) + g
        while s.clock() - t_start < target - 1e-4:
            time.sleep(min(0.01, max(0.0, target - (s.clock() - t_start))))
        ids.append(s.submit(p, d))
    arrival_span = s.clock() - t_start
    s.drain(max_s or 7200)
    st = s.stats()
    sample = []
    for c in sorted(units):
        sample += [q for q in range(count) if _class(specs[q]) == c][:per_class]
    failures = []
    for q, rid in enumerate(ids):
        f = s.failure(rid)
        if f is not None:
            sp = specs[q]
            failures.append({"request": q, "class": _class(sp), "n": sp["n"], "duration_fs": sp["duration"],
                             "field_V_per_A": sp["field"], "r0_A": sp.get("r0"), "error": f[0], "message": f[1]})
    sample = [q for q in sample if s.info(ids[q])["status"] == abi.EDUS_REQ_DONE]
    logs = {q: s.obs(ids[q]) for q in sample}
    s.close()
    # plain FP64 single-solve path, request by request (one request on the GPU at a time)
    cls, errs = {}, {}
    for q in sample:
        u, sec, ref = _single_fp64(*paths[q])
        c = cls.setdefault(_class(specs[q]), [0.0, 0.0, 0])
        c[0] += u
        c[1] += sec
        c[2] += 1
        errs.setdefault(_class(specs[q]), []).append(_rel(_J1(logs[q]), _J1(ref)))
    fp64_stream_s = sum(units[c] / (cls[c][0] / cls[c][1]) for c in units)
    return {
        "metric": "solves/s", "value": st["solves_per_s"], "unit": "solves/s", "higher_is_better": True,
        "dtype": "mixed (fp32 commutator, fp64 rho); Coulomb requests fp64", "data": "synthetic",
        "config": {"workload": f"serving_{count}_requests_nb2-8-16_half_coulomb_r0_5-20A_32-192_10-100fs",
                   "arrival": "Poisson", "arrival_rate_per_s": rate, "capacity_estimate_per_s": capacity,
                   "capacity_rates": cap_rates, "load": rate / capacity, "arrival_span_s": arrival_span,
                   "coulomb_tables": {"r0_values": len(tables), "generation_s": tables_s}},
        "kpoint_steps_per_s": st["kpoint_steps_per_s"], "p50_latency_s": st["p50_latency_s"], "p99_latency_s": st["p99_latency_s"],
        "max_latency_s": st["max_latency_s"], "completed": st["completed"], "failed": st["failed"], "span_s": st["span_s"],
        "device_busy_s": st["device_ms"] * 1e-3,
        "peak_active": st["peak_active"], "peak_bytes": st["peak_bytes"],
        "stream_kpoint_steps_by_class": {k: v for k, v in sorted(units.items())},
        "fp64_request_by_request": {
            "requests": sum(c[2] for c in cls.values()),
            "by_class": {c: {"requests": v[2], "kpoint_steps_per_s": v[0] / v[1]} for c, v in sorted(cls.items())},
            "stream_seconds": fp64_stream_s},
        "speedup_vs_fp64_request_by_request": fp64_stream_s / st["span_s"],
        "j1_rel_l2_vs_fp64": {c: {"max": max(v), "median": float(np.median(v)), "requests": len(v)} for c, v in sorted(errs.items())},
        "failures": failures,
    }
