"""Run a workload for a fixed number of time steps (for ncu / timing).

python -m edus_b200.profile_run --workload cfg1 --steps 60 [--graph] [--n 120]

Workloads: cfg0 (hBN RK4 60x60), cfg1 (hBN + Coulomb AB4 120x120), cfg2
(8-band Wannier RK4 96x96). Eager launches by default so that ncu sees each
kernel; --graph replays the captured CUDA graph of the whole loop instead.
"""
import argparse
import os
import sys
import tempfile

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import edus_b200 as E  # noqa: E402
from edus_b200 import workloads as W  # noqa: E402


def make(name, workdir, n=None):
    if name == "cfg0":
        return W.hbn_rk4(workdir, n=n or 60)
    if name == "cfg1":
        return W.hbn_coulomb(workdir, n=n or 120)
    if name == "cfg2":
        return W.wannier(workdir, n=n or 96)
    raise SystemExit(f"unknown workload {name}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="cfg1")
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--n", type=int, default=None)
    ap.add_argument("--graph", action="store_true")
    a = ap.parse_args()
    d = tempfile.mkdtemp(prefix="edus_prof_")
    p = E.parse_input(make(a.workload, d, a.n))
    ctx = E.Context(E.Problem(p, d), use_graphs=a.graph)
    if a.graph:
        ctx.run()
        ctx.reset()
        ctx.run()
        steps = ctx.problem.info.nsteps
    else:
        ctx.step(a.steps)
        steps = a.steps
    ms, launches = ctx.last_timing()
    print(f"{a.workload}: {steps} steps, {ms:.3f} ms, {launches} launches, {ms * 1e3 / steps:.2f} us/step")


if __name__ == "__main__":
    main()
