"""Run a workload for a fixed number of time steps (for ncu / timing).

Single solve (edus_create / edus_step):
  python -m edus_b200.profile_run --workload hbn_coulomb --steps 60 [--graph] [--n 120]
    hbn_rk4 (hBN RK4 60x60), hbn_coulomb (hBN + Coulomb AB4 120x120), wannier8
    (8-band Wannier RK4 96x96), wannier8_vg (the same in the velocity gauge;
    --precision mixed contracts every stage on the tensor cores). Eager
    launches by default so that ncu sees each kernel; --graph replays the
    captured CUDA graph of the whole loop instead.

Batch (edus_batch_*):
  python -m edus_b200.profile_run --batch wannier8 --instances 2 --precision fp64 \\
      --kt 8 --profile 0 --steps 32 [--eager] [--n 96]
    hbn2 (hBN, core band dropped), hbn3, wannier8, wannier16 instances of an
    n x n grid with the CEP varied; prints k-point steps / s of the timed steps.
"""
import argparse
import os
import sys
import tempfile

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import edus_b200 as E  # noqa: E402
from edus_b200 import abi  # noqa: E402
from edus_b200 import workloads as W  # noqa: E402


def make(name, workdir, n=None):
    if name == "hbn_rk4":
        return W.hbn_rk4(workdir, n=n or 60)
    if name == "hbn_coulomb":
        return W.hbn_coulomb(workdir, n=n or 120)
    if name == "wannier8":
        return W.wannier(workdir, n=n or 96)
    if name == "wannier8_vg":
        path = W.wannier(workdir, n=n or 96)
        with open(path) as f:
            txt = f.read().replace("Wannier\n", "Wannier\nvelocity_gauge\n")
        with open(path, "w") as f:
            f.write(txt)
        return path
    raise SystemExit(f"unknown workload {name}")


def batch_problems(kind, count, n, root):
    out = []
    nw = 16 if kind == "wannier16" else 8
    model = None
    if kind.startswith("wannier"):
        model = W.write_wannier_tb(os.path.join(root, f"W{nw}_tb.dat"), nw=nw, nside=13 if nw == 16 else 11)
    for i in range(count):
        d = os.path.join(root, f"i{i}")
        os.makedirs(d, exist_ok=True)
        if model:
            os.symlink(model, os.path.join(d, f"W{nw}_tb.dat"))
            p = E.parse_input(W.wannier(d, nw=nw, nside=13 if nw == 16 else 11, n=n, t_fin_fs=40.0, name=f"W{nw}",
                                        phase=0.1 * i, write_model=False))
            out.append(E.Problem(p, d, defer_model=True))
        else:
            pb = E.Problem(E.parse_input(W.hbn_rk4(d, n=n, t_fin_fs=40.0, it_res=10, phase=0.1 * i)), d)
            if kind == "hbn2":
                pb.drop_decoupled_core()
            out.append(pb)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="hbn_coulomb")
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--n", type=int, default=None)
    ap.add_argument("--graph", action="store_true")
    ap.add_argument("--batch", default=None, help="hbn2 | hbn3 | wannier8 | wannier16")
    ap.add_argument("--instances", type=int, default=2)
    ap.add_argument("--precision", default="fp64")
    ap.add_argument("--kt", type=int, default=0)
    ap.add_argument("--profile", type=int, default=0)
    ap.add_argument("--eager", action="store_true")
    a = ap.parse_args()
    d = tempfile.mkdtemp(prefix="edus_prof_")
    if a.batch:
        pbs = batch_problems(a.batch, a.instances, a.n or 96, d)
        nb = pbs[0].info.ncv
        prec = abi.EDUS_PREC_MIXED if a.precision == "mixed" else abi.EDUS_PREC_FP64
        b = E.Batch(precision=prec, tile_k={nb: a.kt} if a.kt else None, regs_profile={nb: a.profile},
                    use_graphs=not a.eager, chunk_steps=16)
        for p in pbs:
            b.add(p)
        b.advance(32)
        s0 = b.stats()
        b.advance(a.steps)
        s1 = b.stats()
        rate = (s1["kpoint_steps"] - s0["kpoint_steps"]) / ((s1["device_ms"] - s0["device_ms"]) * 1e-3)
        print(f"{a.batch} x{a.instances} {a.precision} kt={b.tile_k(nb)} profile={a.profile}: {rate:.3e} k-point steps/s, "
              f"{(s1['device_ms'] - s0['device_ms']) / a.steps * 1e3:.1f} us per step")
        return
    p = E.parse_input(make(a.workload, d, a.n))
    prec = abi.EDUS_PREC_MIXED if a.precision == "mixed" else abi.EDUS_PREC_FP64
    ctx = E.Context(E.Problem(p, d), use_graphs=a.graph, precision=prec)
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
