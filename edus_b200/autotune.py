"""Autotuner of the batch engine's tile and launch shapes.

For each band count and precision it times every built stage-kernel variant
(tile length in k points x register profile / kernel form) on a synthetic
batch of the model that uses that band count, keeps the fastest, and caches
the result per GPU name in a JSON file (default edus_b200/tuned.json, or the
path in EDUS_TUNE_CACHE). Batch and Server take the tuned shapes through
tuned_options().

  python -m edus_b200.autotune [--bands 2 8 16] [--precision fp64 mixed]
"""
import argparse
import json
import os
import tempfile
import time

import edus_b200 as E
from edus_b200 import abi
from edus_b200 import workloads as W

# built variants per band count: (tile length, register profile); profile 2
# is the matrix-product form (FP64), profiles 3-5 the staged forms (mixed; 4
# and 5 with the register-blocked commutator, 2 x 2 and 2 x 1 blocks)
VARIANTS = {
    2: [(16, 0), (16, 1), (32, 0), (32, 1), (32, 3)],
    3: [(16, 0), (16, 1), (32, 0), (32, 1), (32, 3)],
    4: [(16, 0), (16, 1), (16, 3)],
    5: [(16, 0), (16, 1), (16, 3)],
    8: [(4, 0), (8, 0), (8, 1), (8, 2), (16, 2), (8, 3), (8, 4), (16, 4), (8, 5), (16, 5)],
    16: [(2, 0), (2, 1), (2, 2), (4, 2), (8, 2), (2, 3), (2, 4), (4, 4), (2, 5), (4, 5)],
}
PREC = {"fp64": abi.EDUS_PREC_FP64, "mixed": abi.EDUS_PREC_MIXED}


def cache_path():
    return os.environ.get("EDUS_TUNE_CACHE", os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuned.json"))


def gpu_name():
    try:
        import torch

        return torch.cuda.get_device_name(0)
    except Exception:
        return "unknown"


def load():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


# band counts below this run in FP64 inside mixed-precision batches (their
# k-gradient needs FP64 stage inputs), so they take the FP64 kernels' tuning
MIXED_MIN_BANDS = 4


def tuned_options(precision):
    """(tile_k, regs_profile) dicts for Batch / Server from the cache (empty if untuned)."""
    cache = load().get(gpu_name(), {})
    entry = dict(cache.get("fp64" if precision == abi.EDUS_PREC_FP64 else "mixed", {}))
    if precision != abi.EDUS_PREC_FP64:
        for n, v in cache.get("fp64", {}).items():
            if int(n) < MIXED_MIN_BANDS:
                entry[n] = v
    tile = {int(n): v["tile_k"] for n, v in entry.items()}
    prof = {int(n): v["regs_profile"] for n, v in entry.items()}
    return tile, prof


def _problems(nbands, count, grid, root):
    out = []
    if nbands in (2, 3):
        for i in range(count):
            d = os.path.join(root, f"h{nbands}_{i}")
            pb = E.Problem(E.parse_input(W.hbn_rk4(d, n=grid, t_fin_fs=40.0, it_res=10, phase=0.3 * i)), d)
            if nbands == 2:
                pb.drop_decoupled_core()
            out.append(pb)
    else:
        nside = 13 if nbands == 16 else 11
        model = W.write_wannier_tb(os.path.join(root, f"W{nbands}_tb.dat"), nw=nbands, nside=nside)
        for i in range(count):
            d = os.path.join(root, f"w{nbands}_{i}")
            os.makedirs(d, exist_ok=True)
            link = os.path.join(d, f"W{nbands}_tb.dat")
            if not os.path.exists(link):
                os.symlink(model, link)
            p = E.parse_input(W.wannier(d, nw=nbands, nside=nside, n=grid, t_fin_fs=40.0, it_res=10, name=f"W{nbands}",
                                        phase=0.3 * i, write_model=False))
            out.append(E.Problem(p, d, defer_model=True))
    return out


def time_variant(problems, precision, nbands, kt, prof, steps):
    b = E.Batch(precision=precision, tile_k={nbands: kt}, regs_profile={nbands: prof}, chunk_steps=16)
    for p in problems:
        b.add(p)
    b.advance(32)
    s0 = b.stats()
    b.advance(steps)
    s1 = b.stats()
    b.close()
    return (s1["kpoint_steps"] - s0["kpoint_steps"]) / ((s1["device_ms"] - s0["device_ms"]) * 1e-3)


def tune(bands=(2, 3, 8, 16), precisions=("fp64", "mixed"), grid=96, steps=96, verbose=True):
    root = tempfile.mkdtemp(prefix="edus_tune_")
    db = load()
    entry = db.setdefault(gpu_name(), {})
    for nb in bands:
        count = {2: 64, 3: 32, 8: 32, 16: 8}.get(nb, 16)
        problems = _problems(nb, count, grid if nb != 16 else 64, root)
        for pn in precisions:
            best = None
            for kt, prof in VARIANTS[nb]:
                if prof == 2 and pn == "mixed":
                    continue  # the matrix-product form is built for FP64 only
                if prof >= 3 and pn == "fp64":
                    continue  # the staged forms are built for mixed precision only
                if nb == 3 and pn == "mixed":
                    continue  # mixed instances carry no core band: 3-band hBN runs as 2 bands
                t0 = time.perf_counter()
                rate = time_variant(problems, PREC[pn], nb, kt, prof, steps)
                if verbose:
                    print(f"{nb:2d} bands {pn:5s} kt={kt:2d} profile={prof}: {rate:.3e} k-point steps/s "
                          f"({time.perf_counter() - t0:.1f} s)", flush=True)
                if best is None or rate > best[0]:
                    best = (rate, kt, prof)
            if best is None:
                continue
            entry.setdefault(pn, {})[str(nb)] = {"tile_k": best[1], "regs_profile": best[2], "kpoint_steps_per_s": best[0],
                                                 "instances": count}
        for p in problems:
            p.close()
    with open(cache_path(), "w") as f:
        json.dump(db, f, indent=1, sort_keys=True)
    return entry


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--bands", type=int, nargs="*", default=[2, 3, 8, 16])
    ap.add_argument("--precision", nargs="*", default=["fp64", "mixed"])
    a = ap.parse_args()
    print(json.dumps(tune(a.bands, a.precision), indent=1))


if __name__ == "__main__":
    main()
