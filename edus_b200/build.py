"""In-tree build of libedus_b200.so (sm_100a) and the edus_run driver.

python -m edus_b200.build        # or edus_b200.build.build()

Compiles every .cu / .cpp under edus_b200/csrc with nvcc for
-gencode arch=compute_100a,code=sm_100a, objects in edus_b200/_build/,
shared library and driver next to this file.
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libedus_b200.so")
EXE = os.path.join(HERE, "edus_run")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-fopenmp,-O3"] + ARCH


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def sources():
    out = []
    for root, _, files in os.walk(CSRC):
        for f in sorted(files):
            if f.endswith((".cu", ".cpp")) and f != "edus_run.cpp":
                out.append(os.path.join(root, f))
    return sorted(out)


def _obj(src):
    rel = os.path.relpath(src, CSRC).replace(os.sep, "_")
    return os.path.join(BUILD, rel + ".o")


def _compile(src, verbose=False):
    obj = _obj(src)
    deps = [src] + [os.path.join(r, f) for r, _, fs in os.walk(CSRC) for f in fs if f.endswith((".hpp", ".cuh", ".h"))]
    deps.append(os.path.join(HERE, "..", "include", "edus_b200.h"))
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(d) for d in deps):
        return obj
    lang = [] if src.endswith(".cu") else ["-x", "cu"] if False else []
    cmd = [nvcc(), "-c", src, "-o", obj] + NVCC_FLAGS + lang
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(verbose=False, jobs=None):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [nvcc(), "-shared", "-o", LIB] + objs + ARCH + ["-Xcompiler", "-fopenmp", "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    drv = os.path.join(CSRC, "edus_run.cpp")
    if os.path.exists(drv) and (not os.path.exists(EXE) or os.path.getmtime(EXE) < max(os.path.getmtime(LIB), os.path.getmtime(drv))):
        cmd = ["g++", "-O2", "-std=c++17", drv, "-o", EXE, "-L" + HERE, "-ledus_b200", "-Wl,-rpath,$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"driver link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
