"""The C ABI library loads, exports every declared entry point and matches the
ctypes struct layouts. No GPU compute here."""
import ctypes as C
import os
import re

import pytest

import edus_b200 as E
from edus_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "edus_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(edus_[a-z0-9_]+)\s*\(", src)))


def test_every_declared_symbol_is_exported():
    L = E.load_library()
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_struct_sizes_match_ctypes():
    L = E.load_library()
    out = (C.c_int64 * 4)()
    assert L.edus_struct_sizes(out) == 0
    assert list(out) == [C.sizeof(abi.Params), C.sizeof(abi.Obs), C.sizeof(abi.ProblemInfo), C.sizeof(abi.Options)]


def test_strerror_covers_codes():
    L = E.load_library()
    for code in range(0, -12, -1):
        s = L.edus_strerror(code).decode()
        assert s and s != "unknown error"
    assert L.edus_abi_version() == 1


def test_no_silent_fallback_without_gpu(workdir):
    """Without a usable CUDA device the context must fail loudly."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from edus_b200 import workloads as W

    p = E.parse_input(W.hbn_rk4(workdir, n=12, t_fin_fs=0.1))
    pb = E.Problem(p, workdir)
    with pytest.raises(E.EdusError) as ei:
        E.Context(pb)
    assert ei.value.code == abi.EDUS_ECUDA


def test_missing_library_raises(monkeypatch, tmp_path):
    from edus_b200 import lib

    monkeypatch.setattr(lib, "_LIB", None)
    monkeypatch.setattr(lib, "library_path", lambda: str(tmp_path / "nope.so"))
    with pytest.raises(E.EdusError):
        lib.load_library()


def test_edus_run_driver_reports_input_errors(tmp_path):
    """The drop-in executable: usage, a missing input and a grammar error end
    with the reference's exit status 1 (usage errors 2) before any GPU work."""
    import subprocess

    from edus_b200 import build

    if not os.path.exists(build.EXE):
        build.build()
    r = subprocess.run([build.EXE, "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and "usage: edus_run" in r.stdout
    r = subprocess.run([build.EXE, "--no-such-flag"], capture_output=True, text=True)
    assert r.returncode == 2
    r = subprocess.run([build.EXE, str(tmp_path / "missing.txt")], capture_output=True, text=True)
    assert r.returncode == 1 and "missing.txt" in r.stderr
    bad = tmp_path / "input.txt"
    bad.write_text("#SYSTEM\nthis is not an input file\n")
    r = subprocess.run([build.EXE, str(bad)], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 1 and "edus_run:" in r.stderr


def test_edus_run_sets_up_a_crystal_input(tmp_path):
    """A Crystal input: the set-up files (kpt.txt, Test_matrices.txt) are
    written before the device run (which needs a GPU: without one the
    executable exits 1 with the CUDA error)."""
    import subprocess

    from edus_b200 import build
    from edus_b200 import workloads as W

    if not os.path.exists(build.EXE):
        build.build()
    W.crystal(str(tmp_path), nb=(1, 1), nkf=7, n=6)
    r = subprocess.run([build.EXE, "input.txt", "."], capture_output=True, text=True, cwd=tmp_path, timeout=120)
    assert r.returncode == 0 or (r.returncode == 1 and "CUDA" in r.stderr), r.stderr
    assert (tmp_path / "kpt.txt").exists() and (tmp_path / "Test_matrices.txt").exists()
