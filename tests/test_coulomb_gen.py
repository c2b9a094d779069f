"""Coulomb coefficient generator (Source_Main/Fourier_Coulomb.cpp:95-500): the
oracle's restatement pinned to the reference's shipped tables, and the GPU
generator against the oracle and against the shipped tables."""
import os
import re
import time

import numpy as np
import pytest

import edus_b200 as E
from oracle_lib import coulomb_generate as oracle_generate

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIPPED = os.path.join(ROOT, "edus_b200", "data", "coulomb_ncut20.npz")

# the Coulomb example of the reference (example/hBN_Coulomb_reading_from_file/input.txt),
# on a small k grid (the tables do not depend on it), without Read_Coulomb_from_files
HBN_COULOMB = """NEWINPUT
tdse{
tightbinding Haldane_CoreBN_Nedge gap=  7.25 t1=  -2.3 t2= 0 phi0= 0.0
dt  0.05 au
t_fin 10 au
}
Coulomb{
qTF 0.01
Ncut NCUT
epsilon_static 1.0
GDIST
labelInput _
Rytova_Keldysh
}
nkPT{
1 12 12
}
laserpump sin2  {
cycles 7
wavelength 206.66666666666666 nm
intensity 500000000000.0 wcm2
polarization 0 1 1
}
observables{
it_resolution 2
Current
}
"""


def _params(tmp_path, ncut=20, gdist=None):
    txt = HBN_COULOMB.replace("NCUT", str(ncut)).replace("GDIST", f"G_distance {gdist}" if gdist else "")
    path = tmp_path / "input.txt"
    path.write_text(txt)
    return E.parse_input(str(path))


def _read_coeffs(cdir, label, ncut, n):
    out = {}
    for q in "ABCD":
        a = np.loadtxt(os.path.join(cdir, f"{q}_coeff{label}.txt"))
        out[q] = (a[:, 0::2] + 1j * a[:, 1::2]).reshape(ncut * ncut, n * n)
    s = np.loadtxt(os.path.join(cdir, f"Screen_const_{label}.txt"))
    out["screen"] = s[:, 0] + 1j * s[:, 1]
    out["VH"] = np.loadtxt(os.path.join(cdir, f"V_Hartree_{label}.txt"))
    return out


def test_oracle_hartree_table_matches_shipped(tmp_path):
    """The oracle's G list (502 657 vectors inside G_distance 400, the value the
    reference's example input carries commented out) and Hartree table (q = 0,
    V = 0 where G0 + G1 < 1e-16) against the shipped V_Hartree_G_num502657_Ncut20_.txt."""
    p = _params(tmp_path, gdist=400)
    o = oracle_generate(p, str(tmp_path), what=1)
    assert o["g_num"] == 502657
    ref = np.load(SHIPPED)["vhartree"]
    assert np.abs(o["VH"] - ref).max() <= 1e-13 * np.abs(ref).max()


@pytest.mark.gpu
def test_generator_matches_oracle_small(tmp_path):
    """GPU generator against the oracle on small grids (41 / 401 Simpson points,
    G_distance 8): every table to 1e-12 of its largest entry."""
    p = _params(tmp_path, ncut=6, gdist=8)
    label, ng = E.coulomb_generate(p, str(tmp_path), n_sum=41, n_sum_screen=401)
    o = oracle_generate(p, str(tmp_path), what=7, n_sum=41, n_sum_screen=401)
    assert ng == o["g_num"] and label == f"G_num{ng}_Ncut6_"
    got = _read_coeffs(str(tmp_path / "Output" / "Coulomb"), label, 6, 3)
    for k in ["A", "B", "C", "D", "screen", "VH"]:
        ref = o[k]
        scale = np.abs(ref).max()
        assert scale > 0, k
        assert np.abs(got[k] - ref).max() <= 1e-12 * scale, k


@pytest.mark.gpu
def test_generator_reproduces_shipped_tables(tmp_path):
    """The full-size generation (4999^2 Simpson points, 502 657 G vectors; 39999^2
    points for the screening constant) against the reference's shipped
    Output/Coulomb/*G_num502657_Ncut20_.txt; a run then reads the tables back."""
    p = _params(tmp_path, gdist=400)
    t0 = time.time()
    label, ng = E.coulomb_generate(p, str(tmp_path))
    dt = time.time() - t0
    assert ng == 502657 and label == "G_num502657_Ncut20_"
    got = _read_coeffs(str(tmp_path / "Output" / "Coulomb"), label, 20, 3)
    ref = np.load(SHIPPED)
    for k, rk in [("A", "A"), ("B", "B"), ("C", "C"), ("D", "D"), ("screen", "screen"), ("VH", "vhartree")]:
        r = ref[rk]
        err = np.abs(got[k] - r).max() / np.abs(r).max()
        print(f"{k}: max |diff| / max |ref| = {err:.3e}")
        assert err < 1e-12, k
    print(f"generation took {dt:.1f} s")
    # the generated tables drive a run as the shipped ones do
    txt = (tmp_path / "input.txt").read_text().replace("labelInput _", f"Read_Coulomb_from_files\nlabelInput {label}")
    (tmp_path / "input.txt").write_text(txt)
    pb = E.Problem(E.parse_input(str(tmp_path / "input.txt")), str(tmp_path))
    assert pb.info.ncv == 3


@pytest.mark.gpu
def test_edus_run_generates_the_tables_it_needs(tmp_path):
    """The drop-in executable on a Coulomb input without Read_Coulomb_from_files:
    it generates Output/Coulomb/* on the device (here with G_distance 3, so the
    reference's full Simpson grids stay cheap), reads them back and runs."""
    import subprocess

    from edus_b200 import build

    _params(tmp_path, ncut=8, gdist=3)
    r = subprocess.run([build.EXE], capture_output=True, text=True, cwd=tmp_path, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    m = re.search(r"Coulomb tables (\S+) \((\d+) G vectors\)", r.stdout)
    assert m and m.group(1) == f"G_num{m.group(2)}_Ncut8_"
    for f in ["A_coeff", "B_coeff", "C_coeff", "D_coeff", "Screen_const_", "V_Hartree_"]:
        assert os.path.exists(tmp_path / "Output" / "Coulomb" / f"{f}{m.group(1)}.txt"), f
    J1 = np.loadtxt(tmp_path / "Output" / "J1.txt")
    assert J1.shape[1] == 7 and np.isfinite(J1).all()


def test_generator_rejects_bad_grids_and_models_without_a_device(tmp_path):
    """Argument errors come back as codes before any device work: Simpson grids
    need an odd number of points, and the generator takes up to 4 bands."""
    from edus_b200 import abi
    from edus_b200 import workloads as W

    p = _params(tmp_path, ncut=4, gdist=3)
    for n_sum, n_scr in [(40, 401), (41, 400), (1, 401)]:
        with pytest.raises(E.EdusError) as ei:
            E.coulomb_generate(p, str(tmp_path), n_sum=n_sum, n_sum_screen=n_scr)
        assert ei.value.code == abi.EDUS_EINVAL
    d = tmp_path / "w8"
    q = E.parse_input(W.wannier(str(d), n=12, t_fin_fs=0.1))
    q.coulomb, q.ncut = 1, 4
    with pytest.raises(E.EdusError) as ei:
        E.coulomb_generate(q, str(d), n_sum=41, n_sum_screen=401)
    assert ei.value.code == abi.EDUS_EUNSUPPORTED
