"""Generate the golden fixtures from the reference's shipped example data.

Run once in a container that has the reference mounted:
    python tests/golden/make_golden.py /root/reference

Writes (all small, committed):
  ab5_input.txt          input.txt of the shipped Adams–Bashforth run
  ab5_golden.npz         its Output/{J1,J2,Losses,EF,TransientAbs}.txt, every
                         4th output row (830 of 3319), at printed precision
  ab5_kgrid.json         its Output/k_grid.txt: SHA-256 of the bytes, line
                         count and the first and last lines
  ab5_test_matrices.txt  its Test_matrices.txt as shipped (byte comparison)
  test_matrices.npz      H, U, dx, dy at k=(0,0.3,0.1) from Test_matrices.txt
  ../../edus_b200/data/coulomb_ncut20.npz
                         Output/Coulomb/{A,B,C,D}_coeff, Screen_const and
                         V_Hartree for G_num=502657, Ncut=20 (3 bands); the
                         Coulomb workload (config 1) reads it, so it ships
                         with the package
"""
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
AB5 = "example/Adams–Bashforth ODE Solver example/AB5_SpectrumNOCOULOMB_Nk_70intens_5000000000.0_t1_-2.3_dt_0.1_delayXUV_0w_Pump__7.00"
CLB = "example/hBN_Coulomb_reading_from_file/Output/Coulomb"
STRIDE = 4


def rows(path):
    out = []
    for line in open(path):
        s = line.split()
        if s:
            out.append([float(x) for x in s])
    return np.array(out)


def parse_cplx(tok):
    m = re.match(r"\(([^,]+),([^)]+)\)", tok)
    return complex(float(m.group(1)), float(m.group(2)))


def test_matrices(path):
    blocks, cur, name = {}, [], None
    for line in open(path):
        line = line.strip()
        if line.endswith(":") or line.startswith("U E_W") or line.startswith("U  U_dagger"):
            if name and cur:
                blocks[name] = np.array(cur)
            name, cur = line.split(":")[0].split(" (")[0].strip(), []
            continue
        toks = [t for t in line.split() if t.startswith("(")]
        if toks and name:
            cur.append([parse_cplx(t) for t in toks])
    if name and cur:
        blocks[name] = np.array(cur)
    return blocks


def kgrid(ref):
    """Fingerprint of the shipped Output/k_grid.txt (byte-exact comparison)."""
    import hashlib
    import json

    with open(os.path.join(ref, AB5, "Output", "k_grid.txt"), "rb") as f:
        raw = f.read()
    lines = raw.decode().splitlines()
    out = {"sha256": hashlib.sha256(raw).hexdigest(), "bytes": len(raw), "lines": len(lines),
           "head": lines[:3], "tail": lines[-3:]}
    with open(os.path.join(HERE, "ab5_kgrid.json"), "w") as f:
        json.dump(out, f, indent=1)


def test_matrices_text(ref):
    with open(os.path.join(ref, AB5, "Test_matrices.txt"), "rb") as f, open(os.path.join(HERE, "ab5_test_matrices.txt"), "wb") as o:
        o.write(f.read())


def main(ref):
    kgrid(ref)
    test_matrices_text(ref)
    g = os.path.join(ref, AB5)
    with open(os.path.join(g, "input.txt")) as f, open(os.path.join(HERE, "ab5_input.txt"), "w") as o:
        o.write(f.read())
    J1 = rows(os.path.join(g, "Output/J1.txt"))
    J2 = rows(os.path.join(g, "Output/J2.txt"))
    Lo = rows(os.path.join(g, "Output/Losses.txt"))
    EF = rows(os.path.join(g, "Output/EF.txt"))
    TA = rows(os.path.join(g, "Output/TransientAbs.txt"))
    n = J1.shape[0]
    sel = np.arange(0, n, STRIDE)
    np.savez_compressed(
        os.path.join(HERE, "ab5_golden.npz"),
        rows=sel, nrows=n, J1=J1[sel], J2=J2[sel], Losses=Lo[sel], EF=EF[sel], TAbs=TA[sel]
    )
    tm = test_matrices(os.path.join(g, "Test_matrices.txt"))
    np.savez_compressed(os.path.join(HERE, "test_matrices.npz"), **{k.replace(" ", "_"): v for k, v in tm.items()})
    c = os.path.join(ref, CLB)
    lab = "G_num502657_Ncut20_"
    coef = {}
    for q in "ABCD":
        a = rows(os.path.join(c, f"{q}_coeff{lab}.txt"))
        coef[q] = a[:, 0::2] + 1j * a[:, 1::2]
    sc = rows(os.path.join(c, f"Screen_const_{lab}.txt"))
    coef["screen"] = sc[:, 0] + 1j * sc[:, 1]
    coef["vhartree"] = rows(os.path.join(c, f"V_Hartree_{lab}.txt"))
    np.savez_compressed(os.path.join(HERE, "..", "..", "edus_b200", "data", "coulomb_ncut20.npz"), label=lab, **coef)
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
