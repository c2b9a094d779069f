"""Generate the Coulomb tables of an input.txt on the GPU (edus_coulomb_generate).

  python -m edus_b200.coulomb_tables input.txt [workdir] [--device N]
      [--n-sum 4999] [--n-sum-screen 39999] [--g-distance G] [--ncut N]

Writes <workdir>/Output/Coulomb/{A,B,C,D}_coeff<label>.txt, V_Hartree_<label>.txt
and Screen_const_<label>.txt, label = G_num<G>_Ncut<Ncut><labelInput>, as the
reference does when its Coulomb section has no Read_Coulomb_from_files. The grid
sizes default to the reference's; smaller ones (odd) give a quick, coarser fit.
"""
import argparse
import os
import sys
import time

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import edus_b200 as E  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("input")
    ap.add_argument("workdir", nargs="?", default=None)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--n-sum", type=int, default=None)
    ap.add_argument("--n-sum-screen", type=int, default=None)
    ap.add_argument("--g-distance", type=float, default=None, help="override the input's G_distance")
    ap.add_argument("--ncut", type=int, default=None, help="override the input's Ncut")
    a = ap.parse_args()
    p = E.parse_input(a.input)
    if a.g_distance is not None:
        p.G_distance = a.g_distance
    if a.ncut is not None:
        p.ncut = a.ncut
    wd = a.workdir or os.path.dirname(os.path.abspath(a.input))
    t0 = time.time()
    label, ng = E.coulomb_generate(p, wd, device=a.device, n_sum=a.n_sum, n_sum_screen=a.n_sum_screen)
    print(f"{label}: {ng} G vectors, {time.time() - t0:.1f} s, tables in {os.path.join(wd, 'Output', 'Coulomb')}")


if __name__ == "__main__":
    main()
