"""Known answers from the reference program itself (anpicon/EDUS), for the parity tests.

Runs oracle/_ref/EDUS.x — the reference's own main_MPI.cpp compiled from its
sources by `make -C oracle ref` (one MPI rank, the Armadillo subset from
oracle/ref_shim/) — on the inputs below and stores, per case, the input text
and the reference's Output/*.txt time series in tests/golden/ref_<case>.npz.
The inputs are written by edus_b200.workloads (seeded; nothing is read from
the reference's examples except the packaged Coulomb tables); the Wannier
model file's SHA-256 is stored so a test can check it regenerates the same
model. Run here, where the reference sources are:

    python tests/golden/make_ref_fixtures.py [case ...]

Cases: the three single-solve configurations at their own sizes (hBN 60x60
RK4 30 fs; hBN 120x120 with the Rytova-Keldysh mean field, AB4 from the
reference's zero derivative history, 30 fs; the 8-band Wannier model 96x96
RK4 40 fs) and small cases of every other solver / option on the path
(Coulomb AB4, diagonal-basis Coulomb, Taylor-6 and RK4 with adaptive dt, the
8- and 16-band Wannier models, per-k snapshot files, the Crystal interface on
seeded synthetic data files, rectangular n1 x n2 grids, Gaussian and
pseudo plane-wave pump envelopes and two pumps, T1 / T2 decoherence, the
reference's other tight-binding models, Adams-Bashforth 1 and 3, Taylor-4 at
constant dt).

Runs with the Coulomb mean field are repeated at several OpenMP thread
counts and every distinct outcome is kept (series keys "J1", "J1#1", ...):
the reference switches its screening correction on when the mean conduction
population n_cond exceeds 1e-20 (headers/RungeKutta.h:77), and before the
pulse n_cond is rounding noise of either sign, so the reference itself gives
one of two results from run to run (their J1 differ by ~3e-8 relative).

    python tests/golden/make_ref_fixtures.py --add [--threads 4,6] CASE   # more runs, merged
"""
import hashlib
import os
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from edus_b200 import workloads as W  # noqa: E402

REF_EXE = os.path.join(ROOT, "oracle", "_ref", "EDUS.x")
SERIES = ("J1", "J2", "Losses", "EF")


def _with(path, old, new):
    txt = open(path).read()
    assert old in txt, old
    open(path, "w").write(txt.replace(old, new, 1))
    return path


def _diag_basis(d):
    return _with(W.hbn_coulomb(d, n=24, t_fin_fs=2.0, it_res=5, rk4_startup=False), "Rytova_Keldysh\n",
                 "Rytova_Keldysh\nCoulomb_diag_basis\n")


def _snapshots(d):
    return _with(W.hbn_rk4(d, n=12, t_fin_fs=1.5, it_res=10), "Current\n", "Current\nPrintPopulation 0 60 15\n")


def _edia(d):
    return _with(W.hbn_coulomb(d, n=24, t_fin_fs=0.3, it_res=10, rk4_startup=False), "Rytova_Keldysh\n",
                 "Rytova_Keldysh\nPrint_new_band_dispersion\n")


def _rect(path, n, n1, n2):
    """The written input with an n1 x n2 grid in place of the n x n one."""
    return _with(path, f"nkpt{{\n1 {n} {n}\n}}", f"nkpt{{\n1 {n1} {n2}\n}}")


def _pump_block(path):
    txt = open(path).read()
    i = txt.index("laserpump sin2 {")
    return txt, i, txt.index("}\n", i) + 2


def _gauss(d):
    """Gaussian pump envelope: sigma 1.5 fs, centred 4 sigma after its t0."""
    path = W.hbn_rk4(d, n=24, t_fin_fs=8.0, it_res=10, field=0.4)
    txt, a, b = _pump_block(path)
    block = ("laserpump gaussian {\nfrequency 0.0146997236011\nintensity 2.12386780644e+12 wcm2\nsigma 1.5 fs\n"
             "polarization 0 0 1\nphase 0.4\n}\n")
    open(path, "w").write(txt[:a] + block + txt[b:])
    return path


def _pw(d):
    """Pseudo plane-wave pump: linear ramp to 2 fs, flat to 5 fs, ramp down to the end of its cycles."""
    path = W.hbn_rk4(d, n=24, t_fin_fs=8.0, it_res=10, field=0.3)
    txt, a, b = _pump_block(path)
    block = ("laserpump pw {\nfrequency 0.0146997236011\nintensity 1.19467564112e+12 wcm2\ncycles 0.67\n"
             "window 2 5 fs\npolarization 0 0 1\nphase 0\n}\n")
    open(path, "w").write(txt[:a] + block + txt[b:])
    return path


def _two_pumps(d):
    """Two sin2 pumps (num_pump_pulses 2): the second polarised across the first and started at 1.5 fs."""
    path = W.hbn_rk4(d, n=24, t_fin_fs=4.0, it_res=5, field=0.3, duration=4.0, extra_tdse="num_pump_pulses 2\n")
    txt, a, b = _pump_block(path)
    second = ("laserpump sin2 {\nfrequency 0.0183746545014\nintensity 5.30966951611e+11 wcm2\ncycles 1.5\n"
              "polarization 0 1 0\nphase 1.1\nt0_pulse 1.5 fs\n}\n")
    open(path, "w").write(txt[:b] + second + txt[b:])
    return path


def _decoherence(d):
    """Population (diagonal) and coherence (off-diagonal) relaxation."""
    path = W.hbn_rk4(d, n=24, t_fin_fs=3.0, it_res=5, field=0.4)
    with open(path, "a") as f:
        f.write("\ndecoherence{\ndiagonal 0.002 au\noffdiagonal 0.01 au\n}\n")
    return path


def _tb_model(model, n=20):
    """The hBN RK4 input with another tight-binding model of the reference in its tdse section, the
    pump polarised along y + z (some models' dipoles have no z component)."""
    def writer(d):
        path = W.hbn_rk4(d, n=n, t_fin_fs=1.5, it_res=5, field=0.4)
        _with(path, "polarization 0 0 1\n", "polarization 0 1 1\n")
        return _with(path, "tightbinding Haldane_CoreBN_Nedge gap= 5.8 t1= 2.3 t2= 0 phi0= 0\n", f"tightbinding {model}\n")
    return writer


# the reference's other tight-binding models (headers/TightBinding.h); grids of 20 points avoid the
# K points, where the gapless graphene models' degenerate eigenvectors are arbitrary. BN1b (one band)
# is left out: the reference program ends with a segmentation fault on it after opening its outputs.
TB_MODELS = {
    "tb_corebn_nedge": "CoreBN_Nedge", "tb_corebn_bedge": "CoreBN_Bedge",
    "tb_haldane_bedge": "Haldane_CoreBN_Bedge gap= 5.8 t1= 2.3 t2= 0.2 phi0= 0.7",
    "tb_gen2d_hexagonal": "gen2d_hexagonal a= 2.5 gap= 5.0 t1= 2.1 t2= 0.15 phi0= 0.4 core= -12 chv_dipole= 0.2 chc_dipole= 0.1",
    "tb_boronnitride": "BoronNitride", "tb_graphene": "Graphene", "tb_coregraphene": "CoreGraphene",
    "tb_graphene_costd": "Graphene_costD", "tb_graphene_symmetricd": "Graphene_symmetricD",
    "tb_graphenezurron": "GrapheneZurron", "tb_dlgraphene": "DLGraphene", "tb_vampa2015": "Vampa2015", "tb_ges": "GeS",
    "tb_ges_hse06": "GeS_HSE06",
}


# name -> (input writer, per-k files to keep)
CASES = {
    "cfg0_hbn60_rk4": (lambda d: W.hbn_rk4(d, n=60, it_res=10), ()),
    "cfg1_hbn120_coulomb_ab4": (lambda d: W.hbn_coulomb(d, n=120, it_res=10, rk4_startup=False), ()),
    "cfg2_wannier8_96_rk4": (lambda d: W.wannier(d, n=96, it_res=10), ()),
    "hbn24_rk4": (lambda d: W.hbn_rk4(d, n=24, t_fin_fs=3.0, it_res=5), ()),
    "hbn24_coulomb_ab4": (lambda d: W.hbn_coulomb(d, n=24, t_fin_fs=2.0, it_res=5, rk4_startup=False), ()),
    "hbn24_coulomb_diag_ab4": (_diag_basis, ()),
    "hbn24_ab2": (lambda d: W.hbn_rk4(d, n=24, t_fin_fs=2.0, it_res=5, solver="Adams_Bashforth 2\n"), ()),
    "hbn24_taylor6_dyn": (lambda d: W.hbn_rk4(d, n=24, t_fin_fs=2.0, it_res=3, dt_fs=0.002,
                                              solver="Taylor\nTaylorOrder 6\ndynamical_dt_evolution\nepsStepAbs 0.02\n"),
                          ()),
    "hbn24_rk4_dyn": (lambda d: W.hbn_rk4(d, n=24, t_fin_fs=2.0, it_res=3,
                                          solver="dynamical_dt_evolution\nepsStepAbs 0.001\n"), ()),
    "wannier8_16_rk4": (lambda d: W.wannier(d, n=16, t_fin_fs=1.0, it_res=5), ()),
    "wannier16_24_rk4": (lambda d: W.wannier(d, nw=16, nside=13, name="W16", n=24, t_fin_fs=1.0, it_res=5), ()),
    "hbn12_snapshots": (_snapshots, ("t_Ek", "P_val_cond_in_Eigenstate_12_", "P_val_in_Eigenstate_11_",
                                     "P_cond_in_Eigenstate_22_", "H_Eigen_", "H_Wannier_cond_", "P_initial_Wannier_",
                                     "Uk_")),
    "hbn24_coulomb_edia": (_edia, ("Edia_", "t_Ek")),
    "crystal12_2band": (lambda d: W.crystal(d, nb=(1, 1), nkf=9, n=12, field=2.0, duration=4.0, t_fin_fs=1.0, it_res=5),
                        ()),
    "crystal10_3band": (lambda d: W.crystal(d, nb=(1, 2), norb=3, nkf=11, n=10, field=1.5, duration=4.0, t_fin_fs=1.0,
                                            it_res=5), ()),
    # rectangular grids (n1 != n2): the stencil shells and the Coulomb row / column passes differ per axis
    "hbn18x24_rk4": (lambda d: _rect(W.hbn_rk4(d, n=18, t_fin_fs=2.0, it_res=5), 18, 18, 24), ()),
    "hbn18x24_coulomb_ab4": (lambda d: _rect(W.hbn_coulomb(d, n=18, t_fin_fs=1.5, it_res=5, rk4_startup=False), 18, 18, 24),
                             ()),
    "wannier8_12x20_rk4": (lambda d: _rect(W.wannier(d, n=12, t_fin_fs=1.0, it_res=5), 12, 12, 20), ()),
    # the other pump envelopes and a second pump (headers/Laser.h:56-76,128-144, headers/ReadInput.h:236-326)
    "hbn24_gauss_rk4": (_gauss, ()),
    "hbn24_pw_rk4": (_pw, ()),
    "hbn24_two_pumps_rk4": (_two_pumps, ()),
    # the Coulomb mean field with RK4
    "hbn24_coulomb_rk4": (lambda d: W.hbn_coulomb(d, n=24, t_fin_fs=1.5, it_res=5, rk4=True), ()),
    # the other Adams-Bashforth orders and Taylor at constant dt
    "hbn24_ab1": (lambda d: W.hbn_rk4(d, n=24, t_fin_fs=1.5, it_res=5, solver="Adams_Bashforth 1\n", dt_fs=0.002), ()),
    "hbn24_ab3": (lambda d: W.hbn_rk4(d, n=24, t_fin_fs=2.0, it_res=5, solver="Adams_Bashforth 3\n"), ()),
    "hbn24_taylor4": (lambda d: W.hbn_rk4(d, n=24, t_fin_fs=2.0, it_res=5, dt_fs=0.005, solver="Taylor\nTaylorOrder 4\n"), ()),
    # dissipation with T1 / T2 (headers/InitParameters.h:203-224, headers/RungeKutta.h:219-254)
    "hbn24_decoherence_rk4": (_decoherence, ()),
}
CASES.update({name: (_tb_model(model), ()) for name, model in TB_MODELS.items()})


def _model_hash(d):
    out = {}
    for f in sorted(os.listdir(d)):
        if f.endswith("_tb.dat") or f in ("kmesh_data.dat", "hk_orthonormal.dat", "bc_betabetap_real.dat",
                                           "bc_betabetap_imag.dat"):
            out[f] = hashlib.sha256(open(os.path.join(d, f), "rb").read()).hexdigest()
    return out


def _run_once(name, threads):
    writer, keep = CASES[name]
    d = tempfile.mkdtemp(prefix=f"edus_ref_{name}_")
    path = writer(d)
    os.makedirs(os.path.join(d, "Output"), exist_ok=True)
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    t0 = time.perf_counter()
    r = subprocess.run([REF_EXE, os.path.basename(path)], cwd=d, env=env, capture_output=True, text=True)
    wall = time.perf_counter() - t0
    if r.returncode != 0:
        raise RuntimeError(f"{name}: reference exited {r.returncode}\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}")
    out = {"input": np.array(open(path).read()), "threads": np.array(threads), "wall_s": np.array(wall)}
    for s in SERIES:
        out[s] = np.loadtxt(os.path.join(d, "Output", f"{s}.txt"), ndmin=2)
    for f, h in _model_hash(d).items():
        out[f"sha256:{f}"] = np.array(h)
    files = sorted(os.listdir(os.path.join(d, "Output")))
    for prefix in keep:
        for f in files:
            if f.startswith(prefix) and f.endswith(".txt"):
                out[f"file:{f}"] = np.array(open(os.path.join(d, "Output", f)).read())
    shutil.rmtree(d, ignore_errors=True)
    return out


def _j1(a):
    return a[:, 1::2] + 1j * a[:, 2::2]


def _distinct(variants, J1):
    for v in variants:
        if np.linalg.norm(_j1(v) - _j1(J1)) <= 1e-10 * np.linalg.norm(_j1(v)):
            return False
    return True


def run_case(name, thread_counts, add=False):
    """Run the reference once per thread count; keep the first run's series
    under the plain keys and each further distinct outcome under "<key>#<i>"."""
    path = os.path.join(HERE, f"ref_{name}.npz")
    out = dict(np.load(path)) if add and os.path.exists(path) else {}
    if out and "runs" not in out:
        out["runs"] = np.array([int(out["threads"])])
    walls = []
    for th in thread_counts:
        r = _run_once(name, th)
        walls.append(r["wall_s"])
        if not out:
            out = r
            out["runs"] = np.array([th])
            continue
        assert str(r["input"]) == str(out["input"])
        out["runs"] = np.append(out["runs"], th)
        nvar = 1 + sum(1 for k in out if k.startswith("J1#"))
        variants = [out["J1"]] + [out[f"J1#{i}"] for i in range(1, nvar)]
        if _distinct(variants, r["J1"]):
            for sname in SERIES:
                out[f"{sname}#{nvar}"] = r[sname]
    np.savez_compressed(path, **out)
    return sum(float(w) for w in walls)


def main(argv):
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    add = "--add" in argv
    given = None
    if "--threads" in argv:
        i = argv.index("--threads")
        given = [int(x) for x in argv[i + 1].split(",")]
        argv = argv[:i] + argv[i + 2:]
    names = [a for a in argv if not a.startswith("--")] or list(CASES)
    # the reference's Coulomb path indexes id_masters[thr_total-4] (headers/Coulomb.h:307-310): >= 4 threads
    threads = max(4, os.cpu_count() or 4)
    for name in names:
        if given:
            counts = given
        elif "coulomb" in name:
            counts = [threads, 4, threads, 4, 6, 5] if not name.startswith("cfg") else [threads, 4]
        else:
            counts = [threads]
        wall = run_case(name, counts, add=add)
        print(f"{name}: {wall:.1f} s over runs on {counts} threads", flush=True)


if __name__ == "__main__":
    main(sys.argv[1:])
