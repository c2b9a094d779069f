"""Synthetic workloads in the reference's input.txt format.

Each function writes an input.txt (and any model / Coulomb files it needs)
into a work directory and returns the path of the input file. Fields are
converted with the reference's own constants: E0 [a.u.] = E [V/A] * 1e10 /
5.14221e11 and I [W/cm^2] = E0^2 * 3.51e16 (headers/Laser.h:29-31).

  hbn_rk4        config 0: Haldane_CoreBN_Nedge (core band decoupled), RK4, no Coulomb
  hbn_coulomb    config 1: same model with the Rytova–Keldysh mean field from the
                 shipped Ncut=20 coefficient files, Adams–Bashforth 4
  wannier        config 2: synthetic nb-band Wannier model (seeded), RK4
  sweep          config 3: seeded pulse sweep mixing both models on uneven grids
"""
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TIME_FS_AU = 1.0 / 0.02418884326505
EV_AU = 1.0 / 27.211396
EFIELD_AU_PER_V_A = 1e10 / 5.14221e11
COULOMB_LABEL = "G_num502657_Ncut20_"
ANG_AU = 1.0 / 0.52917721092  # bohr per angstrom with the reference's space_au_A (headers/Constants.h:31)


def intensity_wcm2(e_v_per_a):
    e0 = e_v_per_a * EFIELD_AU_PER_V_A
    return e0 * e0 * 3.51e16


def _pump(photon_ev, field_v_a, duration_fs, pol="0 0 1", phase=0.0):
    wl = photon_ev * EV_AU
    period_fs = 2 * math.pi / wl / TIME_FS_AU
    cycles = duration_fs / period_fs
    return (
        "laserpump sin2 {\n"
        f"frequency {wl:.12g}\n"
        f"intensity {intensity_wcm2(field_v_a):.12g} wcm2\n"
        f"cycles {cycles:.12g}\n"
        f"polarization {pol}\n"
        f"phase {phase:.12g}\n"
        "}\n"
    )


def write_coulomb_files(workdir, label=COULOMB_LABEL):
    """Output/Coulomb/* in the reference's text format from the packaged data."""
    d = np.load(os.path.join(HERE, "data", "coulomb_ncut20.npz"))
    cdir = os.path.join(workdir, "Output", "Coulomb")
    os.makedirs(cdir, exist_ok=True)
    for q in "ABCD":
        a = d[q]
        with open(os.path.join(cdir, f"{q}_coeff{label}.txt"), "w") as f:
            for row in a:
                f.write("".join(f"{v.real:.20e}    {v.imag:.20e}    " for v in row) + "\n")
    with open(os.path.join(cdir, f"Screen_const_{label}.txt"), "w") as f:
        for v in d["screen"]:
            f.write(f"{v.real:.20g} {v.imag:.20g}\n")
    with open(os.path.join(cdir, f"V_Hartree_{label}.txt"), "w") as f:
        for row in d["vhartree"]:
            f.write("".join(f"{v:.20g}    " for v in row) + "\n")
    return cdir


def hbn_rk4(workdir, n=60, field=0.3, photon=0.4, duration=30.0, dt_fs=0.01, t_fin_fs=None, it_res=1,
            solver="", gap=5.8, t1=2.3, extra_tdse="", probe="", phase=0.0):
    os.makedirs(workdir, exist_ok=True)
    t_fin = duration if t_fin_fs is None else t_fin_fs
    txt = (
        "HBN\n\n"
        "tdse{\n"
        f"tightbinding Haldane_CoreBN_Nedge gap= {gap} t1= {t1} t2= 0 phi0= 0\n"
        f"dt {dt_fs} fs\n"
        f"t_fin {t_fin} fs\n"
        f"{solver}{extra_tdse}"
        "}\n\n"
        f"nkpt{{\n1 {n} {n}\n}}\n\n"
        + _pump(photon, field, duration, phase=phase)
        + probe
        + "\nobservables{\n"
        "Current\n"
        f"it_resolution {it_res}\n"
        "}\n"
    )
    path = os.path.join(workdir, "input.txt")
    with open(path, "w") as f:
        f.write(txt)
    return path


def hbn_coulomb(workdir, n=120, field=0.5, photon=0.4, duration=30.0, dt_fs=0.005, t_fin_fs=None, it_res=10, ab_order=4,
                rk4_startup=True, rk4=False, phase=0.0, r0_ang=None, label=COULOMB_LABEL, tables=None):
    """hBN with the Rytova-Keldysh mean field, Adams-Bashforth (or RK4 with
    rk4=True). Tables: the packaged Ncut=20 files (the reference's shipped ones,
    r0 = 10 A) unless `tables` names an Output/Coulomb directory made for
    r0_ang by coulomb_tables_for (label = its file label)."""
    os.makedirs(workdir, exist_ok=True)
    if tables is None:
        write_coulomb_files(workdir)
    else:
        os.makedirs(os.path.join(workdir, "Output"), exist_ok=True)
        link = os.path.join(workdir, "Output", "Coulomb")
        if not os.path.exists(link):
            os.symlink(tables, link)
    solver = "" if rk4 else f"Adams_Bashforth {ab_order}\n" + ("Adams_Bashforth_RK4_startup\n" if rk4_startup else "")
    path = hbn_rk4(workdir, n=n, field=field, photon=photon, duration=duration, dt_fs=dt_fs, t_fin_fs=t_fin_fs,
                   it_res=it_res, solver=solver, phase=phase)
    with open(path, "a") as f:
        f.write(
            "\nCoulomb{\n"
            "qTF 0.01\n"
            "Ncut 20\n"
            "epsilon_static 1.0\n"
            "Rytova_Keldysh\n"
            + (f"r0 {r0_ang * ANG_AU:.12g}\n" if r0_ang is not None else "")
            + "Read_Coulomb_from_files\n"
            f"labelInput {label}\n"
            "}\n"
        )
    return path


def coulomb_tables_for(root, r0_ang, device=0):
    """Generate (once, on the GPU) the Coulomb tables of the hBN model for a
    screening length r0_ang [A] (Rytova-Keldysh, qTF 0.01, Ncut 20, the
    reference's default G_distance) under root/r0_<r0>/Output/Coulomb.
    Returns (directory of the tables, their file label)."""
    import edus_b200 as E

    d = os.path.join(root, f"r0_{r0_ang:g}")
    cdir = os.path.join(d, "Output", "Coulomb")
    stamp = os.path.join(d, "label.txt")
    if os.path.exists(stamp):
        return cdir, open(stamp).read().strip()
    os.makedirs(d, exist_ok=True)
    path = hbn_rk4(d, n=12, t_fin_fs=0.0)
    with open(path, "a") as f:
        f.write(f"\nCoulomb{{\nqTF 0.01\nNcut 20\nepsilon_static 1.0\nRytova_Keldysh\nr0 {r0_ang * ANG_AU:.12g}\n"
                f"labelInput r0_{r0_ang:g}A_\n}}\n")
    label, _ = E.coulomb_generate(E.parse_input(path), d, device=device)
    with open(stamp, "w") as f:
        f.write(label)
    return cdir, label


def write_wannier_tb(path, nw=8, nside=11, seed=12345, a_ang=2.5, decay_h=1.5, decay_r=1.0, onsite_ev=3.0):
    """Synthetic Wannier90 _tb.dat: H(R) complex Gaussian x exp(-|R|/decay_h a),
    hermitised H(-R) = H(R)^dagger, onsite energies uniform in +-onsite_ev;
    r(R) the same with exp(-|R|/decay_r a). Square lattice, R = (0, R1, R2)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    h = nside // 2
    Rs = [(0, r1, r2) for r1 in range(-h, h + 1) for r2 in range(-h, h + 1)]
    idx = {R: i for i, R in enumerate(Rs)}
    nr = len(Rs)
    HR = np.zeros((nr, nw, nw), complex)
    rR = np.zeros((3, nr, nw, nw), complex)
    for i, R in enumerate(Rs):
        neg = idx[(0, -R[1], -R[2])]
        if neg < i:
            continue
        dist = math.hypot(R[1], R[2])
        g = (rng.standard_normal((nw, nw)) + 1j * rng.standard_normal((nw, nw))) / math.sqrt(2)
        g *= math.exp(-dist / decay_h)
        gr = (rng.standard_normal((3, nw, nw)) + 1j * rng.standard_normal((3, nw, nw))) / math.sqrt(2)
        gr *= 0.5 * math.exp(-dist / decay_r)
        if neg == i:  # R = 0
            g = 0.5 * (g + g.conj().T)
            np.fill_diagonal(g, rng.uniform(-onsite_ev, onsite_ev, nw))
            gr = 0.5 * (gr + gr.conj().transpose(0, 2, 1))
            for x in range(3):
                np.fill_diagonal(gr[x], np.real(np.diag(gr[x])))
            HR[i] = g
            rR[:, i] = gr
        else:
            HR[i] = g
            HR[neg] = g.conj().T
            rR[:, i] = gr
            rR[:, neg] = gr.conj().transpose(0, 2, 1)
    with open(path, "w") as f:
        f.write("synthetic tight-binding model (written by edus_b200.workloads)\n")
        f.write(f"  {10.0:.8f} 0 0\n  0 {a_ang:.8f} 0\n  0 0 {a_ang:.8f}\n")
        f.write(f"{nw}\n{nr}\n")
        for i in range(nr):
            f.write("    1" + ("\n" if (i + 1) % 15 == 0 else ""))
        f.write("\n")
        for i, R in enumerate(Rs):
            f.write(f"\n{R[0]} {R[1]} {R[2]}\n")
            for n_ in range(nw):
                for m in range(nw):
                    v = HR[i, m, n_]
                    f.write(f"{m + 1} {n_ + 1} {v.real:.16e} {v.imag:.16e}\n")
        for i, R in enumerate(Rs):
            f.write(f"\n{R[0]} {R[1]} {R[2]}\n")
            for n_ in range(nw):
                for m in range(nw):
                    x, y, z = rR[0, i, m, n_], rR[1, i, m, n_], rR[2, i, m, n_]
                    f.write(f"{m + 1} {n_ + 1} {x.real:.16e} {x.imag:.16e} {y.real:.16e} {y.imag:.16e} {z.real:.16e} {z.imag:.16e}\n")
    return path


def wannier(workdir, nw=8, nside=11, n=96, field=0.4, photon=0.3, duration=40.0, dt_fs=0.01, t_fin_fs=None, it_res=10,
            seed=12345, name="W8", phase=0.0, write_model=True, pol="0 0 1"):
    os.makedirs(workdir, exist_ok=True)
    if write_model or not os.path.exists(os.path.join(workdir, f"{name}_tb.dat")):
        write_wannier_tb(os.path.join(workdir, f"{name}_tb.dat"), nw=nw, nside=nside, seed=seed)
    nv = nw // 2
    t_fin = duration if t_fin_fs is None else t_fin_fs
    txt = (
        f"{name}\n\n"
        "unitcell angstrom {\n10.0 0 0\n0 2.5 0\n0 0 2.5\n}\n\n"
        f"bands{{\nvalence {nv}\nconduction {nw - nv}\n}}\n\n"
        "tdse{\nWannier\n"
        f"dt {dt_fs} fs\n"
        f"t_fin {t_fin} fs\n"
        "}\n\n"
        f"nkpt{{\n1 {n} {n}\n}}\n\n"
        + _pump(photon, field, duration, pol=pol, phase=phase)
        + "\nobservables{\nCurrent\n"
        f"it_resolution {it_res}\n"
        "}\n"
    )
    path = os.path.join(workdir, "input.txt")
    with open(path, "w") as f:
        f.write(txt)
    return path


def crystal_model(nb=2, norb=None, seed=7, nh=2):
    """Seeded smooth periodic model for the Crystal interface: Hermitian H(k)
    and x, y Berry connections as short Fourier series in the crystal
    coordinates (k1, k2), a.u. Returns a function k1, k2 -> (H, Dx, Dy) of
    norb x norb matrices (norb >= nb; the extra orbitals lie far above)."""
    norb = nb if norb is None else norb
    rng = np.random.Generator(np.random.PCG64(seed))
    terms = []
    for m1 in range(-nh, nh + 1):
        for m2 in range(-nh, nh + 1):
            scale = 0.08 / (1 + m1 * m1 + m2 * m2)
            c = [(rng.standard_normal((norb, norb)) + 1j * rng.standard_normal((norb, norb))) * scale for _ in range(3)]
            terms.append((m1, m2, c))
    onsite = np.diag(np.linspace(-0.2, 0.2, norb) + np.where(np.arange(norb) >= nb, 2.0, 0.0))

    def at(k1, k2):
        out = [np.zeros((norb, norb), np.complex128) for _ in range(3)]
        for m1, m2, c in terms:
            ph = np.exp(2j * np.pi * (m1 * k1 + m2 * k2))
            for x in range(3):
                out[x] += c[x] * ph
        H, Dx, Dy = [(o + o.conj().T) / 2 for o in out]
        H = H + onsite
        H[np.diag_indices(norb)] = H.diagonal().real
        # the files carry an imaginary diagonal in the connections; the model drops it
        Dx = Dx + 1j * 1e-3 * np.eye(norb)
        Dy = Dy - 1j * 2e-3 * np.eye(norb)
        return H, Dx, Dy

    return at


def write_crystal_files(workdir, nb=2, norb=None, nkf=13, seed=7, alat=4.72):
    """The Crystal interface's input files (kmesh_data.dat, hk_orthonormal.dat,
    bc_betabetap_real.dat, bc_betabetap_imag.dat) for `crystal_model` on an
    nkf x nkf grid over [-0.5, 0.5] in each crystal direction, k1 major, the
    lower triangles row by row. Returns (model, grid, a, b) with grid the
    crystal coordinates of the samples and a, b the in-plane lattice rows."""
    norb = nb if norb is None else norb
    model = crystal_model(nb, norb, seed)
    os.makedirs(workdir, exist_ok=True)
    a = np.array([[alat * math.cos(math.pi / 6), alat * math.sin(math.pi / 6)],
                  [alat * math.cos(math.pi / 6), -alat * math.sin(math.pi / 6)]])
    b = 2 * math.pi * np.linalg.inv(a).T
    grid = -0.5 + np.arange(nkf) / (nkf - 1)
    f = lambda v: " ".join(f"{x:.17g}" for x in v)
    with open(os.path.join(workdir, "kmesh_data.dat"), "w") as fp:
        fp.write(f"a0 (bohr)\n{f(a[0])}\na1\n{f(a[1])}\nb0 (1/bohr)\n{f(b[0])}\nb1\n{f(b[1])}\n")
        fp.write("atomic positions\nB 0.0 0.0\nN 0.5 0.5\norbital basis\n")
        fp.write(f"{norb}\nk points along each direction\n{nkf}\nindex kx ky\n")
        i = 0
        for k1 in grid:
            for k2 in grid:
                kc = k1 * b[0] + k2 * b[1]
                i += 1
                fp.write(f"{i} {f(kc)}\n")
    lower = lambda M, part: "".join(" ".join(f"{part(M[i, j]):.17g}" for j in range(i + 1)) + "\n" for i in range(norb))
    with open(os.path.join(workdir, "hk_orthonormal.dat"), "w") as fh, \
            open(os.path.join(workdir, "bc_betabetap_real.dat"), "w") as fr, \
            open(os.path.join(workdir, "bc_betabetap_imag.dat"), "w") as fi:
        for k1 in grid:
            for k2 in grid:
                H, Dx, Dy = model(k1, k2)
                fh.write(lower(H, np.real) + "\n" + lower(H, np.imag) + "\n\n")
                fr.write(lower(Dx, np.real) + "\n" + lower(Dy, np.real) + "\n\n")
                fi.write(lower(Dx, np.imag) + "\n" + lower(Dy, np.imag) + "\n\n")
    return model, grid, a, b


def crystal(workdir, nb=(1, 1), norb=None, nkf=13, n=12, field=0.3, photon=0.4, duration=20.0, dt_fs=0.01,
            t_fin_fs=None, it_res=5, seed=7):
    """input.txt for the Crystal interface (tdse{ Crystal }) with the files of
    `write_crystal_files`; nb = (valence, conduction) bands. Returns the path."""
    write_crystal_files(workdir, nb=sum(nb), norb=norb, nkf=nkf, seed=seed)
    t_fin = duration if t_fin_fs is None else t_fin_fs
    txt = (
        "CRY\n\n"
        f"bands{{\nvalence {nb[0]}\nconduction {nb[1]}\n}}\n\n"
        "tdse{\nCrystal\n"
        f"dt {dt_fs} fs\n"
        f"t_fin {t_fin} fs\n"
        "}\n\n"
        f"nkpt{{\n1 {n} {n}\n}}\n\n"
        + _pump(photon, field, duration)
        + "\nobservables{\nCurrent\n"
        f"it_resolution {it_res}\n"
        "}\n"
    )
    path = os.path.join(workdir, "input.txt")
    with open(path, "w") as fp:
        fp.write(txt)
    return path


def sweep(count=256, seed=20261203, nmin=48, nmax=144, emin=0.05, emax=0.8, dmin=10.0, dmax=60.0, it_res=10,
          dt_fs=0.01):
    """Seeded pulse sweep: half hBN (hbn_rk4 model), half the 8-band Wannier
    model of `wannier`; grid N x N with N even, uniform in [nmin, nmax]; peak
    field log-uniform in [emin, emax] V/A; CEP uniform in [0, 2 pi); pulse
    duration uniform in [dmin, dmax] fs (the run ends with the pulse).
    Returns a list of dicts (kind, n, field, phase, duration, ...)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for i in range(count):
        kind = "hbn" if i % 2 == 0 else "wannier"
        n = 2 * int(rng.integers(nmin // 2, nmax // 2 + 1))
        field = float(math.exp(rng.uniform(math.log(emin), math.log(emax))))
        phase = float(rng.uniform(0.0, 2 * math.pi))
        duration = float(rng.uniform(dmin, dmax))
        out.append(dict(kind=kind, n=n, field=field, phase=phase, duration=duration, it_res=it_res, dt_fs=dt_fs))
    return out


def write_instance(workdir, spec):
    """input.txt (and model file) of one sweep or serving instance."""
    if spec["kind"] == "hbn":
        return hbn_rk4(workdir, n=spec["n"], field=spec["field"], duration=spec["duration"], it_res=spec["it_res"],
                       dt_fs=spec["dt_fs"], phase=spec["phase"])
    return wannier(workdir, nw=spec.get("nw", 8), nside=spec.get("nside", 11), n=spec["n"], field=spec["field"],
                   duration=spec["duration"], it_res=spec["it_res"], dt_fs=spec["dt_fs"], phase=spec["phase"],
                   name=spec.get("name", "W8"), write_model=False)
