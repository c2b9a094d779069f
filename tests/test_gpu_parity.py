"""Parity of the sm_100a path with the CPU oracle (and the reference's golden run).

Tolerances: the FP64 path must match the reference to <= 1e-12 relative in rho_k
and J(t). rho is compared as max |difference| (entries are O(1)); J1 by relative
L2 over t; J2 and populations, whose small values come from cancelling sums over
k, by absolute difference against their noise floor.
"""
import os

import numpy as np
import pytest

import edus_b200 as E
from edus_b200 import abi
from edus_b200 import workloads as W
from conftest import GOLDEN, GOLDEN_INPUT
from oracle_lib import Oracle
from ref_fixtures import snapshot_schedule as _snapshot_schedule

pytestmark = pytest.mark.gpu

RHO_TOL = 1e-13   # max |rho_gpu - rho_oracle|
J1_TOL = 1e-11    # relative L2 over t
TIME_AU_FS = 0.02418884326505


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300))


def run_pair(path, wd, steps, **ctx_kw):
    p = E.parse_input(path)
    pb = E.Problem(p, wd)
    ctx = E.Context(pb, **ctx_kw)
    ctx.step(steps)
    o = Oracle(p, wd)
    lo = o.run(steps)
    return ctx, o, ctx.obs(), lo


def check_logs(g, o, pop_abs=2e-15, j2_abs=0.0):
    assert len(g) == len(o) and len(g) > 0
    for a, b in zip(g, o):
        assert a["t"] == b["t"]
        np.testing.assert_array_equal(a["EF_pump"], b["EF_pump"])
    J1g, J1o = np.array([x["J1"] for x in g]), np.array([x["J1"] for x in o])
    if np.abs(J1o).max() > 1e-14:
        assert rel(J1g, J1o) < J1_TOL
    J2g, J2o = np.array([x["J2"] for x in g]), np.array([x["J2"] for x in o])
    assert np.abs(J2g - J2o).max() <= 1e-9 * max(np.abs(J2o).max(), 1e-20) + j2_abs
    pg, po = np.array([x["pop"] for x in g]), np.array([x["pop"] for x in o])
    assert np.abs(pg - po).max() <= pop_abs
    # polarisation per cell, (1/Nk) sum_k Tr(D rho): an O(1) sum, held like the populations
    Pg, Po = np.array([x["pol"] for x in g]), np.array([x["pol"] for x in o])
    assert np.abs(Pg - Po).max() <= 1e-13 * max(np.abs(Po).max(), 1.0)


def test_rhs_matches_oracle():
    p = E.parse_input(GOLDEN_INPUT)
    pb = E.Problem(p)
    ctx = E.Context(pb)
    o = Oracle(p)
    rng = np.random.default_rng(1)
    P0 = pb.get("P0")
    X = (rng.standard_normal(P0.shape) + 1j * rng.standard_normal(P0.shape)) * 0.01
    P = P0 + X + np.conj(np.transpose(X, (0, 2, 1)))
    for i in range(P.shape[1]):
        P[:, i, i] = P[:, i, i].real
    for EF, e_non0 in [([0.0, 3e-4, -2e-4, 1e-5, 0.0, 0.0], 1), ([0, 0, 0, 0, 0, 0], 0)]:
        ctx.slot_set(abi.SLOT_P0, P)
        ctx.get_derivative(abi.SLOT_P0, EF, p.probe.wl, e_non0)
        g = ctx.slot_get(abi.SLOT_PV)
        r = o.rhs(P, EF, p.probe.wl, e_non0)
        assert np.abs(g - r).max() <= 1e-15 * max(1.0, np.abs(r).max() * 10)
        # Pv is Hermitian with a real diagonal, exactly
        assert np.array_equal(g, np.conj(np.transpose(g, (0, 2, 1))))


def test_stage_updates_match_reference_formulae():
    p = E.parse_input(GOLDEN_INPUT)
    pb = E.Problem(p)
    ctx = E.Context(pb)
    P0 = pb.get("P0")
    ctx.slot_set(abi.SLOT_P0, P0)
    ctx.get_derivative(abi.SLOT_P0, [0, 1e-3, 0, 0, 0, 0], 0.0, 1)
    Pv = ctx.slot_get(abi.SLOT_PV)
    ctx.runge_kutta_ad(abi.SLOT_P0, abi.SLOT_P1, 0.05)  # Runge_Kutta_Ad: P1 = P0 + dt Pv
    # (multiply, then add: bit for bit the unfused arithmetic of the reference's loops)
    np.testing.assert_array_equal(ctx.slot_get(abi.SLOT_P1), P0 + Pv * 0.05)
    ctx.runge_kutta_ac(abi.SLOT_P1, 0.05)  # Runge_Kutta_Ac: P1 += dt Pv
    np.testing.assert_array_equal(ctx.slot_get(abi.SLOT_P1), (P0 + Pv * 0.05) + Pv * 0.05)


def test_golden_run_on_gpu():
    """The whole shipped AB5 run (16591 steps) on the GPU against the golden outputs."""
    p = E.parse_input(GOLDEN_INPUT)
    ctx = E.Context(E.Problem(p))
    ctx.run()
    log = ctx.obs()
    G = np.load(os.path.join(GOLDEN, "ab5_golden.npz"))
    rows = G["rows"]
    assert len(log) == int(G["nrows"])
    J1 = np.array([log[i]["J1"] for i in rows])
    J1r = G["J1"][:, 1::2] + 1j * G["J1"][:, 2::2]
    assert rel(J1, J1r) < 1e-12
    J2 = np.array([log[i]["J2"] for i in rows])
    assert np.abs(J2 - G["J2"][:, 1:]).max() < 1e-10 * np.abs(G["J2"][:, 1:]).max()
    pop = np.array([log[i]["pop"] for i in rows])
    assert np.abs(pop - G["Losses"][:, 1:4]).max() < 1e-13
    assert rel(pop[:, 2], G["Losses"][:, 3]) < 1e-11


def test_rk4_matches_oracle(workdir):
    ctx, o, g, lo = run_pair(W.hbn_rk4(workdir, n=24, t_fin_fs=3.0, it_res=5), workdir, 400)
    assert np.abs(ctx.get_state() - o.get("P0")).max() < RHO_TOL
    check_logs(g, lo)


def test_coulomb_ab4_rk4_startup_matches_oracle(workdir):
    ctx, o, g, lo = run_pair(W.hbn_coulomb(workdir, n=24, t_fin_fs=2.0, it_res=5), workdir, 300)
    assert np.abs(ctx.get_state() - o.get("P0")).max() < RHO_TOL
    check_logs(g, lo)
    P = ctx.get_state()
    np.testing.assert_allclose(ctx.coulomb_hk(abi.SLOT_P0), o.coulomb_hk(P), rtol=0, atol=1e-14)


def test_coulomb_diagonal_basis_matches_oracle(workdir):
    """Coulomb_diag_basis (headers/RungeKutta.h:35-55, 96-123): coefficients of the
    state in the eigenbasis, that basis's screening, X rotated back by U; the
    equilibrium of the filled bands (main_MPI.cpp:291-304)."""
    path = W.hbn_coulomb(workdir, n=24, t_fin_fs=2.0, it_res=5)
    txt = open(path).read().replace("Rytova_Keldysh\n", "Rytova_Keldysh\nCoulomb_diag_basis\n")
    open(path, "w").write(txt)
    ctx, o, g, lo = run_pair(path, workdir, 300)
    assert np.abs(ctx.get_state() - o.get("P0")).max() < RHO_TOL
    # J2 (~7e-9 here) comes from sums over k of O(1e-1) terms that cancel: the
    # two rotations by U of this basis leave its last bits (1.1e-17 measured) at
    # that sum's FP64 rounding floor, so it is compared against the floor
    check_logs(g, lo, j2_abs=1e-16)
    P = ctx.get_state()
    # renormalised H = H + a ~1e-4 mean-field term, compared well below that term
    np.testing.assert_allclose(ctx.coulomb_hk(abi.SLOT_P0), o.coulomb_hk(P), rtol=0, atol=1e-12)


def test_coulomb_ab4_zero_history_matches_oracle(workdir):
    ctx, o, g, lo = run_pair(W.hbn_coulomb(workdir, n=24, t_fin_fs=2.0, it_res=5, rk4_startup=False), workdir, 300)
    assert np.abs(ctx.get_state() - o.get("P0")).max() < RHO_TOL
    check_logs(g, lo)


def test_taylor_dynamic_dt_matches_oracle(workdir):
    solver = "Taylor\nTaylorOrder 6\ndynamical_dt_evolution\nepsStepAbs 0.02\n"
    ctx, o, g, lo = run_pair(W.hbn_rk4(workdir, n=24, t_fin_fs=2.0, it_res=3, solver=solver, dt_fs=0.002), workdir, 300)
    assert np.abs(ctx.get_state() - o.get("P0")).max() < RHO_TOL
    # the adaptive step divides by a population change of ~1e-9 (dyn_dt_evolution.cpp:88):
    # its relative rounding is ~1e-7, so compare times loosely and populations absolutely
    it_g, t_g, dt_g = ctx.clock()
    it_o, t_o, dt_o = o.clock()
    assert it_g == it_o and abs(t_g - t_o) < 1e-6
    pg, po = np.array([x["pop"] for x in g]), np.array([x["pop"] for x in lo])
    assert np.abs(pg - po).max() < 1e-14


def test_rk4_dynamic_dt_matches_oracle(workdir):
    ctx, o, g, lo = run_pair(W.hbn_rk4(workdir, n=24, t_fin_fs=2.0, it_res=3, solver="dynamical_dt_evolution\nepsStepAbs 0.001\n"),
                             workdir, 200)
    assert np.abs(ctx.get_state() - o.get("P0")).max() < 1e-12
    assert ctx.clock()[0] == o.clock()[0]


def _dyn_input(kind, d):
    if kind == "rk4":
        return W.hbn_rk4(d, n=24, t_fin_fs=2.0, it_res=3, solver="dynamical_dt_evolution\nepsStepAbs 0.001\n")
    if kind == "taylor":
        return W.hbn_rk4(d, n=24, t_fin_fs=2.0, it_res=3, dt_fs=0.002,
                         solver="Taylor\nTaylorOrder 6\ndynamical_dt_evolution\nepsStepAbs 0.02\n")
    if kind == "snapshots":
        path = W.hbn_rk4(d, n=12, t_fin_fs=1.5, it_res=10, solver="dynamical_dt_evolution\nepsStepAbs 0.001\n")
        txt = open(path).read().replace("Current\n", "Current\nPrintPopulation 0 60 15\n")
    else:  # Coulomb mean field with RK4 and band-energy snapshots
        path = W.hbn_coulomb(d, n=24, t_fin_fs=0.6, it_res=10, rk4=True)
        txt = open(path).read().replace("tdse{\n", "tdse{\ndynamical_dt_evolution\nepsStepAbs 0.001\n")
        txt = txt.replace("Rytova_Keldysh\n", "Rytova_Keldysh\nPrint_new_band_dispersion\n")
    open(path, "w").write(txt)
    return path


@pytest.mark.parametrize("kind", ["rk4", "taylor", "snapshots", "coulomb"])
def test_adaptive_step_on_device_matches_host_loop(workdir, kind):
    """A whole adaptive run (dynamical_dt_evolution) with the step picked on the
    device (k_dyn_begin / k_dyn_end around captured chunks, no host round trip
    per step) against the host-driven loop (EDUS_DYN_HOST=1: the max copied to
    the host every step, Source_Main/dyn_dt_evolution.cpp:64-133): the same
    number of steps and output instants, the same snapshot times, clock and
    observables within the rounding of the device's sin / cos / exp in the
    laser field; the device run replays after edus_reset."""
    d = f"{workdir}/{kind}"
    path = _dyn_input(kind, d)
    p = E.parse_input(path)
    assert p.dynamical_dt
    pb = E.Problem(p, d)
    dev = E.Context(pb)
    dev.run()
    os.environ["EDUS_DYN_HOST"] = "1"
    try:
        host = E.Context(pb)
        host.run()
    finally:
        del os.environ["EDUS_DYN_HOST"]
    # the device loop launches no host-side step: far fewer host calls, all captured
    assert dev.last_timing()[1] > 0
    it_d, t_d, dt_d = dev.clock()
    it_h, t_h, dt_h = host.clock()
    assert it_d == it_h
    assert abs(t_d - t_h) <= 1e-9 * abs(t_h) and abs(dt_d - dt_h) <= 1e-9 * abs(dt_h)
    gd, gh = dev.obs(), host.obs()
    assert len(gd) == len(gh) > 0
    np.testing.assert_allclose([x["t"] for x in gd], [x["t"] for x in gh], rtol=1e-9)
    np.testing.assert_allclose([x["dt"] for x in gd], [x["dt"] for x in gh], rtol=1e-9)
    assert rel([x["J1"] for x in gd], [x["J1"] for x in gh]) < 1e-9
    assert np.abs(np.array([x["pop"] for x in gd]) - np.array([x["pop"] for x in gh])).max() < 1e-12
    assert np.abs(dev.get_state() - host.get_state()).max() < 1e-10
    od, oh = f"{d}/out_dev", f"{d}/out_host"
    dev.write_outputs(od)
    host.write_outputs(oh)
    if kind in ("snapshots", "coulomb"):
        td = [float(x) for x in open(f"{od}/t_Ek.txt").read().split()]
        th = [float(x) for x in open(f"{oh}/t_Ek.txt").read().split()]
        assert len(td) == len(th) > 0
        np.testing.assert_allclose(td, th, rtol=1e-9)
        names = sorted(f for f in os.listdir(oh) if f.startswith(("P_val", "P_cond", "Edia_")))
        assert names and names == sorted(f for f in os.listdir(od) if f.startswith(("P_val", "P_cond", "Edia_")))
        for f in names:
            a, b = np.loadtxt(f"{od}/{f}"), np.loadtxt(f"{oh}/{f}")
            assert np.all(np.abs(a - b) <= 1e-6 * np.abs(b) + 1e-12), f
    # replay of the captured chunk after a reset
    rho = dev.get_state()
    dev.reset()
    dev.run()
    assert np.array_equal(dev.get_state(), rho)
    assert dev.clock()[0] == it_d


def test_wannier_8band_matches_oracle(workdir):
    ctx, o, g, lo = run_pair(W.wannier(workdir, n=16, t_fin_fs=1.0, it_res=5), workdir, 100)
    assert np.abs(ctx.get_state() - o.get("P0")).max() < RHO_TOL
    check_logs(g, lo)


def test_graph_replay_equals_eager(workdir):
    path = W.hbn_coulomb(workdir, n=24, t_fin_fs=1.0, it_res=5)
    pb = E.Problem(E.parse_input(path), workdir)
    a = E.Context(pb, use_graphs=True)
    a.run()
    sa, la = a.get_state(), a.obs()
    b = E.Context(pb, use_graphs=False)
    b.run()
    assert np.array_equal(sa, b.get_state())
    a.reset()
    a.run()
    assert np.array_equal(sa, a.get_state())
    assert all(np.array_equal(x["J1"], y["J1"]) for x, y in zip(la, a.obs()))


def test_write_outputs_format(workdir, tmp_path):
    p = E.parse_input(GOLDEN_INPUT)
    p.t_fin = -8.0  # a few output instants only
    ctx = E.Context(E.Problem(p))
    ctx.run()
    out = str(tmp_path / "Output")
    ctx.write_outputs(out)
    log = ctx.obs()
    lines = open(os.path.join(out, "J1.txt")).read().splitlines()
    assert len(lines) == len(log)
    # the reference leaves std::scientific set after the first line (Observables_MPI.h:710)
    assert lines[0].startswith("          -0.21")
    assert "e-01" in lines[1].split()[0]
    vals = np.array([[float(x) for x in l.split()] for l in lines])
    J1 = np.array([x["J1"] for x in log])
    np.testing.assert_allclose(vals[:, 1::2], J1.real, rtol=1e-14, atol=1e-300)
    losses = open(os.path.join(out, "Losses.txt")).read().splitlines()
    assert losses[0].split()[0] == "-0.21" and len(losses[0].split()) == 4


def test_edus_run_writes_the_reference_outputs(tmp_path):
    """The drop-in executable on the shipped AB5 input: Output/J1.txt and
    Output/Losses.txt against the golden run, as a user of the reference reads them."""
    import shutil
    import subprocess

    from edus_b200 import build

    shutil.copy(GOLDEN_INPUT, tmp_path / "input.txt")
    r = subprocess.run([build.EXE], capture_output=True, text=True, cwd=tmp_path, timeout=600)
    assert r.returncode == 0, r.stderr
    G = np.load(os.path.join(GOLDEN, "ab5_golden.npz"))
    rows = G["rows"]
    J1 = np.loadtxt(tmp_path / "Output" / "J1.txt")
    assert len(J1) == int(G["nrows"])
    assert rel(J1[rows, 1:], G["J1"][:, 1:]) < 1e-12
    L = np.loadtxt(tmp_path / "Output" / "Losses.txt")
    assert np.abs(L[rows, 1:4] - G["Losses"][:, 1:4]).max() < 1e-13
    import hashlib
    import json

    kg = json.load(open(os.path.join(GOLDEN, "ab5_kgrid.json")))
    assert hashlib.sha256((tmp_path / "Output" / "k_grid.txt").read_bytes()).hexdigest() == kg["sha256"]


@pytest.mark.parametrize("graphs", [True, False])
def test_per_k_snapshots_match_oracle(workdir, graphs):
    """PrintPopulation snapshots: Output/t_Ek.txt holds the reference's schedule and
    every snapshot's three files hold, per k, the top-valence / bottom-conduction
    elements of the state in the model's eigenbasis (get_P_in_dia,
    headers/InitParameters.h:232-255) of the oracle's state at that step, to the
    6 printed digits; a replay after edus_reset writes the same files."""
    d = f"{workdir}/snap{int(graphs)}"
    path = W.hbn_rk4(d, n=12, t_fin_fs=1.5, it_res=10)
    txt = open(path).read().replace("Current\n", "Current\nPrintPopulation 0 60 15\n")
    open(path, "w").write(txt)
    p = E.parse_input(path)
    pb = E.Problem(p, d)
    ctx = E.Context(pb, use_graphs=graphs)
    ctx.run()
    out = f"{d}/Output"
    ctx.write_outputs(out)
    sched = _snapshot_schedule(pb.info.t_start, p.dt, pb.info.nsteps - 1, 10, 0.0, 60.0, 15.0)
    assert len(sched) == 5
    t_ek = [float(x) for x in open(f"{out}/t_Ek.txt").read().split()]
    np.testing.assert_allclose(t_ek, [t * TIME_AU_FS for _, t in sched], rtol=1e-5)
    nb = pb.info.nch + pb.info.nv
    v, c = nb - 1, nb
    o = Oracle(p, d)
    U = o.get("U")
    done = 0
    files = {}
    for m, (it, _) in enumerate(sched):
        o.run(it - done)
        done = it
        P = o.get("P0")
        Pd = np.einsum("kri,kij,kcj->krc", U.conj(), P, U)
        for label, (r, cc) in [("P_val_cond_in_Eigenstate", (v, c)), ("P_val_in_Eigenstate", (v, v)),
                               ("P_cond_in_Eigenstate", (c, c))]:
            name = f"{out}/{label}_{r}{cc}_{m}.txt"
            files[name] = open(name).read()
            got = np.loadtxt(name)
            assert got.shape == (pb.info.nk, 2)
            want = np.stack([Pd[:, r, cc].real, Pd[:, r, cc].imag], axis=1)
            assert np.all(np.abs(got - want) <= 1e-5 * np.abs(want) + 1e-12), (label, m)
    assert not os.path.exists(f"{out}/P_val_in_Eigenstate_{v}{v}_5.txt")
    ctx.reset()
    ctx.run()
    ctx.write_outputs(out)
    for name, text in files.items():
        assert open(name).read() == text


def test_coulomb_band_energy_snapshots_match_oracle(workdir):
    """Print_new_band_dispersion with the Coulomb mean field: Output/Edia_<m>.txt
    holds, per k, the ascending eigenvalues of the renormalised Hamiltonian of
    the last RHS evaluation (headers/Observables_MPI.h:282-303, 440-478) at each
    snapshot of the default print window, against the oracle's."""
    d = f"{workdir}/edia"
    path = W.hbn_coulomb(d, n=24, t_fin_fs=0.3, it_res=10)
    txt = open(path).read().replace("Rytova_Keldysh\n", "Rytova_Keldysh\nPrint_new_band_dispersion\n")
    open(path, "w").write(txt)
    p = E.parse_input(path)
    pb = E.Problem(p, d)
    ctx = E.Context(pb)
    ctx.run()
    out = f"{d}/Output"
    ctx.write_outputs(out)
    sched = _snapshot_schedule(pb.info.t_start, p.dt, pb.info.nsteps - 1, 10, p.print_start, p.print_end, p.print_step)
    assert len(sched) == 2
    t_ek = [float(x) for x in open(f"{out}/t_Ek.txt").read().split()]
    np.testing.assert_allclose(t_ek, [t * TIME_AU_FS for _, t in sched], rtol=1e-5)
    o = Oracle(p, d)
    done = 0
    for m, (it, _) in enumerate(sched):
        o.run(it - done)
        done = it
        want = np.linalg.eigvalsh(o.get("Hr"))
        got = np.loadtxt(f"{out}/Edia_{m}.txt")
        assert got.shape == want.shape
        assert np.abs(got - want).max() < 1e-11
    assert not os.path.exists(f"{out}/Edia_2.txt")
    assert not any(f.startswith("P_val") for f in os.listdir(out))


def test_first_output_step_files_match_oracle(workdir):
    """The files every reference run writes at its first output step
    (Print_initial_H_P, Source_Main/if_resolution.cpp:275-328): eigenvalues of
    the model H (H_Eigen_*), H_cc, the initial state's cc element and U_cc, U_cv,
    per k, against the oracle's tables to the 6 printed digits."""
    d = f"{workdir}/init"
    path = W.hbn_rk4(d, n=12, t_fin_fs=0.05, it_res=1)
    # with kTAbs: the reference opens one TAbsK file per listed k point and writes nothing into it
    txt = open(path).read().replace("Current\n", "Current\nkTAbs\n") + "\nTAbsK{\n1\n0 0.1 0.2\n}\n"
    open(path, "w").write(txt)
    p = E.parse_input(path)
    pb = E.Problem(p, d)
    ctx = E.Context(pb)
    ctx.run()
    out = f"{d}/Output"
    ctx.write_outputs(out)
    o = Oracle(p, d)
    H, U, P0 = o.get("H"), o.get("U"), o.get("P0")
    eps = np.linalg.eigvalsh(H)
    nb = pb.info.nch + pb.info.nv
    v, c = nb - 1, nb
    want = {
        f"H_Eigen_cond_{c}{c}_0": eps[:, c], f"H_Eigen_val_{v}{v}_0": eps[:, v],
        f"H_Eigen_val_cond_{v}{c}_0": np.zeros(pb.info.nk), f"H_Wannier_cond_{c}{c}_0": H[:, c, c],
        f"P_initial_Wannier__{c}{c}_0": P0[:, c, c], f"Uk__{c}{c}_0": U[:, c, c], f"Uk__{c}{v}_0": U[:, c, v],
    }
    assert os.path.getsize(f"{out}/TAbsK_0_0.1_0.2.txt") == 0
    for name, w in want.items():
        got = np.loadtxt(f"{out}/{name}.txt")
        wv = np.stack([np.real(w), np.imag(w)], axis=1)
        assert got.shape == wv.shape, name
        assert np.all(np.abs(got - wv) <= 1e-5 * np.abs(wv) + 1e-12), name


def test_bounded_wait_runs_out_with_etimeout(workdir):
    """A kernel's bounded wait on an mbarrier nothing arrives on runs out: the
    call returns EDUS_ETIMEOUT (no fault, no hang) and the device still runs a
    solve afterwards."""
    L = E.load_library()
    rc = L.edus_selftest_bounded_wait(0, 1000)
    assert rc == abi.EDUS_ETIMEOUT, rc
    assert b"ran out" in L.edus_last_error()
    ctx, o, g, lo = run_pair(W.hbn_rk4(workdir, n=12, t_fin_fs=0.3, it_res=5), workdir, 30)
    assert np.abs(ctx.get_state() - o.get("P0")).max() < RHO_TOL


@pytest.mark.parametrize("kind", ["hbn_rk4", "hbn_coulomb_ab4", "wannier8_rk4", "batch_fp64", "batch_mixed"])
def test_zero_field_keeps_the_initial_state(workdir, kind):
    """Invariants with no field (E = 0 at every step): the initial state is
    stationary (the Coulomb run starts in its own equilibrium, whose
    coefficients are subtracted), so the trace check and the currents keep
    their initial values to rounding, in the single solve and in FP64 and mixed
    batches. (The ground state's currents are those of the stencil gradient
    of H(k), not exactly zero: 5.7e-4 for the 12 x 12 Wannier model in the
    oracle too; a mixed batch takes the populations from FP32 eigenvectors,
    so its trace check starts near 1e-9.)"""
    d = f"{workdir}/{kind}"
    if kind == "hbn_coulomb_ab4":
        path = W.hbn_coulomb(d, n=24, field=0.0, t_fin_fs=0.5, it_res=10)
    elif kind.startswith("wannier") or kind.startswith("batch"):
        path = W.wannier(d, n=12, field=0.0, t_fin_fs=0.5, it_res=10)
    else:
        path = W.hbn_rk4(d, n=24, field=0.0, t_fin_fs=0.5, it_res=10)
    pb = E.Problem(E.parse_input(path), d)
    rho0 = pb.get("P0")
    if kind.startswith("batch"):
        prec = abi.EDUS_PREC_FP64 if kind == "batch_fp64" else abi.EDUS_PREC_MIXED
        b = E.Batch(precision=prec, chunk_steps=8)
        s = b.add(pb)
        for _ in range(1000):
            if b.poll(s)[0] == abi.EDUS_INST_DONE:
                break
            b.advance(8)
        rho, log = b.get_state(s), b.obs(s)
    else:
        ctx = E.Context(pb)
        ctx.run()
        rho, log = ctx.get_state(), ctx.obs()
    assert len(log) > 3
    assert np.abs(rho - rho0).max() < 1e-13
    tr = np.array([x["trace_dev"] for x in log])
    assert np.abs(tr - tr[0]).max() < 1e-13 and abs(tr[0]) < 1e-8
    J1 = np.array([x["J1"] for x in log])
    # relative to the initial current, over the k sum's absolute rounding floor
    assert np.abs(J1 - J1[0]).max() <= 1e-12 * np.abs(J1[0]).max() + 1e-17
