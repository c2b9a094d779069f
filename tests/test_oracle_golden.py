"""Pin of the CPU oracle against the reference's shipped known answer: the full
Adams–Bashforth 5 run of example/Adams–Bashforth ODE Solver example/AB5_...
(70x70 Haldane_CoreBN_Nedge, corehole decoherence, XUV probe, 16591 steps).
Outputs are compared at their printed precision (J1/J2 15 digits, Losses 16,
EF/TransientAbs 8); J2 is a cancelling sum whose noise floor is ~1e-18."""
import os

import numpy as np
import pytest

import edus_b200 as E
from conftest import GOLDEN, GOLDEN_INPUT
from oracle_lib import Oracle

TIME_AU_FS = 0.02418884326505


@pytest.fixture(scope="module")
def golden_run():
    p = E.parse_input(GOLDEN_INPUT)
    o = Oracle(p)
    log = o.run()
    return log, np.load(os.path.join(GOLDEN, "ab5_golden.npz"))


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_oracle_reproduces_golden_currents(golden_run):
    log, G = golden_run
    rows = G["rows"]
    assert len(log) == int(G["nrows"]) == 3319
    t = np.array([log[i]["t"] * TIME_AU_FS for i in rows])
    np.testing.assert_allclose(t, G["J1"][:, 0], atol=1e-7)
    J1 = np.array([log[i]["J1"] for i in rows])
    J1r = G["J1"][:, 1::2] + 1j * G["J1"][:, 2::2]
    assert rel(J1, J1r) < 1e-12
    J2 = np.array([log[i]["J2"] for i in rows])
    J2r = G["J2"][:, 1:]
    assert np.abs(J2 - J2r).max() < 1e-10 * np.abs(J2r).max()


def test_oracle_reproduces_golden_populations(golden_run):
    log, G = golden_run
    rows = G["rows"]
    pop = np.array([log[i]["pop"] for i in rows])
    Lr = G["Losses"][:, 1:4]
    assert np.abs(pop - Lr).max() < 2e-15
    assert rel(pop[:, 2], Lr[:, 2]) < 1e-11


def test_oracle_reproduces_golden_field_and_tabs(golden_run):
    log, G = golden_run
    rows = G["rows"]
    ef = np.array([log[i]["EF_pump"] for i in rows])
    # 8 significant digits in EF.txt: half a unit of the last digit is 5e-8 relative
    assert np.abs(ef - G["EF"][:, 1:]).max() < 5e-8 * np.abs(G["EF"][:, 1:]).max()
    ta = np.array([list(log[i]["EF_probe"]) + [v for c in log[i]["tabs"] for v in (c.real, c.imag)] for i in rows])
    ref = G["TAbs"][:, 1:]
    scale = np.maximum(np.abs(ref).max(axis=0), 1e-300)
    assert (np.abs(ta - ref).max(axis=0) <= 1e-7 * scale + 1e-30).all()


def test_oracle_trace_is_conserved(golden_run):
    log, _ = golden_run
    assert max(abs(x["trace_dev"]) for x in log) < 1e-11


@pytest.mark.parametrize("diag", [0, 1])
def test_oracle_coulomb_equilibrium_is_stationary(workdir, diag):
    """With no field, the Coulomb run starts in its own equilibrium in either
    basis (main_MPI.cpp:276-337: the coefficients of the initial state, or in
    the diagonal basis of the filled bands, are subtracted), so rho stays put
    and the renormalised H stays Hermitian."""
    from edus_b200 import workloads as W

    path = W.hbn_coulomb(workdir, n=12, field=0.0, t_fin_fs=0.1, it_res=5)
    txt = open(path).read()
    if diag:
        txt = txt.replace("Rytova_Keldysh\n", "Rytova_Keldysh\nCoulomb_diag_basis\n")
    open(path, "w").write(txt)
    p = E.parse_input(path)
    o = Oracle(p, workdir)
    rho0 = o.get("P0")
    log = o.run(15)
    assert np.abs(o.get("P0") - rho0).max() < 1e-13
    hk = o.coulomb_hk(o.get("P0"))
    assert np.array_equal(hk, np.conj(np.transpose(hk, (0, 2, 1))))
    assert abs(log[-1]["trace_dev"]) < 1e-12


def test_oracle_polarisation_is_tr_d_rho(workdir):
    """The polarisation record (1/Nk) sum_k Tr(D_x rho(k)) (an output the
    reference does not have) against numpy on the oracle's own state and dipole
    tables, at the start and after 30 RK4 steps inside the pulse; the dipoles
    of the reference's models are real symmetric and rho is Hermitian, so the
    trace is real."""
    from edus_b200 import workloads as W

    p = E.parse_input(W.hbn_rk4(workdir, n=12, t_fin_fs=1.0, it_res=10, field=0.5))
    o = Oracle(p, workdir)
    D = o.get("D")  # [k][i][j][x]
    for steps in (0, 30):
        if steps:
            o.run(steps)
        P = o.get("P0")
        rec = o.observables(P)
        want = np.einsum("kijx,kij->x", D, P) / P.shape[0]
        np.testing.assert_allclose(rec["pol"], want, rtol=1e-12, atol=1e-15)
        assert np.abs(np.imag(rec["pol"])).max() < 1e-14
