"""Host problem setup: the product's grid / stencil / model tables against the
oracle's independent restatement and against the reference's own printouts
(Test_matrices.txt and the shell table of output.log)."""
import os

import numpy as np
import pytest

import edus_b200 as E
from edus_b200 import workloads as W
from conftest import GOLDEN, GOLDEN_INPUT
from oracle_lib import Oracle


def compare_setup(p, wd):
    pb = E.Problem(p, wd)
    o = Oracle(p, wd)
    assert pb.info.nnb == o.info.nnb and pb.info.nshell == o.info.nshell and pb.info.nsteps == o.info.nsteps
    assert np.array_equal(pb.get("nbr"), o.get("nbr"))
    assert np.array_equal(pb.get("kpt"), o.get("kpt"))
    # a shell whose exact weight is 0 (square lattice diagonals) comes out as
    # rounding noise of either least-squares solver: compare against the largest weight
    wo = o.get("weights")
    np.testing.assert_allclose(pb.get("weights"), wo, rtol=0, atol=1e-13 * np.abs(wo).max())
    np.testing.assert_allclose(pb.get("bvec"), o.get("bvec"), rtol=0, atol=1e-15)
    for name in ["H", "U", "D", "P0"]:
        a, b = pb.get(name), o.get(name)
        assert np.abs(a - b).max() <= 1e-14 * max(1.0, np.abs(b).max()), name
    if p.current:
        a, b = pb.get("GE"), o.get("GE")
        assert np.abs(a - b).max() <= 1e-12 * max(1.0, np.abs(b).max())
    return pb, o


def test_golden_setup_matches_oracle():
    p = E.parse_input(GOLDEN_INPUT)
    pb, o = compare_setup(p, ".")
    assert pb.info.nk == 4900 and pb.info.nnb == 12 and pb.info.nsteps == 16591 and pb.info.nprint == 3319
    assert pb.info.n_diss == 5  # main_MPI.cpp log: "n_diss_terms 5"


def test_golden_shells_match_reference_log():
    # output.log:14-31: two shells of six vectors, |b| = 0.02194 and 0.03800 bohr^-1
    p = E.parse_input(GOLDEN_INPUT)
    pb = E.Problem(p)
    b = pb.get("bvec")
    nrm = np.sort(np.unique(np.round(np.linalg.norm(b, axis=1), 5)))
    np.testing.assert_allclose(nrm, [0.02194, 0.03800], atol=1e-5)
    assert np.sum(np.isclose(np.linalg.norm(b, axis=1), 0.02194, atol=1e-5)) == 6


def test_golden_kgrid_file_byte_exact(tmp_path):
    """Output/k_grid.txt of the shipped AB5 run (headers/Observables_MPI.h:492-550),
    byte for byte: the k grid in the reference's order and stream format."""
    import hashlib
    import json

    ref = json.load(open(os.path.join(GOLDEN, "ab5_kgrid.json")))
    pb = E.Problem(E.parse_input(GOLDEN_INPUT))
    out = tmp_path / "Output"
    pb.write_kgrid(str(out))
    raw = (out / "k_grid.txt").read_bytes()
    lines = raw.decode().splitlines()
    assert lines[:3] == ref["head"] and lines[-3:] == ref["tail"] and len(lines) == ref["lines"]
    assert len(raw) == ref["bytes"] and hashlib.sha256(raw).hexdigest() == ref["sha256"]


def test_kpt_listing(tmp_path):
    """kpt.txt (headers/InitParameters.h:17-39): index, grid indices and crystal
    coordinates per k point, the coordinates as k_grid.txt prints them."""
    import json

    pb = E.Problem(E.parse_input(GOLDEN_INPUT))
    pb.write_kpt(str(tmp_path))
    lines = (tmp_path / "kpt.txt").read_text().splitlines()
    assert len(lines) == 4900
    assert lines[0] == "0 0 0 0 0 -0.5 -0.5" and lines[71].startswith("71 0 1 1 ")
    ref = json.load(open(os.path.join(GOLDEN, "ab5_kgrid.json")))
    assert [" ".join(l.split()[4:]) for l in lines[:3]] == ref["head"]
    assert [" ".join(l.split()[4:]) for l in lines[-3:]] == ref["tail"]


def test_test_matrices_file_byte_exact(tmp_path):
    """Test_matrices.txt of the shipped AB5 run (Source_Main/test_matrix_k.cpp),
    byte for byte, rounding residues of U H U^dagger included."""
    pb = E.Problem(E.parse_input(GOLDEN_INPUT))
    pb.write_test_matrices(str(tmp_path))
    got = (tmp_path / "Test_matrices.txt").read_bytes()
    ref = open(os.path.join(GOLDEN, "ab5_test_matrices.txt"), "rb").read()
    assert got == ref


def test_test_matrices_known_answer():
    """Source_Main/test_matrix_k.cpp prints H, U, dx, dy at k = (0, 0.3, 0.1)."""
    p = E.parse_input(GOLDEN_INPUT)
    pb = E.Problem(p)
    H, U, D = pb.model_hud([0.0, 0.3, 0.1])
    ref = np.load(os.path.join(GOLDEN, "test_matrices.npz"))
    np.testing.assert_allclose(H, ref["Energy"], atol=5e-6)
    np.testing.assert_allclose(U, ref["Unitary"], atol=5e-6)
    np.testing.assert_allclose(D[:, :, 0], ref["dx"], atol=5e-6)
    np.testing.assert_allclose(D[:, :, 1], ref["dy"], atol=5e-6)
    np.testing.assert_allclose(U @ U.conj().T, np.eye(3), atol=1e-14)


def test_coulomb_setup_matches_oracle(workdir):
    p = E.parse_input(W.hbn_coulomb(workdir, n=24, t_fin_fs=0.5))
    compare_setup(p, workdir)


def test_wannier_setup_matches_oracle(workdir):
    p = E.parse_input(W.wannier(workdir, n=16, t_fin_fs=0.2))
    pb, _ = compare_setup(p, workdir)
    assert pb.info.nrpts == 121
    HR = pb.get("HR")
    Rv = pb.get("Rvec")
    # hermitised model: H(-R) = H(R)^dagger
    idx = {tuple(r): i for i, r in enumerate(Rv.astype(int))}
    for i, r in enumerate(Rv.astype(int)):
        j = idx[(0, -r[1], -r[2])]
        np.testing.assert_allclose(HR[:, :, j], HR[:, :, i].conj().T, atol=1e-15)


def test_square_lattice_stencil_needs_three_shells(workdir):
    # a square grid cannot satisfy the 4th-moment rows with the nearest shell alone
    p = E.parse_input(W.wannier(workdir, n=16, t_fin_fs=0.2))
    pb = E.Problem(p, workdir)
    assert pb.info.nshell == 3 and pb.info.nnb == 12


def test_problem_rejects_bad_input(workdir):
    p = E.parse_input(W.hbn_rk4(workdir, n=12, t_fin_fs=0.1))
    p.dt = -1
    with pytest.raises(E.EdusError):
        E.Problem(p, workdir)
    p = E.parse_input(W.hbn_rk4(workdir, n=12, t_fin_fs=0.1))
    p.tb_type = b"GaSe_kp2"
    with pytest.raises(E.EdusError) as ei:
        E.Problem(p, workdir)
    assert ei.value.code == E.abi.EDUS_EUNSUPPORTED


def test_deferred_problem_is_refused_by_single_solve_contexts(workdir):
    p = E.parse_input(W.wannier(workdir, n=8, t_fin_fs=0.1))
    pb = E.Problem(p, workdir, defer_model=True)
    assert pb.info.nrpts == 121
    with pytest.raises(E.EdusError) as ei:
        E.Context(pb)
    assert ei.value.code == E.abi.EDUS_EUNSUPPORTED


def _listed_grid_input(workdir, order):
    path = W.hbn_rk4(workdir, n=12, t_fin_fs=0.2, it_res=5)
    dk = 1.0 / 12  # the grid's own arithmetic (headers/InitParameters.h:31-35)
    pts = [(0.0, -0.5 + dk * i, -0.5 + dk * j) for i in range(12) for j in range(12)]
    pts = [pts[q] for q in order]
    lines = "".join(f"{a!r} {b!r} {c!r}\n" for a, b, c in pts)
    txt = open(path).read().replace("nkpt{\n1 12 12\n}", "nkpt read{\n1 12 12\n" + lines + "}")
    open(path, "w").write(txt)
    return path


def test_listed_grid_in_grid_order_equals_the_grid(workdir):
    """nkpt read (headers/ReadInput.h:420-440) with the Monkhorst-Pack points in
    grid order: the same tables as the generated grid."""
    ref = E.Problem(E.parse_input(W.hbn_rk4(f"{workdir}/g", n=12, t_fin_fs=0.2, it_res=5)), f"{workdir}/g")
    p = E.parse_input(_listed_grid_input(f"{workdir}/l", list(range(144))))
    assert p.kpt_read == 1
    pb = E.Problem(p, f"{workdir}/l")
    for name in ["kpt", "nbr", "weights", "bvec", "H", "U", "D", "P0"]:
        assert np.array_equal(pb.get(name), ref.get(name)), name


def test_listed_grid_in_any_order_matches_oracle(workdir):
    """A shuffled list: neighbours found by coordinates (the first match in list
    order, headers/CalculateWeigths.h:140-226), against the oracle's search."""
    order = list(np.random.default_rng(5).permutation(144))
    p = E.parse_input(_listed_grid_input(workdir, order))
    pb, o = compare_setup(p, workdir)
    kpt = pb.get("kpt")
    assert np.array_equal(kpt[0], [0.0, -0.5 + (1.0 / 12) * (order[0] // 12), -0.5 + (1.0 / 12) * (order[0] % 12)])
    nbr = pb.get("nbr")
    assert sorted(set(nbr.ravel().tolist())) == list(range(144))


def test_listed_grid_in_any_order_propagates_as_the_grid(workdir):
    """The oracle's time loop on the shuffled list and on the grid: the same
    currents and populations (sums over k do not depend on the order beyond
    rounding)."""
    order = list(np.random.default_rng(9).permutation(144))
    pl = E.parse_input(_listed_grid_input(f"{workdir}/l", order))
    pg = E.parse_input(W.hbn_rk4(f"{workdir}/g", n=12, t_fin_fs=0.2, it_res=5))
    ll = Oracle(pl, f"{workdir}/l").run(40)
    lg = Oracle(pg, f"{workdir}/g").run(40)
    J1l, J1g = np.array([x["J1"] for x in ll]), np.array([x["J1"] for x in lg])
    # (the k sums run in another order: rounding at the 1e-18 floor of the early, near-zero currents)
    assert np.abs(J1l - J1g).max() <= 1e-12 * np.abs(J1g).max() + 1e-17
    assert np.abs(np.array([x["pop"] for x in ll]) - np.array([x["pop"] for x in lg])).max() < 1e-14


@pytest.mark.parametrize("model,nb", [("CoreBN_Nedge", 3), ("CoreBN_Bedge", 3), ("Graphene", 2), ("CoreGraphene", 4),
                                      ("Graphene_costD", 4), ("Graphene_symmetricD", 4), ("GrapheneZurron", 2),
                                      ("BN1b", 1), ("Vampa2015", 2), ("GeS", 2), ("GeS_HSE06", 2),
                                      ("DLGraphene", 4)])
def test_more_tight_binding_models_match_oracle(workdir, model, nb):
    """Tight-binding models with their closed-form H, U and dipoles
    (headers/TightBinding.h:43-1421): the set-up tables against the oracle's,
    U unitary and U H U^dagger diagonal (the reference's Test_matrices check)."""
    # (DLGraphene's closed-form eigenvectors divide by zero where f = 0, at the K
    # points a grid of 3m points holds, in the reference as here)
    path = W.hbn_rk4(workdir, n=10 if model == "DLGraphene" else 12, t_fin_fs=0.2, it_res=5)
    txt = open(path).read()
    txt = txt.replace(txt.splitlines()[3] + "\n", f"tightbinding {model}\n")
    open(path, "w").write(txt)
    p = E.parse_input(path)
    pb, o = compare_setup(p, workdir)
    assert pb.info.ncv == nb
    H, U = pb.get("H"), pb.get("U")
    UU = np.einsum("kij,klj->kil", U, U.conj())
    assert np.abs(UU - np.eye(nb)).max() < 1e-12
    E2 = np.einsum("kim,kmn,kjn->kij", U, H, U.conj())
    off = E2 - np.einsum("kii->ki", E2)[:, :, None] * np.eye(nb)
    assert np.abs(off).max() < 1e-12 * max(1.0, np.abs(H).max())


@pytest.mark.parametrize("norb", [2, 3])
def test_crystal_setup_matches_oracle(workdir, norb):
    """Crystal interface (headers/Crystal_interface.h, headers/Interpolation.h):
    the lattice, H, U, D and rho0 from the interpolated files against the
    oracle's; a file with more orbitals than bands uses the first ones."""
    p = E.parse_input(W.crystal(workdir, nb=(1, 1), norb=norb, nkf=13, n=12))
    assert p.mode == E.abi.EDUS_MODE_CRYSTAL
    pb, o = compare_setup(p, workdir)
    H, U = pb.get("H"), pb.get("U")
    UU = np.einsum("kij,klj->kil", U, U.conj())
    assert np.abs(UU - np.eye(2)).max() < 1e-12
    E2 = np.einsum("kim,kmn,kjn->kij", U, H, U.conj())
    assert np.abs(E2[:, 0, 1]).max() < 1e-12 and np.all(E2[:, 0, 0].real <= E2[:, 1, 1].real)
    D = pb.get("D")
    assert np.abs(D[..., 0]).max() == 0.0
    assert np.abs(D[:, [0, 1], [0, 1], :].imag).max() == 0.0
    # Hermitian dipoles: the crystal model keeps them as read (no symmetrisation)
    assert np.abs(D[:, 0, 1, 1:] - D[:, 1, 0, 1:].conj()).max() == 0.0
    assert np.abs(D[:, 0, 1, 1:].imag).max() > 1e-3


def test_crystal_model_reproduces_the_file_samples(workdir):
    """The bicubic fit passes through the samples: at the file's grid points
    gHUD returns the file's H and connections (upper triangle conjugated, D in
    the order z, x, y, real diagonals), and the lattice is the file's."""
    path = W.crystal(workdir, nb=(1, 2), norb=3, nkf=11, n=10)
    model, grid, a, b = W.write_crystal_files(workdir, nb=3, norb=3, nkf=11)
    pb = E.Problem(E.parse_input(path), workdir)
    for i1 in [0, 3, 7, 10]:
        for i2 in [0, 5, 9, 10]:
            k1, k2 = grid[i1], grid[i2]
            H, U, D = pb.model_hud([0.0, k1, k2])
            Hf, Dx, Dy = model(k1, k2)
            np.testing.assert_allclose(H, Hf, rtol=0, atol=1e-13)
            np.testing.assert_allclose(D[..., 1], Dx - 1j * np.diag(Dx.diagonal().imag), rtol=0, atol=1e-13)
            np.testing.assert_allclose(D[..., 2], Dy - 1j * np.diag(Dy.diagonal().imag), rtol=0, atol=1e-13)
            assert np.abs(D[..., 0]).max() == 0.0
    kc = pb.get("kpt")
    assert kc.shape == (100, 3)


def test_oracle_runs_a_crystal_problem(workdir):
    """The oracle's RHS reads the full dipole matrix, so it runs Crystal inputs
    with their Hermitian dipoles: populations stay normalised and the state
    responds to the pump (the checker a device path will be held to)."""
    p = E.parse_input(W.crystal(workdir, nb=(1, 1), nkf=9, n=8, field=2.0, duration=4.0, t_fin_fs=0.6, it_res=10))
    log = Oracle(p, workdir).run(60)
    pops = np.array([x["pop"] for x in log])
    # holes in the valence band = electrons in the conduction band
    assert pops[-1, 1] > 1e-8
    assert np.abs(pops[:, 0] - pops[:, 1]).max() < 1e-6 * pops[-1, 1]
    assert max(abs(x["trace_dev"]) for x in log) < 1e-12
    J1 = np.array([x["J1"] for x in log])
    assert np.abs(J1[-1]).max() > 0


def test_crystal_files_missing_or_short_are_errors(workdir):
    """A Crystal input without its files, or with fewer orbitals than bands,
    is an error code (the reference would read past its arrays)."""
    path = W.crystal(workdir, nb=(1, 1), norb=2, nkf=7, n=6)
    os.remove(os.path.join(workdir, "bc_betabetap_imag.dat"))
    with pytest.raises(E.EdusError) as ei:
        E.Problem(E.parse_input(path), workdir)
    assert ei.value.code == E.abi.EDUS_EIO
    path = W.crystal(workdir, nb=(2, 1), norb=2, nkf=7, n=6)  # 2 orbitals in the files, 3 bands in the input
    with pytest.raises(E.EdusError) as ei:
        E.Problem(E.parse_input(path), workdir)
    assert ei.value.code == E.abi.EDUS_EINVAL
