"""The CPU oracle against the reference program's own outputs.

The fixtures (tests/golden/ref_<case>.npz) are Output/*.txt of the reference
itself, compiled from its sources (tests/golden/make_ref_fixtures.py). The
reference parses each input with its own Read_Input, so these tests also pin
the product's input parser, whose edus_params the oracle runs on: a parse that
differs from the reference's shows up as a different time series.
"""
import numpy as np
import pytest

import edus_b200 as E
import ref_fixtures as RF
from oracle_lib import Oracle

# cases the oracle finishes in seconds; the configuration-sized ones run against the GPU path
SMALL = ["hbn24_rk4", "hbn24_coulomb_ab4", "hbn24_coulomb_diag_ab4", "hbn24_ab2", "hbn24_rk4_dyn", "hbn24_taylor6_dyn",
         "wannier8_16_rk4", "wannier16_24_rk4", "hbn24_coulomb_edia", "hbn12_snapshots", "crystal12_2band",
         "crystal10_3band", "hbn18x24_rk4", "hbn18x24_coulomb_ab4", "wannier8_12x20_rk4", "hbn24_gauss_rk4",
         "hbn24_pw_rk4", "hbn24_two_pumps_rk4", "hbn24_decoherence_rk4", "hbn24_ab1", "hbn24_ab3",
         "hbn24_taylor4", "hbn24_coulomb_rk4"] + sorted(RF.TB_MODELS)

# J2 of the diagonal-basis run (~7e-9) sits at the FP64 floor of its k sum after two rotations by U;
# the 0.3 fs band-dispersion run ends as the pulse starts, so its currents (J2 ~3e-13) are
# summation noise, compared absolutely (the case pins the per-k Edia files)
J2_ABS = {"hbn24_coulomb_diag_ab4": 1e-16, "hbn24_coulomb_edia": 1e-17}
# RK4 with adaptive dt divides by a population change of ~1e-9 to set each step: the reference
# itself, run with 4, 6 and 8 OpenMP threads, spreads by 1.5e-10 relative L2 in J1
J1_TOL = {"hbn24_coulomb_edia": 1e-9, "hbn24_rk4_dyn": 2e-10}


@pytest.mark.parametrize("name", sorted(RF.CASES))
def test_fixture_inputs_regenerate(name, workdir):
    RF.write_input(name, workdir)


# the tight-binding models' runs are short: J2 of the weakly driven ones is summation noise
# (~1e-18), compared absolutely; the currents of Graphene_costD, Graphene_symmetricD and
# Vampa2015 stay near 1e-11 and agree to the k sum's absolute floor (2e-18, as the others)
TB_J2_ABS = 1e-17


@pytest.mark.parametrize("name", SMALL)
def test_oracle_matches_reference_run(name, workdir):
    path = RF.write_input(name, workdir)
    o = Oracle(E.parse_input(path), workdir)
    log = o.run()
    tb = name in RF.TB_MODELS
    RF.compare_log(log, RF.load(name), j1_tol=J1_TOL.get(name, RF.J1_TOL),
                   j2_abs=TB_J2_ABS if tb else J2_ABS.get(name, 0.0), j1_abs=RF.J1_ABS_FLOOR if tb else 0.0)


def test_oracle_band_dispersion_files_match_reference(workdir):
    """Print_new_band_dispersion: the eigenvalues of the renormalised H at each
    snapshot (Output/Edia_<m>.txt of the reference) against the oracle's."""
    name = "hbn24_coulomb_edia"
    fx = RF.load(name)
    p = E.parse_input(RF.write_input(name, workdir))
    o = Oracle(p, workdir)
    info = o.info
    sched = RF.snapshot_schedule(info.t_start, p.dt, info.nsteps - 1, p.it_resolution, p.print_start, p.print_end,
                                 p.print_step)
    files = sorted(k for k in fx.files if k.startswith("file:Edia_"))
    assert len(files) == len(sched) == 2
    TIME_AU_FS = 0.02418884326505
    np.testing.assert_allclose(RF.per_k_file(fx, "t_Ek.txt").ravel(), [t * TIME_AU_FS for _, t in sched], rtol=1e-5)
    done = 0
    for m, (it, _) in enumerate(sched):
        o.run(it - done)
        done = it
        want = RF.per_k_file(fx, f"Edia_{m}.txt")
        got = np.linalg.eigvalsh(o.get("Hr"))
        assert got.shape == want.shape
        # the file prints 6 significant digits
        assert np.all(np.abs(got - want) <= 5e-6 * np.abs(want) + 1e-12), m


def test_shim_build_recipe_names_the_reference_sources():
    """oracle/Makefile compiles the reference's main_MPI.cpp where it lies, with
    the two shim headers, into oracle/_ref/ (git-ignored)."""
    import os

    from conftest import ROOT

    mk = open(os.path.join(ROOT, "oracle", "Makefile")).read()
    assert "$(REFERENCE)/main_MPI.cpp" in mk and "-I ref_shim" in mk
    ign = open(os.path.join(ROOT, ".gitignore")).read().split()
    assert "oracle/_ref/" in ign
    for f in ("mpi.h", "armadillo"):
        assert os.path.exists(os.path.join(ROOT, "oracle", "ref_shim", f))


def _vg_case(workdir, n):
    import os

    from edus_b200 import workloads as W

    os.makedirs(workdir, exist_ok=True)
    W.write_wannier_tb(os.path.join(workdir, "W2_tb.dat"), nw=2, nside=3)
    return W.wannier(workdir, nw=2, nside=3, name="W2", n=n, t_fin_fs=4.0, it_res=5, field=0.2, write_model=False)


def test_velocity_gauge_keyword_is_parsed(workdir):
    path = _vg_case(workdir, 8)
    txt = open(path).read().replace("Wannier\n", "Wannier\nvelocity_gauge\n")
    open(path, "w").write(txt)
    assert E.parse_input(path).velocity_gauge == 1


def test_oracle_velocity_gauge_converges_to_length_gauge(workdir):
    """The velocity-gauge restatement (rho'(k) = rho(k + A), H and D at k + A,
    no k-gradient term) and the reference's length gauge describe the same
    dynamics: their J1 differ by the length gauge's finite-difference
    k-gradient error, which falls by more than 8x per grid doubling on a
    nearest-neighbour model (14.5x and 15.5x measured, 32 -> 64 -> 128)."""
    diffs = []
    for n in (32, 64):
        d = f"{workdir}/n{n}"
        p = E.parse_input(_vg_case(d, n))
        lg = Oracle(p, d).run()
        p.velocity_gauge = 1
        o = Oracle(p, d)
        vg = o.run()
        assert max(abs(x["trace_dev"]) for x in vg) < 1e-12
        diffs.append(RF.rel_l2([x["J1"] for x in vg], [x["J1"] for x in lg]))
    assert diffs[0] < 2e-2 and diffs[1] < diffs[0] / 8, diffs
