"""The sm_100a path against the reference program's own outputs, at the
configurations' own sizes.

Fixtures: tests/golden/ref_<case>.npz, the Output/*.txt series of the
reference itself (anpicon/EDUS compiled from its sources, one MPI rank; see
tests/golden/make_ref_fixtures.py), on the same input text:

  cfg0_hbn60_rk4           hBN 60x60, RK4, 30 fs (3021 steps)
  cfg1_hbn120_coulomb_ab4  hBN 120x120 + Rytova-Keldysh mean field (shipped Ncut=20
                           tables), AB4 from the reference's zero derivative
                           history, 30 fs (6043 steps)
  cfg2_wannier8_96_rk4     8-band Wannier model 96x96, RK4, 40 fs (4001 steps)
  and small cases of the other solvers and options.

Tolerances (written per test): FP64 paths J1 <= 5e-12 relative L2 over t
(J1 is a k sum that cancels to ~1e-6 of its terms; the reference itself run
with 4 and 8 OpenMP threads differs by 1.1e-12 on the short runs),
populations <= 1e-13 absolute (Losses.txt prints 16 digits), J2 <= 1e-9 of
its largest value (a k sum that cancels to ~1e-8). Runs with the Coulomb mean
field are compared with the closest of the reference's own outcomes (it
switches its screening on when noise-level populations exceed 1e-20, so its
runs split into two results ~3e-8 apart). Mixed precision (FP32 H, D and commutator, FP64 state): J1 <= 1e-6
relative L2 against the reference; the populations' and rho's errors are
asserted against the bounds stated beside each test.
"""
import math
import os

import numpy as np
import pytest

import edus_b200 as E
import ref_fixtures as RF
from edus_b200 import abi
from edus_b200 import workloads as W
from oracle_lib import Oracle

pytestmark = pytest.mark.gpu

SERIES_CASES = ["cfg0_hbn60_rk4", "cfg1_hbn120_coulomb_ab4", "cfg2_wannier8_96_rk4", "hbn24_rk4", "hbn24_coulomb_ab4",
                "hbn24_coulomb_diag_ab4", "hbn24_ab2", "hbn24_rk4_dyn", "hbn24_taylor6_dyn", "wannier8_16_rk4",
                "wannier16_24_rk4", "crystal12_2band", "crystal10_3band", "hbn18x24_rk4", "hbn18x24_coulomb_ab4",
                "wannier8_12x20_rk4", "hbn24_gauss_rk4", "hbn24_pw_rk4", "hbn24_two_pumps_rk4",
                "hbn24_decoherence_rk4", "hbn24_ab1", "hbn24_ab3", "hbn24_taylor4",
                "hbn24_coulomb_rk4"] + sorted(RF.TB_MODELS)
# per-case tolerances, measured on the reference itself (tests/test_reference_pins.py): J2 of the
# diagonal-basis run sits at its k sum's FP64 floor. RK4 with adaptive dt sets each step from a
# population change of ~1e-9, so rounding moves the time grid: the reference itself spreads by
# 1.5e-10 in J1 between runs with 4, 6 and 8 threads, the GPU sits 5.3e-10 from it.
J2_ABS = {"hbn24_coulomb_diag_ab4": 1e-16, "hbn24_rk4_dyn": 1e-16}
J1_TOL = {"hbn24_rk4_dyn": 1e-9}
# the 8-band runs' populations sum 4000 RK4 steps of O(1) valence terms: 1.5e-13 measured at 40 fs
POP_ABS = {"cfg2_wannier8_96_rk4": 5e-13}
MIXED_J1 = 1e-6


def _drain(b, slots, chunk=64):
    for _ in range(1000000):
        if all(b.poll(s)[0] == abi.EDUS_INST_DONE for s in slots):
            return
        b.advance(chunk)
    raise AssertionError("batch did not finish")


# the other tight-binding models' short runs: J2 of the weakly driven ones is summation noise,
# and three of them keep their currents near 1e-11, where J1 is compared absolutely
TB_J2_ABS, TB_J1_ABS = 1e-17, 1e-16


@pytest.mark.parametrize("name", SERIES_CASES)
def test_single_solve_matches_reference_run(name, workdir):
    path = RF.write_input(name, workdir)
    ctx = E.Context(E.Problem(E.parse_input(path), workdir))
    ctx.run()
    tb = name in RF.TB_MODELS
    RF.compare_log(ctx.obs(), RF.load(name), j1_tol=J1_TOL.get(name, RF.J1_TOL), pop_abs=POP_ABS.get(name, 1e-13),
                   j2_abs=TB_J2_ABS if tb else J2_ABS.get(name, 0.0), j1_abs=TB_J1_ABS if tb else 0.0)


def test_crystal_runs_in_contexts_and_batches_refuse_it(workdir):
    """The Crystal interface keeps Hermitian dipoles: single-solve contexts run it
    (the lower dipole entries read as conj(D_ij)); the batch kernels read one
    symmetric dipole plane per band pair and refuse it."""
    nm = "crystal10_3band"
    p = E.parse_input(RF.write_input(nm, workdir))
    pb = E.Problem(p, workdir)
    ctx = E.Context(pb)
    ctx.step(40)
    o = Oracle(p, workdir)
    o.run(40)
    assert np.abs(ctx.get_state() - o.get("P0")).max() < 1e-13
    b = E.Batch(precision=abi.EDUS_PREC_FP64)
    with pytest.raises(E.EdusError) as ei:
        b.add(pb)
    assert ei.value.code == abi.EDUS_EUNSUPPORTED


def test_config1_rk4_startup_window_matches_oracle(workdir):
    """The bench's configuration-1 solve (AB4 with the RK4 start-up this build
    adds; the reference has no start-up) on its 120x120 grid: 640 steps, 42
    field-free and 598 inside the pulse, against the oracle's restatement.

    The screening constant is zeroed here: its correction switches on when the
    mean conduction population exceeds 1e-20 (headers/RungeKutta.h:77), and
    before the pulse that population is rounding noise whose sign differs
    between the oracle (+3e-19 at t = -0.11 fs) and the GPU (-2e-18), which
    moves rho by 4.6e-10 from the pulse onset. With the correction on, the
    GPU's full configuration-1 run is held to the reference's own outcome
    (test_single_solve_matches_reference_run)."""
    path = W.hbn_coulomb(workdir, n=120, it_res=10)
    import glob

    for f in glob.glob(f"{workdir}/Output/Coulomb/Screen_const_*.txt"):
        rows = len(open(f).read().split("\n")) - 1
        open(f, "w").write("".join("0 0\n" for _ in range(rows)))
    p = E.parse_input(path)
    ctx = E.Context(E.Problem(p, workdir))
    ctx.step(640)
    o = Oracle(p, workdir)
    lo = o.run(640)
    assert np.abs(ctx.get_state() - o.get("P0")).max() < 1e-13
    g = ctx.obs()
    assert len(g) == len(lo) == 64
    J1g, J1o = np.array([x["J1"] for x in g]), np.array([x["J1"] for x in lo])
    assert RF.rel_l2(J1g, J1o) < RF.J1_TOL
    assert np.abs(np.array([x["pop"] for x in g]) - np.array([x["pop"] for x in lo])).max() < 1e-14


def test_fp64_batch_matches_reference_runs(workdir):
    """FP64 batch instances (one batch: hBN 60x60 with its decoupled core band
    dropped, the 8-band 96x96 model built on the device, the 16-band model,
    and rectangular 18x24 hBN / 12x20 8-band grids) against the reference's
    output for the same inputs."""
    names = ["cfg0_hbn60_rk4", "cfg2_wannier8_96_rk4", "wannier16_24_rk4", "hbn18x24_rk4", "wannier8_12x20_rk4"]
    pbs = []
    for nm in names:
        d = f"{workdir}/{nm}"
        pb = E.Problem(E.parse_input(RF.write_input(nm, d)), d, defer_model=nm.startswith(("cfg2", "wannier")))
        if nm.startswith(("cfg0", "hbn")):
            pb.drop_decoupled_core()
        pbs.append(pb)
    b = E.Batch(precision=abi.EDUS_PREC_FP64)
    slots = [b.add(pb) for pb in pbs]
    _drain(b, slots)
    for nm, s in zip(names, slots):
        bands = (1, 2) if nm.startswith(("cfg0", "hbn")) else None
        RF.compare_log(b.obs(s), RF.load(nm), pop_abs=POP_ABS.get(nm, 1e-13), bands=bands)


def test_fp64_batch_runs_every_tight_binding_model_as_the_reference(workdir):
    """The reference's other tight-binding models (2, 3 and 4 bands, hexagonal,
    orthorhombic and rectangular-cell lattices) as instances of one FP64
    batch, against the reference's output for the same inputs."""
    names = sorted(RF.TB_MODELS)
    pbs = []
    for nm in names:
        d = f"{workdir}/{nm}"
        pbs.append(E.Problem(E.parse_input(RF.write_input(nm, d)), d))
    b = E.Batch(precision=abi.EDUS_PREC_FP64)
    slots = [b.add(pb) for pb in pbs]
    _drain(b, slots)
    for nm, s in zip(names, slots):
        RF.compare_log(b.obs(s), RF.load(nm), j2_abs=TB_J2_ABS, j1_abs=TB_J1_ABS)
    b.close()


def test_served_fp64_matches_reference_runs(workdir):
    """Requests through the server (FP64) against the reference's output."""
    names = ["cfg0_hbn60_rk4", "cfg2_wannier8_96_rk4", "hbn24_rk4", "wannier16_24_rk4"]
    s = E.Server(precision=abi.EDUS_PREC_FP64)
    ids = []
    for nm in names:
        d = f"{workdir}/{nm}"
        ids.append(s.submit(E.parse_input(RF.write_input(nm, d)), d))
    s.drain(600)
    for nm, rid in zip(names, ids):
        bands = (1, 2) if nm.startswith(("cfg0", "hbn")) else None
        RF.compare_log(s.obs(rid), RF.load(nm), pop_abs=POP_ABS.get(nm, 1e-13), bands=bands)
    s.close()


def test_mixed_batch_config2_within_1e6_of_reference(workdir):
    """Configuration 2 in mixed precision (batch, model built on the device with
    the tensor-core contraction): J1 <= 1e-6 relative L2 over the 40 fs against
    the reference's own output (2.9e-8 measured); populations within 1e-8
    absolute of the reference's (4.8e-9 measured; the conduction populations
    reach ~1e-2); rho within 2e-6 of the FP64 batch."""
    nm = "cfg2_wannier8_96_rk4"
    pb = E.Problem(E.parse_input(RF.write_input(nm, workdir)), workdir, defer_model=True)
    out = {}
    for prec in (abi.EDUS_PREC_MIXED, abi.EDUS_PREC_FP64):
        b = E.Batch(precision=prec)
        s = b.add(pb)
        _drain(b, [s])
        out[prec] = (b.obs(s), b.get_state(s))
        b.close()
    log, rho = out[abi.EDUS_PREC_MIXED]
    err = RF.compare_log(log, RF.load(nm), j1_tol=MIXED_J1, pop_abs=1e-8, j2_rel=1e-5)
    assert np.abs(rho - out[abi.EDUS_PREC_FP64][1]).max() < 2e-6, err


def _hardest_sweep_instances():
    """Of the seeded 256-instance sweep, per kind the instance with the largest
    field and the largest grid with the longest pulse (the largest errors)."""
    specs = W.sweep(256)
    pick = []
    for kind in ("hbn", "wannier"):
        ks = [(i, s) for i, s in enumerate(specs) if s["kind"] == kind]
        pick.append(max(ks, key=lambda x: x[1]["field"]))
        pick.append(max(ks, key=lambda x: x[1]["n"] * x[1]["n"] * x[1]["duration"]))
    return pick


def test_mixed_sweep_instances_within_1e6_of_fp64(workdir):
    """Configuration-3 instances (their own grids, fields and durations) in one
    mixed-precision batch against the plain FP64 single-solve path (held to the
    reference above): J1 <= 1e-6 relative L2; populations <= 1e-8 absolute;
    rho <= 2e-6 absolute."""
    pick = _hardest_sweep_instances()
    pbs, refs = [], []
    for i, spec in pick:
        d = f"{workdir}/s{i}"
        os.makedirs(d, exist_ok=True)
        if spec["kind"] == "wannier":
            W.write_wannier_tb(f"{d}/W8_tb.dat")
        p = E.parse_input(W.write_instance(d, spec))
        single = E.Problem(p, d)
        if spec["kind"] == "hbn":
            single.drop_decoupled_core()
        ctx = E.Context(single)
        ctx.run()
        refs.append((ctx.obs(), ctx.get_state()))
        ctx.close()
        pb = E.Problem(p, d, defer_model=spec["kind"] == "wannier")
        if spec["kind"] == "hbn":
            pb.drop_decoupled_core()
        pbs.append(pb)
    b = E.Batch(precision=abi.EDUS_PREC_MIXED)
    slots = [b.add(pb) for pb in pbs]
    _drain(b, slots)
    for (i, spec), s, (log, rho) in zip(pick, slots, refs):
        lb = b.obs(s)
        assert len(lb) == len(log)
        j1 = RF.rel_l2([x["J1"] for x in lb], [x["J1"] for x in log])
        pe = np.abs(np.array([x["pop"] for x in lb]) - np.array([x["pop"] for x in log])).max()
        re = np.abs(b.get_state(s) - rho).max()
        assert j1 <= MIXED_J1 and pe <= 1e-8 and re <= 2e-6, (i, spec, j1, pe, re)


def test_served_mixed_16band_within_1e6_of_fp64(workdir):
    """A configuration-4 16-band request (13x13 R vectors) served in mixed
    precision next to an 8-band one, against the plain FP64 single solve."""
    specs = [dict(kind="wannier", nw=16, nside=13, name="W16", n=48, field=0.8, phase=1.0, duration=30.0, it_res=10,
                  dt_fs=0.01),
             dict(kind="wannier", nw=8, nside=11, name="W8", n=64, field=0.8, phase=2.0, duration=20.0, it_res=10,
                  dt_fs=0.01)]
    s = E.Server(precision=abi.EDUS_PREC_MIXED)
    ids, refs = [], []
    for q, spec in enumerate(specs):
        d = f"{workdir}/r{q}"
        os.makedirs(d, exist_ok=True)
        W.write_wannier_tb(f"{d}/{spec['name']}_tb.dat", nw=spec["nw"], nside=spec["nside"])
        p = E.parse_input(W.write_instance(d, spec))
        ids.append(s.submit(p, d))
        ctx = E.Context(E.Problem(p, d))
        ctx.run()
        refs.append(ctx.obs())
        ctx.close()
    s.drain(600)
    for rid, log in zip(ids, refs):
        lb = s.obs(rid)
        assert len(lb) == len(log)
        j1 = RF.rel_l2([x["J1"] for x in lb], [x["J1"] for x in log])
        pe = np.abs(np.array([x["pop"] for x in lb]) - np.array([x["pop"] for x in log])).max()
        assert j1 <= MIXED_J1 and pe <= 1e-8, (j1, pe)
    s.close()
    assert math.isfinite(j1)


def test_batch_coulomb_instance_matches_oracle_and_reference(workdir):
    """A Coulomb instance in a mixed-precision batch beside non-Coulomb ones (it
    runs as its own FP64 context on its own stream): rho within 1e-13 of the
    oracle, J(t) against the reference's own outcomes, and bit for bit the
    single-solve result."""
    nm = "hbn24_coulomb_ab4"
    d = f"{workdir}/{nm}"
    p = E.parse_input(RF.write_input(nm, d))
    pb = E.Problem(p, d)
    others = []
    for q, (n, tf) in enumerate([(16, 0.8), (20, 0.5)]):
        dd = f"{workdir}/o{q}"
        o = E.Problem(E.parse_input(W.hbn_rk4(dd, n=n, t_fin_fs=tf, it_res=4)), dd)
        o.drop_decoupled_core()
        others.append(o)
    b = E.Batch(precision=abi.EDUS_PREC_MIXED, chunk_steps=8)
    s0 = b.add(others[0])
    sc = b.add(pb)
    b.advance(16)
    s1 = b.add(others[1])
    _drain(b, [s0, sc, s1], chunk=16)
    rho, log = b.get_state(sc), b.obs(sc)
    o = Oracle(p, d)
    o.run()
    assert np.abs(rho - o.get("P0")).max() < 1e-13
    RF.compare_log(log, RF.load(nm), pop_abs=1e-13)
    ctx = E.Context(pb)
    ctx.run()
    assert np.array_equal(rho, ctx.get_state())
    assert all(np.array_equal(x["J1"], y["J1"]) for x, y in zip(log, ctx.obs()))
    st = b.stats()
    assert st["done"] == 3
    b.close()


def test_batch_of_coulomb_instances_only_drains(workdir):
    """A batch holding only Coulomb instances: advance waits for them in turn."""
    b = E.Batch(precision=abi.EDUS_PREC_FP64)
    slots = []
    for q in range(3):
        d = f"{workdir}/c{q}"
        slots.append(b.add(E.Problem(E.parse_input(W.hbn_coulomb(d, n=12 + 2 * q, t_fin_fs=0.3, it_res=5)), d)))
    _drain(b, slots)
    for s in slots:
        assert len(b.obs(s)) > 0
        b.release(s)
    assert b.stats()["bytes_used"] == 0


@pytest.mark.parametrize("nw,nside,n", [(8, 11, 16), (16, 13, 10), (2, 3, 24)])
def test_velocity_gauge_matches_oracle(workdir, nw, nside, n):
    """Velocity gauge (tdse{ velocity_gauge }): H and D rebuilt at k + A(t) for
    every RK4 stage on the device, against the oracle's restatement: rho within
    1e-13, J1 within the FP64 tolerance, populations within 1e-13; a replay of
    the captured loop after edus_reset gives the same state."""
    name = f"W{nw}"
    W.write_wannier_tb(f"{workdir}/{name}_tb.dat", nw=nw, nside=nside)
    path = W.wannier(workdir, nw=nw, nside=nside, name=name, n=n, t_fin_fs=1.5, it_res=5, field=0.5, write_model=False)
    txt = open(path).read().replace("Wannier\n", "Wannier\nvelocity_gauge\n")
    open(path, "w").write(txt)
    p = E.parse_input(path)
    assert p.velocity_gauge == 1
    ctx = E.Context(E.Problem(p, workdir))
    ctx.run()
    g, rho = ctx.obs(), ctx.get_state()
    o = Oracle(p, workdir)
    lo = o.run()
    assert np.abs(rho - o.get("P0")).max() < 1e-13
    assert len(g) == len(lo)
    assert RF.rel_l2([x["J1"] for x in g], [x["J1"] for x in lo]) < RF.J1_TOL
    assert np.abs(np.array([x["pop"] for x in g]) - np.array([x["pop"] for x in lo])).max() < 1e-13
    ctx.reset()
    ctx.run()
    assert np.array_equal(ctx.get_state(), rho)


@pytest.mark.parametrize("nw,nside,n", [(8, 11, 16), (16, 13, 10), (8, 9, 40)])
def test_velocity_gauge_tensor_core_contraction(workdir, nw, nside, n):
    """Velocity gauge with the stage contraction on the tensor cores (context
    precision EDUS_PREC_MIXED: exact 8-bit BF16 slices, FP32 sums exact per
    segment, FP64 across segments; FP64 state and commutator) against the FP64
    oracle: J1 within the mixed-precision bar 1e-6, rho and populations within
    1e-8."""
    name = f"W{nw}"
    W.write_wannier_tb(f"{workdir}/{name}_tb.dat", nw=nw, nside=nside)
    path = W.wannier(workdir, nw=nw, nside=nside, name=name, n=n, t_fin_fs=1.5, it_res=5, field=0.5, write_model=False)
    txt = open(path).read().replace("Wannier\n", "Wannier\nvelocity_gauge\n")
    open(path, "w").write(txt)
    p = E.parse_input(path)
    ctx = E.Context(E.Problem(p, workdir), precision=abi.EDUS_PREC_MIXED)
    ctx.run()
    g, rho = ctx.obs(), ctx.get_state()
    o = Oracle(p, workdir)
    lo = o.run()
    drho = float(np.abs(rho - o.get("P0")).max())
    j1 = RF.rel_l2([x["J1"] for x in g], [x["J1"] for x in lo])
    dpop = float(np.abs(np.array([x["pop"] for x in g]) - np.array([x["pop"] for x in lo])).max())
    assert j1 < 1e-6 and drho < 1e-8 and dpop < 1e-8, (j1, drho, dpop)
    # the single-issuer TMA form and the cp.async-staged form give the
    # warp-specialised form's sums bit for bit (every segment's FP32 sums are
    # exact, so staging and issue order cannot change them)
    for form in ("tma", "cpasync"):
        os.environ["EDUS_TC_GEMM"] = form
        try:
            alt = E.Context(E.Problem(p, workdir), precision=abi.EDUS_PREC_MIXED)
            alt.run()
        finally:
            del os.environ["EDUS_TC_GEMM"]
        assert np.array_equal(alt.get_state(), rho), form
        assert all(np.array_equal(x["J1"], y["J1"]) for x, y in zip(g, alt.obs())), form
