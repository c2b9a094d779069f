"""Batched engine (edus_batch_*): every instance of a batch against the
single-solve path on the same input.

FP64 instances reproduce the single-solve FP64 path (same host field table,
same arithmetic; only the order of the observable reductions differs):
rho to 1e-13 absolute, J1 to 1e-11 relative L2 (the tolerance of the single-solve
parity tests: these short runs have currents near the summation noise). Mixed-precision instances
(FP32 H, D and commutator, FP64 rho) are held to 1e-5 relative L2 in J1 on
these short runs; the configuration-sized runs are held to 1e-6
(tests/test_gpu_reference.py), and bench.py reports the sweep's errors.
"""
import os

import numpy as np
import pytest

import edus_b200 as E
from edus_b200 import abi
from edus_b200 import workloads as W

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def single(problem):
    ctx = E.Context(problem, use_graphs=False)
    ctx.run()
    return ctx.get_state(), ctx.obs()


def drain(batch, slots, chunk=16):
    for _ in range(100000):
        if all(batch.poll(s)[0] == abi.EDUS_INST_DONE for s in slots):
            return
        batch.advance(chunk)
    raise AssertionError("batch did not finish")


def J1(log):
    return np.array([x["J1"] for x in log])


def problems(workdir):
    out = []
    for i, (n, tf) in enumerate([(16, 0.6), (20, 0.4), (12, 0.8)]):
        d = f"{workdir}/hbn{i}"
        out.append(E.Problem(E.parse_input(W.hbn_rk4(d, n=n, t_fin_fs=tf, it_res=3, field=0.3 + 0.1 * i)), d))
    d = f"{workdir}/wan"
    out.append(E.Problem(E.parse_input(W.wannier(d, n=12, t_fin_fs=0.4, it_res=4)), d))
    return out


def test_fp64_batch_matches_single_solves(workdir):
    pbs = problems(workdir)
    ref = [single(p) for p in pbs]
    b = E.Batch(precision=abi.EDUS_PREC_FP64, chunk_steps=8)
    slots = [b.add(p, tag=i) for i, p in enumerate(pbs)]
    drain(b, slots, 8)
    for s, (rho, log) in zip(slots, ref):
        assert np.abs(b.get_state(s) - rho).max() < 1e-13
        lb = b.obs(s)
        assert len(lb) == len(log)
        assert all(x["t"] == y["t"] for x, y in zip(lb, log))
        assert rel(J1(lb), J1(log)) < 1e-11
        J2b, J2s = np.array([x["J2"] for x in lb]), np.array([x["J2"] for x in log])
        assert rel(J2b, J2s) < 1e-10
        pg, po = np.array([x["pop"] for x in lb]), np.array([x["pop"] for x in log])
        assert np.abs(pg - po).max() < 1e-14
        Pb, Ps = np.array([x["pol"] for x in lb]), np.array([x["pol"] for x in log])
        assert np.abs(Pb - Ps).max() < 1e-13 * max(np.abs(Ps).max(), 1.0)
    st = b.stats()
    assert st["done"] == len(slots) and st["kpoint_steps"] > 0 and st["device_ms"] > 0


def test_late_admission_gives_the_same_result(workdir):
    """Continuous batching: an instance admitted while others run equals its solo run."""
    pbs = problems(workdir)
    b = E.Batch(chunk_steps=8)
    first = [b.add(p) for p in pbs[:2]]
    b.advance(24)
    late = b.add(pbs[2])
    b.advance(8)
    b.release(first[0])            # leaves while the others run
    again = b.add(pbs[3])          # reuses memory of the released slot
    drain(b, [first[1], late, again], 8)
    for s, p in [(first[1], pbs[1]), (late, pbs[2]), (again, pbs[3])]:
        rho, log = single(p)
        assert np.abs(b.get_state(s) - rho).max() < 1e-13
        assert rel(J1(b.obs(s)), J1(log)) < 1e-11


def test_graph_and_eager_chunks_agree(workdir):
    pbs = problems(workdir)[:2]
    out = []
    for g in (True, False):
        b = E.Batch(chunk_steps=4, use_graphs=g)
        slots = [b.add(p) for p in pbs]
        drain(b, slots, 4)
        out.append([b.get_state(s) for s in slots])
    for x, y in zip(*out):
        assert np.array_equal(x, y)


def test_mixed_precision_error_is_small(workdir):
    """Mixed precision keeps rho - rho_eq in FP64 and needs problems without
    core bands: the hBN problems lose their decoupled core band (the remaining
    block evolves exactly as in the full problem)."""
    pbs = problems(workdir)
    ref = [single(p) for p in pbs]
    for p in pbs:
        if p.info.nch:
            p.drop_decoupled_core()
    b = E.Batch(precision=abi.EDUS_PREC_MIXED)
    slots = [b.add(p) for p in pbs]
    drain(b, slots)
    for s, p, (rho, log) in zip(slots, pbs, ref):
        off = rho.shape[1] - p.info.ncv
        assert np.abs(b.get_state(s) - rho[:, off:, off:]).max() < 1e-5
        assert rel(J1(b.obs(s)), J1(log)) < 1e-5


def test_mixed_batch_skips_stencil_residue_vectors(workdir):
    """On a 98 x 98 square grid the in-plane stencil steps carry a z component
    of 7.4e-17 (rounding of the grid-vector differences): a z-polarised pump
    makes their gradient coefficients 5e-15 of the largest. The FP32
    commutator skips them; the instance still follows its FP64 single solve
    to FP32 rounding, beside a 96 x 96 instance of the same class."""
    p98 = E.parse_input(W.wannier(f"{workdir}/w98", n=98, t_fin_fs=0.3, it_res=4))
    p96 = E.parse_input(W.wannier(f"{workdir}/w96", n=96, t_fin_fs=0.3, it_res=4))
    pb98 = E.Problem(p98, f"{workdir}/w98")
    bz = pb98.get("bvec")[:, 2]
    assert np.any((bz != 0) & (np.abs(bz) < 1e-12))  # the residue this test is about
    rho64, log64 = single(pb98)
    b = E.Batch(precision=abi.EDUS_PREC_MIXED, chunk_steps=8)
    s98 = b.add(E.Problem(p98, f"{workdir}/w98"))
    s96 = b.add(E.Problem(p96, f"{workdir}/w96"))
    drain(b, [s98, s96], 8)
    assert np.abs(b.get_state(s98) - rho64).max() < 1e-5
    assert rel(J1(b.obs(s98)), J1(log64)) < 1e-5


def test_mixed_batch_runs_small_band_classes_in_fp64(workdir):
    """A mixed-precision batch runs the 2- and 3-band classes in FP64 (their
    k-gradient needs FP64 stage inputs), core bands included: the 3-band hBN
    instance equals its FP64 single solve as the FP64 batch does."""
    d = f"{workdir}/core"
    pb = E.Problem(E.parse_input(W.hbn_rk4(d, n=12, t_fin_fs=0.3, it_res=3)), d)
    rho, log = single(pb)
    b = E.Batch(precision=abi.EDUS_PREC_MIXED, chunk_steps=8)
    s = b.add(pb)
    drain(b, [s], 8)
    assert np.abs(b.get_state(s) - rho).max() < 1e-13
    # a 0.3 fs run: J1 (~4e-8) is a k sum at its rounding floor, summed in another order
    assert rel(J1(b.obs(s)), J1(log)) < 5e-11


def test_admission_by_hbm_budget(workdir):
    pbs = problems(workdir)
    probe = E.Batch()
    need = probe.footprint(pbs[0])
    probe.close()
    b = E.Batch(hbm_budget_bytes=int(need * 2.5))
    a = b.try_add(pbs[0])
    c = b.try_add(pbs[0])
    assert a is not None and c is not None
    assert b.try_add(pbs[0]) is None          # the third does not fit
    st = b.stats()
    assert st["active"] == 2 and st["bytes_used"] == 2 * need
    b.release(a)
    assert b.try_add(pbs[0]) is not None      # fits again once a slot is released


def test_unsupported_instances_are_refused(workdir):
    """Adaptive dt (with or without the Coulomb mean field) does not run in a batch."""
    dyn = "dynamical_dt_evolution\nepsStepAbs 0.001\n"
    d = f"{workdir}/dyn"
    p = E.Problem(E.parse_input(W.hbn_rk4(d, n=12, t_fin_fs=0.2, solver=dyn)), d)
    d2 = f"{workdir}/dyncoul"
    path = W.hbn_coulomb(d2, n=12, t_fin_fs=0.2, rk4=True)
    open(path, "a").write("")
    txt = open(path).read().replace("t_fin", dyn + "t_fin", 1)
    open(path, "w").write(txt)
    q = E.Problem(E.parse_input(path), d2)
    b = E.Batch()
    for pb in (p, q):
        with pytest.raises(E.EdusError) as ei:
            b.add(pb)
        assert ei.value.code == abi.EDUS_EUNSUPPORTED


@pytest.mark.parametrize("nw,nside,name", [(8, 11, "W8"), (16, 13, "W16")])
def test_device_built_wannier_model_matches_host_build(workdir, nw, nside, name):
    """A deferred problem (model tabulated on the device at admission) evolves
    like the host-tabulated one: rho0 is the same projector, J(t) and the
    populations agree (eigenvector phases differ and cancel)."""
    d = f"{workdir}/{name}"
    p = E.parse_input(W.wannier(d, nw=nw, nside=nside, n=12, t_fin_fs=0.3, it_res=4, name=name))
    host = E.Problem(p, d)
    dev = E.Problem(p, d, defer_model=True)
    b = E.Batch(chunk_steps=8)
    sh, sd = b.add(host), b.add(dev)
    assert np.abs(b.get_state(sh) - b.get_state(sd)).max() < 1e-13
    drain(b, [sh, sd], 8)
    assert np.abs(b.get_state(sh) - b.get_state(sd)).max() < 1e-12
    lh, ld = b.obs(sh), b.obs(sd)
    assert rel(J1(ld), J1(lh)) < 1e-10
    ph, pd = np.array([x["pop"] for x in lh]), np.array([x["pop"] for x in ld])
    assert np.abs(ph - pd).max() < 1e-12


@pytest.mark.parametrize("kt", [8, 16])
def test_matrix_product_form_matches_single_solve(workdir, kt):
    """Register profile 2 (C = P H~^T in register blocks) against the single-solve path."""
    d = f"{workdir}/w8mm"
    p = E.parse_input(W.wannier(d, n=12, t_fin_fs=0.4, it_res=4))
    pb = E.Problem(p, d)
    rho, log = single(pb)
    # built for FP64 only (a mixed batch runs the element-parallel form)
    b = E.Batch(precision=abi.EDUS_PREC_FP64, chunk_steps=8, tile_k={8: kt}, regs_profile={8: 2})
    s = b.add(pb)
    drain(b, [s], 8)
    assert np.abs(b.get_state(s) - rho).max() < 1e-13
    assert rel(J1(b.obs(s)), J1(log)) < 1e-11


def test_matrix_product_form_16_bands(workdir):
    d = f"{workdir}/w16mm"
    p = E.parse_input(W.wannier(d, nw=16, nside=13, n=10, t_fin_fs=0.2, it_res=5, name="W16"))
    out = {}
    for prof, kt in [(0, 2), (2, 2), (2, 4), (2, 8)]:
        b = E.Batch(chunk_steps=8, tile_k={16: kt}, regs_profile={16: prof})
        s = b.add(E.Problem(p, d))
        drain(b, [s], 8)
        out[(prof, kt)] = (b.get_state(s), J1(b.obs(s)))
    ref_rho, ref_j = out[(0, 2)]
    for key, (rho, j) in out.items():
        assert np.abs(rho - ref_rho).max() < 1e-13, key
        assert rel(j, ref_j) < 1e-11, key


@pytest.mark.parametrize("nw,nside,name", [(8, 11, "W8"), (16, 13, "W16")])
def test_tensor_core_model_build(workdir, nw, nside, name):
    """Mixed precision with the model contracted on the tensor cores (exact 8-bit
    slices in BF16 with kind::f16 MMAs, FP32 sums exact per segment, FP64 sums
    across segments and FP64 band energies) against the FP64 CUDA-core build:
    the same dynamics to FP32 rounding."""
    d = f"{workdir}/{name}"
    p = E.parse_input(W.wannier(d, nw=nw, nside=nside, n=12, t_fin_fs=0.4, it_res=4, name=name))
    ref = E.Batch(precision=abi.EDUS_PREC_FP64, chunk_steps=8)
    s = ref.add(E.Problem(p, d, defer_model=True))
    rho0 = ref.get_state(s)
    drain(ref, [s], 8)
    rho64, j64 = ref.get_state(s), J1(ref.obs(s))
    runs = {}
    for tc in (False, True):
        b = E.Batch(precision=abi.EDUS_PREC_MIXED, chunk_steps=8, tc_contraction=tc)
        s = b.add(E.Problem(p, d, defer_model=True))
        # the ground-state projector of the tensor-core build is taken from its
        # FP32 tables (the FP64 build's from FP64 H(k))
        assert np.abs(b.get_state(s) - rho0).max() < (1e-6 if tc else 1e-13)
        drain(b, [s], 8)
        assert np.abs(b.get_state(s) - rho64).max() < 1e-5
        assert rel(J1(b.obs(s)), j64) < 1e-5
        runs[tc] = (b.get_state(s), J1(b.obs(s)))
    # exact slices: the tensor-core tables equal the FP64 build's to the FP32 rounding
    assert np.abs(runs[True][0] - runs[False][0]).max() < 1e-6
    assert rel(runs[True][1], runs[False][1]) < 1e-6
    # the single-issuer TMA and the cp.async-staged GEMM forms give the
    # warp-specialised form's sums bit for bit
    for form in ("tma", "cpasync"):
        os.environ["EDUS_TC_GEMM"] = form
        try:
            b = E.Batch(precision=abi.EDUS_PREC_MIXED, chunk_steps=8, tc_contraction=True)
            s = b.add(E.Problem(p, d, defer_model=True))
        finally:
            del os.environ["EDUS_TC_GEMM"]
        drain(b, [s], 8)
        assert np.array_equal(b.get_state(s), runs[True][0]), form
        assert np.array_equal(J1(b.obs(s)), runs[True][1]), form


def test_staged_form_equals_element_parallel_form(workdir):
    """Register profile 3 (operands staged with cp.async, one tile ahead) does
    the arithmetic of profile 0 in the same order: the same state and
    observables for 2-, 8- and 16-band instances, and a fallback to profile 0
    for an instance whose field uses all three components."""
    reqs = []
    d = f"{workdir}/h"
    hb = E.Problem(E.parse_input(W.hbn_rk4(d, n=20, t_fin_fs=0.5, it_res=3, field=0.4)), d).drop_decoupled_core()
    reqs.append(hb)
    d = f"{workdir}/w8"
    reqs.append(E.Problem(E.parse_input(W.wannier(d, n=12, t_fin_fs=0.4, it_res=4)), d))
    d = f"{workdir}/w16"
    reqs.append(E.Problem(E.parse_input(W.wannier(d, nw=16, nside=13, n=10, t_fin_fs=0.2, it_res=5, name="W16")), d))
    d = f"{workdir}/w8xyz"
    reqs.append(E.Problem(E.parse_input(W.wannier(d, n=12, t_fin_fs=0.3, it_res=4, pol="0.3 0.5 0.8")), d))
    out = {0: [], 3: []}
    for prof in (0, 3):
        # the three-component instance runs in a batch of its own: it sends its whole class to profile 0
        for group in (reqs[:3], reqs[3:]):
            b = E.Batch(precision=abi.EDUS_PREC_MIXED, chunk_steps=8, regs_profile={2: prof, 8: prof, 16: prof})
            slots = [b.add(p) for p in group]
            drain(b, slots, 8)
            out[prof] += [(b.get_state(s), J1(b.obs(s))) for s in slots]
    for (r0, j0), (r3, j3) in zip(out[0], out[3]):
        assert np.array_equal(r0, r3)
        assert np.array_equal(j0, j3)


@pytest.mark.parametrize("nw,nside,name,kt", [(8, 11, "W8", 8), (8, 11, "W8", 16), (16, 13, "W16", 2), (16, 13, "W16", 4)])
def test_blocked_commutator_form(workdir, nw, nside, name, kt):
    """Register profile 4 (commutator from register blocks of C = P H~^T), also
    with tiles the element-parallel form is not built for, against profile 3:
    the same dynamics to FP32 rounding."""
    d = f"{workdir}/{name}"
    p = E.parse_input(W.wannier(d, nw=nw, nside=nside, n=12, t_fin_fs=0.4, it_res=4, name=name))
    out = {}
    for prof in (3, 4):
        b = E.Batch(precision=abi.EDUS_PREC_MIXED, chunk_steps=8, regs_profile={nw: prof},
                    tile_k={nw: kt if prof == 4 else (8 if nw == 8 else 2)})
        s = b.add(E.Problem(p, d))
        drain(b, [s], 8)
        out[prof] = (b.get_state(s), J1(b.obs(s)))
    assert np.abs(out[4][0] - out[3][0]).max() < 1e-6
    assert rel(out[4][1], out[3][1]) < 1e-6
    # profile 5 (2 x 1 blocks of C) sums every entry of C in the same order as profile 4
    b = E.Batch(precision=abi.EDUS_PREC_MIXED, chunk_steps=8, regs_profile={nw: 5}, tile_k={nw: kt})
    s = b.add(E.Problem(p, d))
    drain(b, [s], 8)
    assert np.array_equal(b.get_state(s), out[4][0])
    assert np.array_equal(J1(b.obs(s)), out[4][1])


def test_16_band_single_solve_matches_batch(workdir):
    """The single-solve FP64 path for 16 bands against the FP64 batch engine."""
    d = f"{workdir}/w16s"
    pb = E.Problem(E.parse_input(W.wannier(d, nw=16, nside=13, n=10, t_fin_fs=0.2, it_res=5, name="W16")), d)
    rho, log = single(pb)
    b = E.Batch(precision=abi.EDUS_PREC_FP64, chunk_steps=8)
    s = b.add(pb)
    drain(b, [s], 8)
    assert np.abs(b.get_state(s) - rho).max() < 1e-13
    assert rel(J1(b.obs(s)), J1(log)) < 1e-11


@pytest.mark.parametrize("kind,n", [("w8", 10), ("w8", 6), ("hbn", 10), ("w16", 6)])
def test_staged_forms_on_ragged_grids(workdir, kind, n):
    """Grids whose rows are not whole tiles (tiles crossing rows, the wrap-around
    stencil path, instances smaller than a tile): the staged forms (profile 3
    for 2 bands, 4 for 8 and 16) against the element-parallel form (profile 0)
    and the FP64 single solve."""
    d = f"{workdir}/{kind}{n}"
    if kind == "hbn":
        p = E.parse_input(W.hbn_rk4(d, n=n, t_fin_fs=0.3, it_res=3, field=0.5))
        nb, prof, kts = 2, 3, (32,)
    elif kind == "w8":
        p = E.parse_input(W.wannier(d, n=n, t_fin_fs=0.3, it_res=4))
        nb, prof, kts = 8, 4, (8, 16)
    else:
        p = E.parse_input(W.wannier(d, nw=16, nside=13, n=n, t_fin_fs=0.2, it_res=5, name="W16"))
        nb, prof, kts = 16, 4, (2, 4)
    rho64, log64 = single(E.Problem(p, d))

    def run(profile, kt):
        pb = E.Problem(p, d)
        if kind == "hbn":
            pb.drop_decoupled_core()
        b = E.Batch(precision=abi.EDUS_PREC_MIXED, chunk_steps=8, regs_profile={nb: profile}, tile_k={nb: kt})
        s = b.add(pb)
        drain(b, [s], 8)
        return b.get_state(s), J1(b.obs(s))

    ref_rho, ref_j = run(0, 32 if nb == 2 else (8 if nb == 8 else 2))
    assert rel(ref_j, J1(log64)) < 1e-5
    for kt in kts:
        rho, j = run(prof, kt)
        assert np.abs(rho - ref_rho).max() < 1e-6
        assert rel(j, ref_j) < 1e-6
