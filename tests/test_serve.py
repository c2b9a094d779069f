"""Serving loop (edus_server_*): requests submitted while others run are
admitted by HBM footprint, run concurrently, and give the same result as when
run alone.

An instance's arithmetic and the order of its observable reductions depend
only on its own tiles, so "alone" and "in the mix" agree bit for bit in both
precisions. The FP64 served result is also checked against the single-solve
path (J1 1e-11 relative L2, populations 1e-14).
"""
import time

import numpy as np
import pytest

import edus_b200 as E
from edus_b200 import abi
from edus_b200 import workloads as W

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def requests(workdir):
    """(params, workdir) of a small mix: hBN (core band dropped -> 2 bands),
    8-band and 16-band Wannier models, uneven grids and durations, and an hBN
    request with the Rytova-Keldysh mean field (3 bands, FP64 context)."""
    out = []
    for i, (n, tf, f) in enumerate([(16, 0.5, 0.3), (22, 0.3, 0.6), (12, 0.7, 0.1)]):
        d = f"{workdir}/h{i}"
        out.append((E.parse_input(W.hbn_rk4(d, n=n, t_fin_fs=tf, it_res=3, field=f, phase=0.4 * i)), d))
    d = f"{workdir}/w8"
    out.append((E.parse_input(W.wannier(d, n=12, t_fin_fs=0.3, it_res=4)), d))
    d = f"{workdir}/w16"
    out.append((E.parse_input(W.wannier(d, nw=16, nside=13, n=10, t_fin_fs=0.2, it_res=5, name="W16")), d))
    d = f"{workdir}/coul"
    out.append((E.parse_input(W.hbn_coulomb(d, n=14, t_fin_fs=0.4, it_res=3, field=0.6)), d))
    return out


def serve(reqs, precision, stagger_s=0.0, **kw):
    s = E.Server(precision=precision, chunk_steps=8, **kw)
    ids = []
    for q, (p, d) in enumerate(reqs):
        ids.append(s.submit(p, d))
        if stagger_s and q % 2:
            time.sleep(stagger_s)
    s.drain(300)
    out = [s.obs(i) for i in ids]
    infos = [s.info(i) for i in ids]
    st = s.stats()
    s.close()
    return out, infos, st


@pytest.mark.parametrize("precision", [abi.EDUS_PREC_FP64, abi.EDUS_PREC_MIXED])
def test_each_result_is_the_same_alone_and_in_the_mix(workdir, precision):
    reqs = requests(workdir)
    mix, infos, st = serve(reqs, precision, stagger_s=0.02)
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["p50_latency_s"] > 0 and st["p99_latency_s"] >= st["p50_latency_s"]
    assert infos[0]["nbands"] == 2          # the hBN core band was dropped
    assert infos[4]["nbands"] == 16
    assert infos[5]["nbands"] == 3          # Coulomb keeps the core band (FP64 context)
    for q, req in enumerate(reqs):
        alone, _, _ = serve([req], precision)
        a, b = alone[0], mix[q]
        assert len(a) == len(b) > 0
        for x, y in zip(a, b):
            assert np.array_equal(x["J1"], y["J1"]) and np.array_equal(x["pop"], y["pop"])


def test_fp64_served_solves_match_the_single_solve_path(workdir):
    reqs = requests(workdir)[:4]
    out, infos, _ = serve(reqs, abi.EDUS_PREC_FP64)
    for (p, d), log, info in zip(reqs, out, infos):
        ctx = E.Context(E.Problem(p, d), use_graphs=False)
        ctx.run()
        ref = ctx.obs()
        assert len(ref) == len(log)
        J = lambda L: np.array([x["J1"] for x in L])
        assert rel(J(log), J(ref)) < 1e-11
        off = ctx.problem.info.ncv - info["nbands"]   # dropped core columns
        pg = np.array([x["pop"] for x in log])
        po = np.array([x["pop"][off:] for x in ref])
        assert np.abs(pg - po).max() < 1e-14


def test_admission_waits_for_memory(workdir):
    reqs = requests(workdir)[:3]
    probe = E.Batch()
    pb = E.Problem(*reqs[1]).drop_decoupled_core()
    need = probe.footprint(pb)
    probe.close()
    many = [reqs[1]] * 6
    out, infos, st = serve(many, abi.EDUS_PREC_FP64, hbm_budget_bytes=int(need * 2.5))
    assert st["completed"] == 6 and st["peak_active"] <= 2
    for o in out[1:]:
        assert all(np.array_equal(x["J1"], y["J1"]) for x, y in zip(o, out[0]))


def test_unsupported_request_fails_alone(workdir):
    """A request the batch does not run (adaptive dt) fails alone."""
    reqs = requests(workdir)[:2]
    d = f"{workdir}/dyn"
    bad = (E.parse_input(W.hbn_rk4(d, n=12, t_fin_fs=0.2, solver="dynamical_dt_evolution\nepsStepAbs 0.001\n")), d)
    s = E.Server(chunk_steps=8)
    ids = [s.submit(*reqs[0]), s.submit(*bad), s.submit(*reqs[1])]
    s.drain(300)
    st = [s.info(i)["status"] for i in ids]
    assert st == [abi.EDUS_REQ_DONE, abi.EDUS_REQ_FAILED, abi.EDUS_REQ_DONE]
    assert s.info(ids[1])["error"] == abi.EDUS_EUNSUPPORTED
    with pytest.raises(E.EdusError):
        s.obs(ids[1])
    s.close()


@pytest.mark.parametrize("precision", [abi.EDUS_PREC_FP64, abi.EDUS_PREC_MIXED])
def test_diverging_request_fails_alone(workdir, precision):
    """Health check at retirement: an RK4 step 100x past its stability limit
    overflows (floating point only, nothing faults); that request fails with
    EDUS_ENONFINITE or EDUS_ETRACE while the others complete."""
    reqs = requests(workdir)[:2]
    d = f"{workdir}/unstable"
    bad = (E.parse_input(W.hbn_rk4(d, n=12, t_fin_fs=120.0, it_res=5, dt_fs=1.0, field=0.5)), d)
    s = E.Server(precision=precision, chunk_steps=8)
    ids = [s.submit(*reqs[0]), s.submit(*bad), s.submit(*reqs[1])]
    s.drain(300)
    st = [s.info(i)["status"] for i in ids]
    assert st == [abi.EDUS_REQ_DONE, abi.EDUS_REQ_FAILED, abi.EDUS_REQ_DONE]
    assert s.info(ids[1])["error"] in (abi.EDUS_ENONFINITE, abi.EDUS_ETRACE)
    with pytest.raises(E.EdusError):
        s.obs(ids[1])
    s.close()


def test_served_coulomb_request_matches_the_single_solve_path(workdir):
    """A Coulomb request in the mix runs as its own FP64 context: bit for bit the
    single-solve result on the same input."""
    reqs = requests(workdir)
    out, infos, _ = serve(reqs, abi.EDUS_PREC_MIXED, stagger_s=0.01)
    p, d = reqs[5]
    ctx = E.Context(E.Problem(p, d))
    ctx.run()
    ref = ctx.obs()
    assert len(ref) == len(out[5]) > 0
    for x, y in zip(out[5], ref):
        assert np.array_equal(x["J1"], y["J1"]) and np.array_equal(x["pop"], y["pop"])
