"""edus_observables_static (reduction scratch in a fixed device array) against
edus_observables on the same state, two calls in a row, through the C ABI."""
import ctypes as C

import numpy as np
import pytest

import edus_b200 as E
from edus_b200 import abi
from edus_b200 import workloads as W

pytestmark = pytest.mark.gpu


def static_call(ctx):
    L = ctx._L
    L.edus_observables_static.argtypes = [C.c_void_p, C.c_void_p]
    L.edus_observables_static.restype = C.c_int
    o = abi.Obs()
    rc = L.edus_observables_static(ctx._h, C.byref(o))
    return rc, o


def static_obs(ctx):
    rc, o = static_call(ctx)
    assert rc == 0, ctx._L.edus_last_error()
    return abi.obs_to_dict(o, ctx.n)


def same(a, b):
    for key in ("J1", "J2", "pop", "tabs", "pol"):
        x, y = np.asarray(a[key]), np.asarray(b[key])
        assert np.abs(x - y).max() <= 1e-14 * max(np.abs(y).max(), 1e-300), key
    # the trace check and the population extremes of the same reduction
    for key in ("trace_dev", "n_cond", "p_cond_max", "p_min"):
        assert abs(a[key] - b[key]) <= 1e-14 * max(abs(b[key]), 1.0), key
    assert a["t"] == b["t"] and a["dt"] == b["dt"]


@pytest.mark.parametrize("kind", ["rk4", "coulomb"])
def test_static_scratch_observables_match(workdir, kind):
    if kind == "rk4":
        path = W.hbn_rk4(workdir, n=24, t_fin_fs=1.0, it_res=5)
    else:
        path = W.hbn_coulomb(workdir, n=24, t_fin_fs=1.0, it_res=5)
    ctx = E.Context(E.Problem(E.parse_input(path), workdir), use_graphs=False)
    ctx.step(40)
    ref = ctx.observables()
    first = static_obs(ctx)
    second = static_obs(ctx)
    same(first, ref)
    same(second, ref)
    assert abs(ref["J1"]).max() > 0
    ctx.step(7)
    same(static_obs(ctx), ctx.observables())


def test_static_scratch_refuses_grids_beyond_its_limit(workdir):
    """730 x 730 = 532 900 k points exceed the 524 288 the array holds: the call
    returns EDUS_EINVAL before touching the device."""
    path = W.hbn_rk4(workdir, n=730, t_fin_fs=-0.2, it_res=1)
    pb = E.Problem(E.parse_input(path), workdir)
    pb.drop_decoupled_core()
    ctx = E.Context(pb, use_graphs=False)
    rc, _ = static_call(ctx)
    assert rc == abi.EDUS_EINVAL
    assert b"static observable scratch" in ctx._L.edus_last_error()
    assert ctx.observables()["t"] == pytest.approx(ctx.clock()[1])
