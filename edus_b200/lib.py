"""ctypes bindings of libedus_b200.so (include/edus_b200.h)."""
import ctypes as C
import os

import numpy as np

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


class EdusError(RuntimeError):
    def __init__(self, code, where, message):
        super().__init__(f"{where}: {message} (code {code})")
        self.code = code


def library_path():
    return os.path.join(_HERE, "libedus_b200.so")


def load_library():
    """Load the in-tree library; raise (never fall back) if it is absent."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = library_path()
    if not os.path.exists(path):
        raise EdusError(-1, "load_library", f"{path} is missing; run `python -m edus_b200.build`")
    L = C.CDLL(path)
    vp, i32, dbl, cp, sz = C.c_void_p, C.c_int32, C.c_double, C.c_char_p, C.c_size_t
    P = C.POINTER
    sigs = {
        "edus_parse_input": (C.c_int, [cp, P(abi.Params)]),
        "edus_params_default": (C.c_int, [P(abi.Params)]),
        "edus_problem_create": (C.c_int, [P(abi.Params), cp, P(vp)]),
        "edus_problem_info_get": (C.c_int, [vp, P(abi.ProblemInfo)]),
        "edus_problem_drop_decoupled_core": (C.c_int, [vp]),
        "edus_problem_create_deferred": (C.c_int, [P(abi.Params), cp, P(vp)]),
        "edus_problem_get": (C.c_int, [vp, cp, vp, sz]),
        "edus_problem_free": (None, [vp]),
        "edus_problem_write_kgrid": (C.c_int, [vp, cp]),
        "edus_problem_write_kpt": (C.c_int, [vp, cp]),
        "edus_problem_write_test_matrices": (C.c_int, [vp, cp]),
        "edus_model_hud": (C.c_int, [vp, P(dbl), vp, vp, vp]),
        "edus_struct_sizes": (C.c_int, [P(C.c_int64)]),
        "edus_options_default": (C.c_int, [P(abi.Options)]),
        "edus_create": (C.c_int, [vp, P(abi.Options), P(vp)]),
        "edus_destroy": (None, [vp]),
        "edus_set_state": (C.c_int, [vp, vp]),
        "edus_get_state": (C.c_int, [vp, vp]),
        "edus_step": (C.c_int, [vp, i32]),
        "edus_run": (C.c_int, [vp]),
        "edus_reset": (C.c_int, [vp]),
        "edus_clock": (C.c_int, [vp, P(i32), P(dbl), P(dbl)]),
        "edus_obs_count": (C.c_int, [vp, P(i32)]),
        "edus_obs_get": (C.c_int, [vp, i32, i32, P(abi.Obs)]),
        "edus_observables": (C.c_int, [vp, P(abi.Obs)]),
        "edus_write_outputs": (C.c_int, [vp, cp]),
        "edus_last_timing": (C.c_int, [vp, P(dbl), P(C.c_int64)]),
        "edus_profile": (C.c_int, [vp, i32, P(dbl), P(C.c_int64), P(dbl), P(C.c_int64)]),
        "edus_profile_ex": (C.c_int, [vp, i32, i32, P(dbl), P(C.c_int64), P(dbl), P(C.c_int64)]),
        "edus_get_derivative": (C.c_int, [vp, i32, P(dbl), dbl, i32]),
        "edus_runge_kutta_ad": (C.c_int, [vp, i32, i32, dbl]),
        "edus_runge_kutta_ac": (C.c_int, [vp, i32, dbl]),
        "edus_slot_copy": (C.c_int, [vp, i32, i32]),
        "edus_slot_set": (C.c_int, [vp, i32, vp]),
        "edus_slot_get": (C.c_int, [vp, i32, vp]),
        "edus_coulomb_hk": (C.c_int, [vp, i32, vp]),
        "edus_coulomb_gen_options_default": (C.c_int, [P(abi.CoulombGenOptions)]),
        "edus_coulomb_generate": (C.c_int, [P(abi.Params), cp, P(abi.CoulombGenOptions), C.c_char_p, i32, P(i32)]),
        "edus_observables_static": (C.c_int, [vp, P(abi.Obs)]),
        "edus_batch_options_default": (C.c_int, [P(abi.BatchOptions)]),
        "edus_batch_create": (C.c_int, [P(abi.BatchOptions), P(vp)]),
        "edus_batch_destroy": (None, [vp]),
        "edus_batch_footprint": (C.c_int, [vp, vp, P(C.c_int64)]),
        "edus_batch_add": (C.c_int, [vp, vp, C.c_int64, P(i32)]),
        "edus_batch_advance": (C.c_int, [vp, i32]),
        "edus_batch_poll": (C.c_int, [vp, i32, P(i32), P(i32), P(C.c_int64)]),
        "edus_batch_obs_count": (C.c_int, [vp, i32, P(i32)]),
        "edus_batch_obs_get": (C.c_int, [vp, i32, i32, i32, P(abi.Obs)]),
        "edus_batch_get_state": (C.c_int, [vp, i32, vp]),
        "edus_batch_release": (C.c_int, [vp, i32]),
        "edus_batch_stats_get": (C.c_int, [vp, P(abi.BatchStats)]),
        "edus_batch_tile_k": (C.c_int, [vp, i32, P(i32)]),
        "edus_batch_profile": (C.c_int, [vp, i32, P(abi.KernelTime), i32, P(i32)]),
        "edus_selftest_bounded_wait": (C.c_int, [i32, i32]),
        "edus_server_options_default": (C.c_int, [P(abi.ServerOptions)]),
        "edus_server_create": (C.c_int, [P(abi.ServerOptions), P(vp)]),
        "edus_server_submit": (C.c_int, [vp, P(abi.Params), cp, P(C.c_int64)]),
        "edus_server_info": (C.c_int, [vp, C.c_int64, P(abi.RequestInfo)]),
        "edus_server_obs": (C.c_int, [vp, C.c_int64, i32, i32, P(abi.Obs)]),
        "edus_server_forget": (C.c_int, [vp, C.c_int64]),
        "edus_server_drain": (C.c_int, [vp, dbl]),
        "edus_server_stats_get": (C.c_int, [vp, P(abi.ServerStats)]),
        "edus_server_clock": (dbl, [vp]),
        "edus_server_destroy": (None, [vp]),
        "edus_strerror": (cp, [C.c_int]),
        "edus_last_error": (cp, []),
        "edus_abi_version": (C.c_int, []),
    }
    for name, (res, args) in sigs.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _LIB = L
    return L


def _check(rc, where):
    if rc != 0:
        L = load_library()
        msg = L.edus_last_error().decode(errors="replace") or L.edus_strerror(rc).decode()
        raise EdusError(rc, where, msg)


def default_params():
    L = load_library()
    p = abi.Params()
    _check(L.edus_params_default(C.byref(p)), "edus_params_default")
    return p


def parse_input(path):
    L = load_library()
    p = abi.Params()
    _check(L.edus_parse_input(os.fsencode(path), C.byref(p)), "edus_parse_input")
    return p


def coulomb_generate(params, workdir, device=0, n_sum=None, n_sum_screen=None):
    """Coulomb tables of a run computed on the GPU (edus_coulomb_generate):
    writes workdir/Output/Coulomb/*<label>.txt; returns (label, number of G)."""
    L = load_library()
    o = abi.CoulombGenOptions()
    _check(L.edus_coulomb_gen_options_default(C.byref(o)), "edus_coulomb_gen_options_default")
    o.device = device
    if n_sum is not None:
        o.n_sum = n_sum
    if n_sum_screen is not None:
        o.n_sum_screen = n_sum_screen
    lab = C.create_string_buffer(512)
    ng = C.c_int32()
    _check(L.edus_coulomb_generate(C.byref(params), os.fsencode(workdir), C.byref(o), lab, 512, C.byref(ng)),
           "edus_coulomb_generate")
    return lab.value.decode(), ng.value


class Problem:
    """Host-side problem (grid, stencil, model tables, initial state)."""

    def __init__(self, params, workdir=".", defer_model=False):
        L = load_library()
        self._L = L
        self.params = params
        self._h = C.c_void_p()
        if defer_model:
            _check(L.edus_problem_create_deferred(C.byref(params), os.fsencode(workdir), C.byref(self._h)),
                   "edus_problem_create_deferred")
        else:
            _check(L.edus_problem_create(C.byref(params), os.fsencode(workdir), C.byref(self._h)), "edus_problem_create")
        self.info = abi.ProblemInfo()
        _check(L.edus_problem_info_get(self._h, C.byref(self.info)), "edus_problem_info_get")

    def drop_decoupled_core(self):
        """Remove core bands nothing in the run couples (edus_problem_drop_decoupled_core)."""
        L = load_library()
        _check(L.edus_problem_drop_decoupled_core(self._h), "edus_problem_drop_decoupled_core")
        self.info = abi.ProblemInfo()
        _check(L.edus_problem_info_get(self._h, C.byref(self.info)), "edus_problem_info_get")
        return self

    def get(self, name):
        i = self.info
        n, nk = i.ncv, i.nk
        shapes = {
            "kpt": ((nk, 3), np.float64),
            "H": ((nk, n, n), np.complex128),
            "U": ((nk, n, n), np.complex128),
            "D": ((nk, n, n, 3), np.complex128),
            "GE": ((nk, n, n, 3), np.complex128),
            "P0": ((nk, n, n), np.complex128),
            "nbr": ((nk, i.nnb), np.int32),
            "bvec": ((i.nnb, 3), np.float64),
            "weights": ((i.nnb,), np.float64),
            "T": ((16, 16), np.float64),
            "HR": ((n, n, i.nrpts), np.complex128),
            "rR": ((3, n, n, i.nrpts), np.complex128),
            "Rvec": ((i.nrpts, 3), np.float64),
        }
        shp, dt = shapes[name]
        a = np.zeros(shp, dtype=dt)
        _check(self._L.edus_problem_get(self._h, name.encode(), a.ctypes.data, a.nbytes), f"edus_problem_get({name})")
        return a

    def write_kgrid(self, outdir):
        """outdir/k_grid.txt in the reference's format (edus_problem_write_kgrid)."""
        _check(self._L.edus_problem_write_kgrid(self._h, os.fsencode(outdir)), "edus_problem_write_kgrid")

    def write_kpt(self, workdir):
        """workdir/kpt.txt as the reference's BZ_parameters writes it (edus_problem_write_kpt)."""
        _check(self._L.edus_problem_write_kpt(self._h, os.fsencode(workdir)), "edus_problem_write_kpt")

    def write_test_matrices(self, workdir):
        """workdir/Test_matrices.txt as the reference's set-up prints it."""
        _check(self._L.edus_problem_write_test_matrices(self._h, os.fsencode(workdir)), "edus_problem_write_test_matrices")

    def model_hud(self, kcrys):
        """H, U, D of the model at one crystal k point (gHUD)."""
        n = self.info.ncv
        H = np.zeros((n, n), np.complex128)
        U = np.zeros((n, n), np.complex128)
        D = np.zeros((n, n, 3), np.complex128)
        k = (C.c_double * 3)(*[float(x) for x in kcrys])
        _check(self._L.edus_model_hud(self._h, k, H.ctypes.data, U.ctypes.data, D.ctypes.data), "edus_model_hud")
        return H, U, D

    def close(self):
        if self._h:
            self._L.edus_problem_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Context:
    """Device context: all state resident on one GPU."""

    def __init__(self, problem, device=0, precision=-1, use_graphs=True):
        L = load_library()
        self._L = L
        self.problem = problem
        o = abi.Options()
        _check(L.edus_options_default(C.byref(o)), "edus_options_default")
        o.device = device
        o.precision = precision
        o.use_graphs = 1 if use_graphs else 0
        self._h = C.c_void_p()
        _check(L.edus_create(problem._h, C.byref(o), C.byref(self._h)), "edus_create")
        self.n = problem.info.ncv
        self.nk = problem.info.nk

    def _state_buf(self):
        return np.zeros((self.nk, self.n, self.n), dtype=np.complex128)

    def get_state(self):
        a = self._state_buf()
        _check(self._L.edus_get_state(self._h, a.ctypes.data), "edus_get_state")
        return a

    def set_state(self, rho):
        a = np.ascontiguousarray(rho, dtype=np.complex128)
        _check(self._L.edus_set_state(self._h, a.ctypes.data), "edus_set_state")

    def step(self, nsteps):
        _check(self._L.edus_step(self._h, int(nsteps)), "edus_step")

    def run(self):
        _check(self._L.edus_run(self._h), "edus_run")

    def reset(self):
        _check(self._L.edus_reset(self._h), "edus_reset")

    def clock(self):
        it, t, dt = C.c_int32(), C.c_double(), C.c_double()
        _check(self._L.edus_clock(self._h, C.byref(it), C.byref(t), C.byref(dt)), "edus_clock")
        return it.value, t.value, dt.value

    def obs(self):
        n = C.c_int32()
        _check(self._L.edus_obs_count(self._h, C.byref(n)), "edus_obs_count")
        buf = (abi.Obs * max(n.value, 1))()
        _check(self._L.edus_obs_get(self._h, 0, n.value, buf), "edus_obs_get")
        return [abi.obs_to_dict(buf[i], self.n) for i in range(n.value)]

    def observables(self):
        o = abi.Obs()
        _check(self._L.edus_observables(self._h, C.byref(o)), "edus_observables")
        return abi.obs_to_dict(o, self.n)

    def write_outputs(self, outdir):
        _check(self._L.edus_write_outputs(self._h, os.fsencode(outdir)), "edus_write_outputs")

    def last_timing(self):
        ms, launches = C.c_double(), C.c_int64()
        _check(self._L.edus_last_timing(self._h, C.byref(ms), C.byref(launches)), "edus_last_timing")
        return ms.value, launches.value

    def profile(self, nsteps, reps=1):
        """Device time of the fused RHS kernel and of the Coulomb pair over nsteps (eager);
        reps > 1 repeats each idempotent RHS launch back to back between its events."""
        a, b, c, d = C.c_double(), C.c_int64(), C.c_double(), C.c_int64()
        _check(self._L.edus_profile_ex(self._h, int(nsteps), int(reps), C.byref(a), C.byref(b), C.byref(c), C.byref(d)),
               "edus_profile_ex")
        return {"rhs_ms": a.value, "rhs_launches": b.value, "coulomb_ms": c.value, "coulomb_launches": d.value}

    # ODE_solver-level mirror ---------------------------------------------
    def get_derivative(self, slot, EF, wx2, e_non0):
        ef = (C.c_double * 6)(*[float(x) for x in np.asarray(EF).ravel()])
        _check(self._L.edus_get_derivative(self._h, int(slot), ef, float(wx2), int(e_non0)), "edus_get_derivative")

    def slot_set(self, slot, rho):
        a = np.ascontiguousarray(rho, dtype=np.complex128)
        _check(self._L.edus_slot_set(self._h, int(slot), a.ctypes.data), "edus_slot_set")

    def slot_get(self, slot):
        a = self._state_buf()
        _check(self._L.edus_slot_get(self._h, int(slot), a.ctypes.data), "edus_slot_get")
        return a

    def runge_kutta_ad(self, src, dst, dt):
        _check(self._L.edus_runge_kutta_ad(self._h, int(src), int(dst), float(dt)), "edus_runge_kutta_ad")

    def runge_kutta_ac(self, dst, dt):
        _check(self._L.edus_runge_kutta_ac(self._h, int(dst), float(dt)), "edus_runge_kutta_ac")

    def coulomb_hk(self, slot):
        a = self._state_buf()
        _check(self._L.edus_coulomb_hk(self._h, int(slot), a.ctypes.data), "edus_coulomb_hk")
        return a

    def close(self):
        if self._h:
            self._L.edus_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _tuned(precision):
    """Tile lengths and register profiles of the autotuner's cache for this GPU."""
    from . import autotune

    return autotune.tuned_options(precision)


class Batch:
    """Many solves advanced together on one GPU (edus_batch_* of the C ABI)."""

    def __init__(self, device=0, precision=abi.EDUS_PREC_FP64, max_instances=1024, chunk_steps=16, use_graphs=True,
                 hbm_budget_bytes=0, tile_k=None, regs_profile=None, tuned=True, tc_contraction=True):
        L = load_library()
        if tuned and tile_k is None and regs_profile is None:
            tile_k, regs_profile = _tuned(precision)
        self._L = L
        o = abi.BatchOptions()
        _check(L.edus_batch_options_default(C.byref(o)), "edus_batch_options_default")
        o.device = device
        o.precision = precision
        o.max_instances = max_instances
        o.chunk_steps = chunk_steps
        o.use_graphs = 1 if use_graphs else 0
        o.hbm_budget_bytes = int(hbm_budget_bytes)
        for n, k in (tile_k or {}).items():
            o.tile_k[n] = k
        for n, r in (regs_profile or {}).items():
            o.regs_profile[n] = r
        o.tc_contraction = 1 if tc_contraction else 0
        self._h = C.c_void_p()
        _check(L.edus_batch_create(C.byref(o), C.byref(self._h)), "edus_batch_create")
        self._n = {}
        self._nk = {}

    def footprint(self, problem):
        b = C.c_int64()
        _check(self._L.edus_batch_footprint(self._h, problem._h, C.byref(b)), "edus_batch_footprint")
        return b.value

    def add(self, problem, tag=0):
        s = C.c_int32()
        _check(self._L.edus_batch_add(self._h, problem._h, int(tag), C.byref(s)), "edus_batch_add")
        self._n[s.value] = problem.info.ncv
        self._nk[s.value] = problem.info.nk
        return s.value

    def try_add(self, problem, tag=0):
        """Slot, or None when the HBM budget or the slots are used up."""
        s = C.c_int32()
        rc = self._L.edus_batch_add(self._h, problem._h, int(tag), C.byref(s))
        if rc == abi.EDUS_ENOMEM:
            return None
        _check(rc, "edus_batch_add")
        self._n[s.value] = problem.info.ncv
        self._nk[s.value] = problem.info.nk
        return s.value

    def advance(self, nsteps):
        _check(self._L.edus_batch_advance(self._h, int(nsteps)), "edus_batch_advance")

    def poll(self, slot):
        st, it, tag = C.c_int32(), C.c_int32(), C.c_int64()
        _check(self._L.edus_batch_poll(self._h, int(slot), C.byref(st), C.byref(it), C.byref(tag)), "edus_batch_poll")
        return st.value, it.value, tag.value

    def obs(self, slot):
        n = C.c_int32()
        _check(self._L.edus_batch_obs_count(self._h, int(slot), C.byref(n)), "edus_batch_obs_count")
        buf = (abi.Obs * max(n.value, 1))()
        if n.value:
            _check(self._L.edus_batch_obs_get(self._h, int(slot), 0, n.value, buf), "edus_batch_obs_get")
        return [abi.obs_to_dict(buf[i], self._n[slot]) for i in range(n.value)]

    def get_state(self, slot):
        n, nk = self._n[slot], self._nk[slot]
        a = np.zeros((nk, n, n), dtype=np.complex128)
        _check(self._L.edus_batch_get_state(self._h, int(slot), a.ctypes.data), "edus_batch_get_state")
        return a

    def release(self, slot):
        _check(self._L.edus_batch_release(self._h, int(slot)), "edus_batch_release")
        self._n.pop(slot, None)
        self._nk.pop(slot, None)

    def stats(self):
        s = abi.BatchStats()
        _check(self._L.edus_batch_stats_get(self._h, C.byref(s)), "edus_batch_stats_get")
        return {f: getattr(s, f) for f, _ in abi.BatchStats._fields_ if f != "pad"}

    def profile(self, nsteps):
        """Advance nsteps with a CUDA-event pair around every launch: list of
        {nbands, kind (0 observables, 1-4 RK4 stage 0-3), launches, total_ms, kpoints}."""
        cap = 64
        buf = (abi.KernelTime * cap)()
        n = C.c_int32()
        _check(self._L.edus_batch_profile(self._h, int(nsteps), buf, cap, C.byref(n)), "edus_batch_profile")
        return [{f: getattr(buf[i], f) for f, _ in abi.KernelTime._fields_} for i in range(n.value)]

    def tile_k(self, nbands):
        k = C.c_int32()
        _check(self._L.edus_batch_tile_k(self._h, int(nbands), C.byref(k)), "edus_batch_tile_k")
        return k.value

    def close(self):
        if self._h:
            self._L.edus_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Request loop over one batch (edus_server_* of the C ABI): submit solves at
    any time; they are admitted by HBM footprint and run concurrently."""

    def __init__(self, device=0, precision=abi.EDUS_PREC_FP64, max_instances=1024, chunk_steps=16,
                 hbm_budget_bytes=0, setup_threads=4, drop_decoupled_core=True, max_bypass_s=2.0, tile_k=None,
                 regs_profile=None, tuned=True, trace_tol=None):
        L = load_library()
        if tuned and tile_k is None and regs_profile is None:
            tile_k, regs_profile = _tuned(precision)
        self._L = L
        o = abi.ServerOptions()
        _check(L.edus_server_options_default(C.byref(o)), "edus_server_options_default")
        o.batch.device = device
        o.batch.precision = precision
        o.batch.max_instances = max_instances
        o.batch.chunk_steps = chunk_steps
        o.batch.hbm_budget_bytes = int(hbm_budget_bytes)
        for n, k in (tile_k or {}).items():
            o.batch.tile_k[n] = k
        for n, r in (regs_profile or {}).items():
            o.batch.regs_profile[n] = r
        o.setup_threads = setup_threads
        o.drop_decoupled_core = 1 if drop_decoupled_core else 0
        o.max_bypass_s = max_bypass_s
        if trace_tol is not None:
            o.trace_tol = trace_tol
        self._h = C.c_void_p()
        _check(L.edus_server_create(C.byref(o), C.byref(self._h)), "edus_server_create")
        self._keep = {}

    def submit(self, params, workdir="."):
        rid = C.c_int64()
        _check(self._L.edus_server_submit(self._h, C.byref(params), os.fsencode(workdir), C.byref(rid)), "edus_server_submit")
        self._keep[rid.value] = params
        return rid.value

    def info(self, rid):
        o = abi.RequestInfo()
        _check(self._L.edus_server_info(self._h, int(rid), C.byref(o)), "edus_server_info")
        return {f: getattr(o, f) for f, _ in abi.RequestInfo._fields_}

    def failure(self, rid):
        """(error code, message) of a failed request, else None."""
        i = self.info(rid)
        if i["status"] != abi.EDUS_REQ_FAILED:
            return None
        return i["error"], self._L.edus_last_error().decode(errors="replace")

    def obs(self, rid):
        i = self.info(rid)
        if i["status"] == abi.EDUS_REQ_FAILED:
            msg = self._L.edus_last_error().decode(errors="replace")
            raise EdusError(i["error"], "edus_server_obs", msg)
        buf = (abi.Obs * max(i["nobs"], 1))()
        if i["nobs"]:
            _check(self._L.edus_server_obs(self._h, int(rid), 0, i["nobs"], buf), "edus_server_obs")
        return [abi.obs_to_dict(buf[q], i["nbands"]) for q in range(i["nobs"])]

    def forget(self, rid):
        _check(self._L.edus_server_forget(self._h, int(rid)), "edus_server_forget")
        self._keep.pop(rid, None)

    def drain(self, timeout_s=600.0):
        _check(self._L.edus_server_drain(self._h, float(timeout_s)), "edus_server_drain")

    def stats(self):
        s = abi.ServerStats()
        _check(self._L.edus_server_stats_get(self._h, C.byref(s)), "edus_server_stats_get")
        return {f: getattr(s, f) for f, _ in abi.ServerStats._fields_ if f != "pad"}

    def clock(self):
        return self._L.edus_server_clock(self._h)

    def close(self):
        if self._h:
            self._L.edus_server_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
