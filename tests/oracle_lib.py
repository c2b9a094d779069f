"""ctypes wrapper of the CPU oracle (oracle/liboracle.so) for the tests.

The oracle is test infrastructure: it is only ever the checker here.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from edus_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "liboracle.so")
_L = None


def load():
    global _L
    if _L is not None:
        return _L
    src = os.path.join(ORACLE_DIR, "edus_oracle.c")
    if not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)
    L = C.CDLL(ORACLE_SO)
    vp, P = C.c_void_p, C.POINTER
    L.orc_create.argtypes = [P(abi.Params), C.c_char_p, P(vp)]
    L.orc_free.argtypes = [vp]
    L.orc_info.argtypes = [vp, P(abi.ProblemInfo)]
    L.orc_get.argtypes = [vp, C.c_char_p, vp, C.c_size_t]
    L.orc_set.argtypes = [vp, C.c_char_p, vp, C.c_size_t]
    L.orc_run.argtypes = [vp, C.c_int, P(abi.Obs), C.c_int, P(C.c_int)]
    L.orc_rhs.argtypes = [vp, vp, vp, P(C.c_double), C.c_double, C.c_int]
    L.orc_coulomb_hk.argtypes = [vp, vp, vp]
    L.orc_observables.argtypes = [vp, vp, P(abi.Obs)]
    L.orc_clock.argtypes = [vp, P(C.c_int), P(C.c_double), P(C.c_double)]
    L.orc_coulomb_generate.argtypes = [P(abi.Params), C.c_char_p, C.c_int, C.c_int, C.c_int, vp, vp, vp, vp, vp, vp,
                                       P(C.c_int)]
    _L = L
    return L


def coulomb_generate(params, workdir, what, n_sum=4999, n_sum_screen=39999):
    """The oracle's Coulomb coefficient generator (Source_Main/Fourier_Coulomb.cpp:95-500):
    dict of VH [n][n], A..D [ncut^2][n^2], screen [n^2] (complex) and g_num."""
    L = load()
    n = params.nb[0] + params.nb[1] + params.nb[2]
    nc = params.ncut * params.ncut * n * n
    A, B, Cc, D = (np.zeros(nc, np.complex128) for _ in range(4))
    sc = np.zeros(n * n, np.complex128)
    VH = np.zeros(n * n, np.float64)
    ng = C.c_int()
    rc = L.orc_coulomb_generate(C.byref(params), os.fsencode(workdir), int(what), int(n_sum), int(n_sum_screen),
                                A.ctypes.data, B.ctypes.data, Cc.ctypes.data, D.ctypes.data, sc.ctypes.data,
                                VH.ctypes.data, C.byref(ng))
    if rc != 0:
        raise RuntimeError(f"orc_coulomb_generate failed: {rc}")
    sh = (params.ncut * params.ncut, n * n)
    return {"VH": VH.reshape(n, n), "A": A.reshape(sh), "B": B.reshape(sh), "C": Cc.reshape(sh), "D": D.reshape(sh),
            "screen": sc, "g_num": ng.value}


class Oracle:
    def __init__(self, params, workdir="."):
        self.L = load()
        self.h = C.c_void_p()
        rc = self.L.orc_create(C.byref(params), os.fsencode(workdir), C.byref(self.h))
        if rc != 0:
            raise RuntimeError(f"orc_create failed: {rc}")
        self.info = abi.ProblemInfo()
        self.L.orc_info(self.h, C.byref(self.info))
        self.n = self.info.ncv
        self.nk = self.info.nk
        # adaptive dt shrinks the step: the output count is not known in advance
        self.dynamic = bool(params.dynamical_dt)

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
            "Hr": ((nk, n, n), np.complex128),
            "nbr": ((nk, i.nnb), np.int32),
            "bvec": ((i.nnb, 3), np.float64),
            "weights": ((i.nnb,), np.float64),
        }
        shp, dt = shapes[name]
        a = np.zeros(shp, dtype=dt)
        rc = self.L.orc_get(self.h, name.encode(), a.ctypes.data, a.nbytes)
        if rc != 0:
            raise RuntimeError(f"orc_get({name}) failed")
        return a

    def set(self, name, arr):
        a = np.ascontiguousarray(arr)
        rc = self.L.orc_set(self.h, name.encode(), a.ctypes.data, a.nbytes)
        if rc != 0:
            raise RuntimeError(f"orc_set({name}) failed")

    def run(self, max_steps=-1):
        res = max(self.L and 1, 1)
        cap = self.info.nprint + 4 if max_steps < 0 else max_steps + 4
        if self.dynamic and max_steps < 0:
            cap = 1 << 16
        cap = max(cap, 16)
        log = (abi.Obs * cap)()
        n = C.c_int()
        self.L.orc_run(self.h, int(max_steps), log, cap, C.byref(n))
        del res
        return [abi.obs_to_dict(log[i], self.n) for i in range(min(n.value, cap))]

    def rhs(self, P, EF, wx2, e_non0):
        P = np.ascontiguousarray(P, dtype=np.complex128)
        Pv = np.zeros_like(P)
        ef = (C.c_double * 6)(*[float(x) for x in np.asarray(EF).ravel()])
        self.L.orc_rhs(self.h, P.ctypes.data, Pv.ctypes.data, ef, float(wx2), int(e_non0))
        return Pv

    def coulomb_hk(self, P):
        P = np.ascontiguousarray(P, dtype=np.complex128)
        hk = np.zeros_like(P)
        rc = self.L.orc_coulomb_hk(self.h, P.ctypes.data, hk.ctypes.data)
        if rc != 0:
            raise RuntimeError("orc_coulomb_hk failed")
        return hk

    def observables(self, P):
        P = np.ascontiguousarray(P, dtype=np.complex128)
        o = abi.Obs()
        self.L.orc_observables(self.h, P.ctypes.data, C.byref(o))
        return abi.obs_to_dict(o, self.n)

    def clock(self):
        it, t, dt = C.c_int(), C.c_double(), C.c_double()
        self.L.orc_clock(self.h, C.byref(it), C.byref(t), C.byref(dt))
        return it.value, t.value, dt.value

    def close(self):
        if self.h:
            self.L.orc_free(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
