"""ctypes mirror of include/edus_b200.h (structs, enums, error codes).

Kept field-for-field identical to the C header; tests check the sizes
against the library's own sizeof values.
"""
import ctypes as C

EDUS_OK = 0
EDUS_EINVAL = -1
EDUS_ENOMEM = -2
EDUS_ECUDA = -3
EDUS_ENONFINITE = -4
EDUS_ETRACE = -5
EDUS_ETIMEOUT = -6
EDUS_ECANCELLED = -7
EDUS_EIO = -8
EDUS_EPARSE = -9
EDUS_EUNSUPPORTED = -10
EDUS_ENOTREADY = -11

EDUS_MODE_TB = 1
EDUS_MODE_WANNIER = 2
EDUS_MODE_CRYSTAL = 3
EDUS_SOLVER_RK4 = 0
EDUS_SOLVER_AB = 1
EDUS_SOLVER_TAYLOR = 2
EDUS_ENV_NONE = 0
EDUS_ENV_SIN2 = 1
EDUS_ENV_GAUSS = 2
EDUS_ENV_PW = 3
EDUS_PREC_FP64 = 0
EDUS_PREC_MIXED = 1

EDUS_MAX_PUMPS = 8
EDUS_MAX_TABSK = 64
EDUS_MAX_HOPPING = 8
EDUS_MAX_BANDS = 16
EDUS_STRLEN = 256

SLOT_P0, SLOT_P1, SLOT_P2, SLOT_PV = 0, 1, 2, 3


class Laser(C.Structure):
    _fields_ = [
        ("envelope_kind", C.c_int32),
        ("envelope_only", C.c_int32),
        ("wl", C.c_double),
        ("period", C.c_double),
        ("lambdanm", C.c_double),
        ("intensity", C.c_double),
        ("A0", C.c_double),
        ("E0", C.c_double),
        ("t0", C.c_double),
        ("tf", C.c_double),
        ("ncycle", C.c_double),
        ("sigma", C.c_double),
        ("w1", C.c_double),
        ("w2", C.c_double),
        ("phase", C.c_double),
        ("pol1", C.c_double * 3),
        ("pol2", C.c_double * 3),
    ]


class Params(C.Structure):
    _fields_ = [
        ("ref_coord", C.c_char * EDUS_STRLEN),
        ("mode", C.c_int32),
        ("tb_type", C.c_char * 64),
        ("hopping", C.c_double * EDUS_MAX_HOPPING),
        ("n_hopping", C.c_int32),
        ("a", (C.c_double * 3) * 3),
        ("b", (C.c_double * 3) * 3),
        ("nk", C.c_int32 * 3),
        ("nb", C.c_int32 * 3),
        ("conduction_shift", C.c_double),
        ("fermi_energy", C.c_double),
        ("dt", C.c_double),
        ("t_fin", C.c_double),
        ("solver", C.c_int32),
        ("order", C.c_int32),
        ("dynamical_dt", C.c_int32),
        ("eps_step_abs", C.c_double),
        ("ab_rk4_startup", C.c_int32),
        ("gap_correction", C.c_double),
        ("n_pumps", C.c_int32),
        ("pump", Laser * EDUS_MAX_PUMPS),
        ("probe", Laser),
        ("delay", C.c_double),
        ("T1", C.c_double),
        ("T2", C.c_double),
        ("Tch", C.c_double),
        ("current", C.c_int32),
        ("tabs", C.c_int32),
        ("it_resolution", C.c_int32),
        ("print_population", C.c_int32),
        ("print_start", C.c_double),
        ("print_end", C.c_double),
        ("print_step", C.c_double),
        ("coulomb", C.c_int32),
        ("ncut", C.c_int32),
        ("qTF", C.c_double),
        ("r0", C.c_double),
        ("epsilon_static", C.c_double),
        ("G_distance", C.c_double),
        ("rytova_keldysh", C.c_int32),
        ("diag_basis", C.c_int32),
        ("read_from_files", C.c_int32),
        ("print_band_dispersion", C.c_int32),
        ("coulomb_label", C.c_char * EDUS_STRLEN),
        ("sample_110", C.c_int32),
        ("vectorization", C.c_int32),
        ("precision", C.c_int32),
        ("tabs_k", C.c_int32),
        ("n_tabs_k", C.c_int32),
        ("tabs_k_pts", (C.c_double * 3) * EDUS_MAX_TABSK),
        ("kpt_read", C.c_int32),
        ("kpt_offset", C.c_int64),
        ("input_path", C.c_char * EDUS_STRLEN),
        ("velocity_gauge", C.c_int32),
    ]


class Obs(C.Structure):
    _fields_ = [
        ("t", C.c_double),
        ("EF_pump", C.c_double * 3),
        ("EF_probe", C.c_double * 3),
        ("J1", C.c_double * 6),
        ("J2", C.c_double * 3),
        ("pop", C.c_double * EDUS_MAX_BANDS),
        ("tabs", C.c_double * 6),
        ("trace_dev", C.c_double),
        ("p_cond_max", C.c_double),
        ("p_min", C.c_double),
        ("n_cond", C.c_double),
        ("dt", C.c_double),
        ("pol", C.c_double * 6),
    ]


class ProblemInfo(C.Structure):
    _fields_ = [
        ("ncv", C.c_int32),
        ("nch", C.c_int32),
        ("nv", C.c_int32),
        ("nc", C.c_int32),
        ("nk", C.c_int32),
        ("n1", C.c_int32),
        ("n2", C.c_int32),
        ("nshell", C.c_int32),
        ("nnb", C.c_int32),
        ("nrpts", C.c_int32),
        ("n_diss", C.c_int32),
        ("nsteps", C.c_int32),
        ("nprint", C.c_int32),
        ("t_start", C.c_double),
        ("det_a", C.c_double),
        ("jacobian", C.c_double),
        ("dk", C.c_double * 3),
    ]


class Options(C.Structure):
    _fields_ = [
        ("device", C.c_int32),
        ("precision", C.c_int32),
        ("use_graphs", C.c_int32),
        ("health_checks", C.c_int32),
        ("trace_tol", C.c_double),
        ("hbm_budget_bytes", C.c_int64),
    ]


def obs_to_dict(o, ncv):
    import numpy as np

    return {
        "t": o.t,
        "EF_pump": np.array(o.EF_pump[:]),
        "EF_probe": np.array(o.EF_probe[:]),
        "J1": np.array(o.J1[0::2]) + 1j * np.array(o.J1[1::2]),
        "J2": np.array(o.J2[:]),
        "pop": np.array(o.pop[:ncv]),
        "tabs": np.array(o.tabs[0::2]) + 1j * np.array(o.tabs[1::2]),
        "trace_dev": o.trace_dev,
        "p_cond_max": o.p_cond_max,
        "p_min": o.p_min,
        "n_cond": o.n_cond,
        "dt": o.dt,
        "pol": np.array(o.pol[0::2]) + 1j * np.array(o.pol[1::2]),
    }


class BatchOptions(C.Structure):
    _fields_ = [
        ("device", C.c_int32),
        ("precision", C.c_int32),
        ("max_instances", C.c_int32),
        ("chunk_steps", C.c_int32),
        ("use_graphs", C.c_int32),
        ("tile_k", C.c_int32 * (EDUS_MAX_BANDS + 1)),
        ("regs_profile", C.c_int32 * (EDUS_MAX_BANDS + 1)),
        ("tc_contraction", C.c_int32),
        ("pad", C.c_int32),
        ("hbm_budget_bytes", C.c_int64),
    ]


class BatchStats(C.Structure):
    _fields_ = [
        ("ticks", C.c_int64),
        ("active", C.c_int32),
        ("done", C.c_int32),
        ("free_slots", C.c_int32),
        ("pad", C.c_int32),
        ("bytes_used", C.c_int64),
        ("bytes_budget", C.c_int64),
        ("device_ms", C.c_double),
        ("kpoint_steps", C.c_double),
        ("launches", C.c_int64),
        ("h2d_bytes", C.c_int64),
        ("d2h_bytes", C.c_int64),
    ]


class KernelTime(C.Structure):
    _fields_ = [
        ("nbands", C.c_int32),
        ("kind", C.c_int32),
        ("launches", C.c_int64),
        ("total_ms", C.c_double),
        ("kpoints", C.c_int64),
    ]


EDUS_INST_FREE, EDUS_INST_RUNNING, EDUS_INST_DONE = 0, 1, 2


class ServerOptions(C.Structure):
    _fields_ = [
        ("batch", BatchOptions),
        ("setup_threads", C.c_int32),
        ("drop_decoupled_core", C.c_int32),
        ("max_bypass_s", C.c_double),
        ("trace_tol", C.c_double),
    ]


class CoulombGenOptions(C.Structure):
    _fields_ = [("device", C.c_int32), ("n_sum", C.c_int32), ("n_sum_screen", C.c_int32)]


class RequestInfo(C.Structure):
    _fields_ = [
        ("status", C.c_int32),
        ("error", C.c_int32),
        ("nbands", C.c_int32),
        ("nobs", C.c_int32),
        ("nk", C.c_int64),
        ("steps", C.c_int64),
        ("footprint_bytes", C.c_int64),
        ("t_submit", C.c_double),
        ("t_ready", C.c_double),
        ("t_admit", C.c_double),
        ("t_done", C.c_double),
    ]


class ServerStats(C.Structure):
    _fields_ = [
        ("submitted", C.c_int64),
        ("completed", C.c_int64),
        ("failed", C.c_int64),
        ("running", C.c_int64),
        ("waiting", C.c_int64),
        ("span_s", C.c_double),
        ("solves_per_s", C.c_double),
        ("kpoint_steps_per_s", C.c_double),
        ("p50_latency_s", C.c_double),
        ("p99_latency_s", C.c_double),
        ("max_latency_s", C.c_double),
        ("device_ms", C.c_double),
        ("peak_bytes", C.c_int64),
        ("peak_active", C.c_int32),
        ("pad", C.c_int32),
    ]


EDUS_REQ_QUEUED, EDUS_REQ_SETUP, EDUS_REQ_READY, EDUS_REQ_RUNNING, EDUS_REQ_DONE, EDUS_REQ_FAILED = range(6)
