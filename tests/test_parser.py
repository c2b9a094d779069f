"""input.txt reader (headers/ReadInput.h grammar) against the reference's own
printout of the shipped AB5 run (example/.../output.log:60-110) and unit rules."""
import math

import pytest

import edus_b200 as E
from edus_b200 import abi
from conftest import GOLDEN_INPUT

EV = 1 / 27.211396
FS = 1 / 0.02418884326505


def test_golden_input_fields():
    p = E.parse_input(GOLDEN_INPUT)
    assert p.ref_coord == b"NEWINPUT"
    assert p.mode == abi.EDUS_MODE_TB and p.tb_type == b"Haldane_CoreBN_Nedge"
    assert list(p.nk) == [1, 70, 70] and list(p.nb) == [1, 1, 1]
    assert p.hopping[0] == pytest.approx(7.25 * EV, rel=1e-15)
    assert p.hopping[1] == pytest.approx(-2.3 * EV, rel=1e-15)
    assert p.dt == 0.1 and p.t_fin == pytest.approx(1650.36549334624544)
    assert p.solver == abi.EDUS_SOLVER_AB and p.order == 5 and not p.ab_rk4_startup
    assert p.it_resolution == 5 and p.current and p.tabs
    assert p.Tch == pytest.approx(0.00396892)
    # output.log: pump Energy 0.25713 au, A0 1.46786e-03, E0 3.77426e-04, tf 1.71053e+02
    pu = p.pump[0]
    assert pu.wl == pytest.approx(0.25713, abs=5e-6)
    assert pu.A0 == pytest.approx(1.46786e-03, rel=1e-5)
    assert pu.E0 == pytest.approx(3.77426e-04, rel=1e-5)
    assert pu.t0 == 0 and pu.tf == pytest.approx(1.71053e02, rel=1e-5)
    assert list(pu.pol1) == [0, 1, 0] and list(pu.pol2) == [0, 0, 1]
    # probe: E0 1.68790e-05, t0 8.48367e+01, tf 8.62165e+01, sigma 0.08 fs
    pr = p.probe
    assert pr.envelope_kind == abi.EDUS_ENV_GAUSS and pr.envelope_only
    assert pr.E0 == pytest.approx(1.68790e-05, rel=1e-5)
    assert pr.t0 == pytest.approx(8.48367e01, rel=1e-5)
    assert pr.tf == pytest.approx(8.62165e01, rel=1e-5)
    assert pr.sigma == pytest.approx(0.08 * FS, rel=1e-15)
    # unit cell area 19.329 (output.log:6)
    a = p.a
    assert abs(a[1][1] * a[2][2] - a[1][2] * a[2][1]) == pytest.approx(19.329, rel=1e-4)


def _write(tmp_path, text):
    f = tmp_path / "input.txt"
    f.write_text(text)
    return str(f)


BASE = """X
tdse{{
tightbinding Haldane_CoreBN_Nedge gap= 5 t1= 2 t2= 0 phi0= 0
{tdse}
}}
nkpt{{
1 12 12
}}
{extra}
"""


def test_units_and_defaults(tmp_path):
    pump = "laserpump sin2 {\ncycles 3\nt0_pulse 2.0 fs\nfrequency 0.0147\nintensity 1e12 wcm2\npolarization circular 0 1 1 0 1 0\n}\n"
    p = E.parse_input(_write(tmp_path, BASE.format(tdse="dt 0.01 fs", extra=pump)))
    assert p.dt == pytest.approx(0.01 * FS)
    L = p.pump[0]
    # t0 is applied last: tf = t0 + cycles * period
    assert L.t0 == pytest.approx(2.0 * FS)
    assert L.tf == pytest.approx(2.0 * FS + 3 * 2 * math.pi / 0.0147)
    # circular polarisation: Gram-Schmidt of (0,1,0) against (0,1,1)/sqrt2
    p1, p2 = list(L.pol1), list(L.pol2)
    assert abs(sum(x * y for x, y in zip(p1, p2))) < 1e-12
    assert math.isclose(sum(x * x for x in p2), 1.0, rel_tol=1e-12)
    # default final time: the pump duration rounded down to whole steps (runge_kutta_init.cpp)
    nstep = int(3 * L.period / p.dt)
    assert p.t_fin == pytest.approx(nstep * p.dt)
    assert p.tabs == 1 and p.it_resolution == 10 and p.ncut == 30  # variables.cpp defaults


def test_order_dependent_laser_setters(tmp_path):
    # cycles before the frequency: tf is set when the frequency arrives
    a = "laserpump sin2 {\ncycles 2\nfrequency 0.02\nintensity 1e11\npolarization 0 0 1\n}\n"
    b = "laserpump sin2 {\nfrequency 0.02\nintensity 1e11\ncycles 2\npolarization 0 0 1\n}\n"
    pa = E.parse_input(_write(tmp_path, BASE.format(tdse="dt 0.1", extra=a)))
    pb = E.parse_input(_write(tmp_path, BASE.format(tdse="dt 0.1", extra=b)))
    assert pa.pump[0].tf == pytest.approx(pb.pump[0].tf)
    assert pa.pump[0].E0 == pytest.approx(math.sqrt(1e11 / 3.51e16))


def test_solver_keys(tmp_path):
    p = E.parse_input(_write(tmp_path, BASE.format(tdse="dt 0.1\nTaylor\nTaylorOrder 6\ndynamical_dt_evolution\nepsStepAbs 0.02", extra="")))
    assert p.solver == abi.EDUS_SOLVER_TAYLOR and p.order == 6 and p.dynamical_dt and p.eps_step_abs == 0.02
    p = E.parse_input(_write(tmp_path, BASE.format(tdse="dt 0.1\nAdams_Bashforth 9", extra="")))
    assert p.solver == abi.EDUS_SOLVER_AB and p.order == 5  # capped at 5 as in ReadInput.h:557-559


def test_coulomb_and_decoherence(tmp_path):
    extra = ("Coulomb{\nqTF 0.01\nNcut 20\n# G_distance 400\nRead_Coulomb_from_files\nlabelInput G_num1_\nRytova_Keldysh\n}\n"
             "decoherence{\ncorehole 100 meV\ndiagonal 0.001 au\n}\n")
    p = E.parse_input(_write(tmp_path, BASE.format(tdse="dt 0.1", extra=extra)))
    assert p.coulomb and p.ncut == 20 and p.read_from_files and p.rytova_keldysh
    assert p.coulomb_label == b"G_num1_" and p.qTF == 0.01
    assert p.Tch == pytest.approx(0.1 * EV) and p.T1 == 0.001


@pytest.mark.parametrize(
    "extra,code",
    [
        ("observables{\nnot_a_key\n}\n", abi.EDUS_EPARSE),
        ("this line has no brace\n", abi.EDUS_EPARSE),
        ("decoherence{\ncorehole 1 furlongs\n}\n", abi.EDUS_EPARSE),
        ("laserpump sin2 {\nsigma 2\n}\n", abi.EDUS_EPARSE),
        ("laserpump sin2 {\npolarization linear 0 0 1\n}\n", abi.EDUS_EPARSE),
        ("TAbsK{\n1\n0 0.1 0.2\n}\nobservables{\nkTAbs\n}\n", abi.EDUS_EPARSE),
        ("observables{\nkTAbs\n}\nTAbsK{\n2 3\n}\n", abi.EDUS_EPARSE),
        ("observables{\nkTAbs\n}\nTAbsK{\n2\n0 0.1 0.2\n0 0.3\n}\n", abi.EDUS_EPARSE),
        ("observables{\nkTAbs\n}\nTAbsK{\n65\n}\n", abi.EDUS_EUNSUPPORTED),
    ],
)
def test_errors_are_codes_not_exits(tmp_path, extra, code):
    with pytest.raises(E.EdusError) as ei:
        E.parse_input(_write(tmp_path, BASE.format(tdse="dt 0.1", extra=extra)))
    assert ei.value.code == code


def test_tabsk_section(tmp_path):
    """headers/ReadInput.h:1032, 1047-1083: kTAbs in the observables, then the
    TAbsK section with the number of k points and one point per line."""
    extra = "observables{\nCurrent\nkTAbs\n}\nTAbsK{\n\n2\n0 0.1 0.2\n0 -0.25 0.5\n}\n"
    p = E.parse_input(_write(tmp_path, BASE.format(tdse="dt 0.1", extra=extra)))
    assert p.tabs_k == 1 and p.n_tabs_k == 2 and p.current == 1
    assert [list(p.tabs_k_pts[i]) for i in range(2)] == [[0.0, 0.1, 0.2], [0.0, -0.25, 0.5]]


def test_missing_file():
    with pytest.raises(E.EdusError) as ei:
        E.parse_input("/nonexistent/input.txt")
    assert ei.value.code == abi.EDUS_EIO
