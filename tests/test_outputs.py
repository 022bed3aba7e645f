"""Result extraction (Outputs.jl): polarisation basis changes, derived outputs and the
@outputs-style request parsing, on results of the oracle's analyze (CPU)."""
import cmath
import math

import numpy as np
import pytest

import oracle
from pssfss_b200.elements import diagstrip, rectstrip
from pssfss_b200.layers import Layer
from pssfss_b200.outputs import (H, L, R, TE, TM, V, extract_result, getsijmn, obsmat, outputs,
                                 sourcemat, theta_phi)
from pssfss_b200.units import Length, mm

NORMAL = {"θ": 0.0, "ϕ": 0.0}


@pytest.fixture(scope="module")
def patch_result():
    sh = rectstrip(Lx=6, Ly=6, Px=10, Py=10, Nx=6, Ny=6, units=mm)
    return oracle.analyze([Layer(), sh, Layer(epsr=2.2, width=Length(1, mm)), Layer()], [12.0], NORMAL)[0]


def test_basis_changes_at_normal_incidence(patch_result):
    r = patch_result
    S = lambda i, j, m, n: getsijmn(i, j, m, n, r)
    # with ϕ = 0 the Ludwig-3 horizontal field is the TM mode's and the vertical the TE mode's
    for i, j in ((1, 1), (2, 1), (1, 2), (2, 2)):
        assert S(i, j, H, H) == S(i, j, TM, TM) and S(i, j, V, V) == S(i, j, TE, TE)
    for mat in (sourcemat(1, R, r), sourcemat(2, L, r), obsmat(1, R, r), obsmat(2, H, r)):
        assert np.abs(mat.conj().T @ mat - np.eye(2)).max() < 1e-15
    # power of each incident wave in every basis, to the GSM's own unitarity
    g = np.block([[r.gsm[(1, 1)], r.gsm[(1, 2)]], [r.gsm[(2, 1)], r.gsm[(2, 2)]]])
    err = np.abs(g.conj().T @ g - np.eye(4)).max()
    for basis in ((TE, TM), (H, V), (R, L)):
        for n in basis:
            assert abs(sum(abs(S(i, 1, m, n)) ** 2 for i in (1, 2) for m in basis) - 1) <= 2 * err + 1e-12
    # a square patch treats both hands alike: transmission keeps the hand, reflection reverses it
    assert abs(abs(S(2, 1, R, R)) - abs(S(2, 1, TE, TE))) < 1e-3 and abs(S(2, 1, L, R)) < 1e-2
    assert abs(abs(S(1, 1, L, R)) - abs(S(1, 1, TE, TE))) < 1e-3 and abs(S(1, 1, R, R)) < 1e-2


def test_derived_outputs_and_extraction(patch_result):
    r = patch_result
    ops = outputs("FGHz", "theta", "phi", "s21db(te,te)", "S21ANG(TE,TE)", "s11mag(1,1)", "ar21db(h)",
                  "dipd21", "ΔIL21", "s21real(r,h)", "psi1")
    row = extract_result(r, ops)
    assert row.shape == (1, len(ops))
    s = getsijmn(2, 1, 1, 1, r)
    assert row[0, 0] == 12.0 and row[0, 1] == 0.0 and row[0, 2] == 0.0
    assert math.isclose(row[0, 3], 20 * math.log10(abs(s)), rel_tol=1e-14)
    assert math.isclose(row[0, 4], math.degrees(cmath.phase(s)), rel_tol=1e-14)
    assert math.isclose(row[0, 5], abs(getsijmn(1, 1, 1, 1, r)), rel_tol=1e-14)
    assert row[0, 6] > 30          # a square patch passes a linear wave nearly linear
    ratio = getsijmn(2, 1, 1, 1, r) / getsijmn(2, 1, 2, 2, r)
    assert math.isclose(row[0, 7], math.degrees(cmath.phase(ratio)), abs_tol=1e-12)
    assert math.isclose(row[0, 8], 10 * math.log10(abs(ratio) ** 2), abs_tol=1e-12)
    assert row[0, 9] == getsijmn(2, 1, R, H, r).real and math.isnan(row[0, 10])
    assert extract_result([r, r], ops).shape == (2, len(ops))
    with pytest.raises(ValueError):
        outputs("s21xx(te,te)")


def test_axial_ratio_of_a_diagonal_polariser():
    # a strip along the cell diagonal splits a horizontal wave into unequal, dephased
    # components along and across the strip: an elliptical transmitted wave
    d = diagstrip(P=10, w=1, orient=45, Nl=12, Nw=2, units=mm)
    r = oracle.analyze([Layer(), d, Layer()], [12.0], NORMAL)[0]
    ar_h, ar_v = extract_result(r, outputs("ar21db(h)", "ar21db(v)"))[0]
    assert 3 < ar_h < 20 and abs(ar_h - ar_v) < 0.1


def test_outlist_csv_and_result_file(patch_result, tmp_path):
    # analyze's file outputs: each outlist CSV gets a header of labels and a row per result;
    # a result file reads back to the same extracted numbers
    from pssfss_b200.outputs import extract_result_file, read_result_file, write_outlist
    ops = outputs("FGHz", "s21db(te,te)", "s11(h,h)")
    csv, res = tmp_path / "out.csv", tmp_path / "pssfss.res"
    write_outlist([patch_result, patch_result], [(str(csv), ops)], str(res))
    lines = csv.read_text().splitlines()
    assert lines[0] == "FGHZ,S21DB(TE,TE),S11(H,H)" and len(lines) == 3
    cells = lines[1].split(",")
    assert float(cells[0]) == 12.0 and float(cells[1]) == extract_result(patch_result, ops)[0, 1].real
    assert complex(cells[2].replace("im", "j")) == getsijmn(1, 1, H, H, patch_result)
    assert len(read_result_file(str(res))) == 2
    assert np.array_equal(extract_result_file(str(res), ops), extract_result([patch_result] * 2, ops))


def test_analysis_log_report(tmp_path):
    # the logfile of analyze: banner, the layer / sheet tables of report_layers_sheets
    # (PSSFSS.jl:706-745), skipped points, per-sheet timings; nothing without a file name
    from pssfss_b200.analyze import AnalysisLog, make_plan
    from pssfss_b200.elements import meander
    strata = [Layer(), meander(a=5, b=10, h=6, w1=0.3, w2=0.3, ntri=300, units=mm),
              Layer(epsr=2.2, tandel=0.001, width=Length(1, mm)), Layer()]
    plan = make_plan(strata, [8.0, 12.0], NORMAL)
    fn = str(tmp_path / "pssfss.log")
    log = AnalysisLog(fn)
    log.start()
    log.report(plan)
    log.skipped(plan, [8.0, 12.0])
    log.sheet_sweep(1, 2, {"fill": 1.5})
    log.finish()
    text = open(fn).read()
    assert "Starting pssfss_b200 analysis" in text and "exiting" in text
    assert "     2    1.0000  mm    2.20 0.0010    1.00 0.0000     0" in text
    assert "   1     1           meander   0.0  J    368   646   279     460   62556" in text
    assert "1.500 ms fill" in text and "Skipping" not in text
    quiet = AnalysisLog(None)
    quiet.start()
    quiet.report(plan)
    quiet.finish()


def test_psi_steering_equals_angle_steering():
    # steering by the incremental phase shifts (ψ₁, ψ₂) - the branch of getsttuple that the
    # reference leaves broken (PSSFSS.jl:612) - reproduces angle steering with the same β00
    sh = rectstrip(Lx=6, Ly=0.5, Px=8, Py=8, Nx=8, Ny=2, units=mm)
    strata = [Layer(), sh, Layer()]
    f, th, ph = 12.0, 25.0, 30.0
    k = 2 * math.pi * f * 1e9 / 299792458.0
    b00 = k * math.sin(math.radians(th)) * np.array([math.cos(math.radians(ph)), math.sin(math.radians(ph))])
    p = 8e-3  # cell period in metres
    psi = {"ψ₁": math.degrees(b00[0] * p), "ψ₂": math.degrees(b00[1] * p)}
    ra = oracle.analyze(strata, [f], {"θ": th, "ϕ": ph})[0]
    rp = oracle.analyze(strata, [f], psi)[0]
    assert np.allclose(rp.beta00, ra.beta00, rtol=1e-12)
    for key in ((1, 1), (1, 2), (2, 1), (2, 2)):
        assert np.abs(rp.gsm[key] - ra.gsm[key]).max() < 1e-9
    assert rp.steering == psi and math.isnan(extract_result(rp, outputs("theta"))[0, 0])
    th_rp, ph_rp = theta_phi(rp)   # the angles recovered from β00
    assert math.isclose(th_rp, th, rel_tol=1e-9) and math.isclose(ph_rp, ph, rel_tol=1e-9)
