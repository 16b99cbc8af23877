"""md_run's McMD / ALSD weight file (.nf, read by inmcmd.f90:21-38) written and read by the
host (no GPU)."""
import numpy as np

from j_presto_b200 import ge


def _nf():
    return dict(coef=np.array([[1.25, -0.5, 1e-3], [0.75, 0.125, -2e-4]]), low=np.array([0.0, 0.4]),
                high=np.array([0.4, 1.0]), alphalw=1.2, alphaup=0.9, celw=-5000.0, ceup=-3000.0,
                tempce=300.0, lower=20.0, upper=15.0)


def test_round_trip_and_line_layout(tmp_path):
    p = tmp_path / "w.nf"
    ge.write_nf(p, _nf(), alsd=True)
    lines = p.read_text().splitlines()
    # nwindow ndeg; 3 coefficients + bounds per window; alphas; range; T0; ALSD walls
    assert lines[0].split() == ["2", "2"] and len(lines) == 1 + 2 * 4 + 3 + 1
    assert float(lines[4].split()[1]) == 0.4 and float(lines[-1].split()[0]) == 20.0
    nf = ge.read_nf(p, alsd=True)
    ref = _nf()
    for k in ("coef", "low", "high"):
        np.testing.assert_array_equal(nf[k], ref[k])
    for k in ("alphalw", "alphaup", "celw", "ceup", "tempce", "lower", "upper"):
        assert nf[k] == ref[k]


def test_reads_fortran_style_numbers(tmp_path):
    """List-directed input: extra values on a line are ignored, D exponents accepted."""
    p = tmp_path / "f.nf"
    p.write_text("1 1 ! one window\n 0.5D+00\n -1.0d-1\n 0.0 1.0\n 1.0 2.0\n -1.0D3 1.0D3\n 300.0\n")
    nf = ge.read_nf(p)
    np.testing.assert_allclose(nf["coef"], [[0.5, -0.1]])
    assert (nf["celw"], nf["ceup"], nf["tempce"]) == (-1000.0, 1000.0, 300.0)
