"""McMD weight iteration (GEprep distrib_MULT + lstsquare_final) on the host: the library's
jp_ge_fit / jp_lstsq_windows against the numpy restatement in oracle/ge_fit.py, and both
against closed-form cases.  No GPU needed.

Tolerances: both restatements evaluate every sum and product in the reference's sequential
order (integer powers as successive products, matmul as column-order loops), so fitted
values agree to 1e-12 relative even though the degree-8 normal equations (power sums up to
dx^16) would amplify reordered rounding to ~1e-6; coefficients are compared through the
function they define.
"""
import numpy as np
import pytest

from oracle import ge_fit as ora
from j_presto_b200 import systems

R_KCAL = 8.31451 / 4.184 * 1e-3


def poly_eval(coef, low, high, x):
    """Windowed polynomial at x (window search as md_run's verlethe)."""
    out = np.empty_like(x)
    for n, xv in enumerate(x):
        j = 0
        while j != len(low) - 1 and xv >= high[j]:
            j += 1
        out[n] = np.polynomial.polynomial.polyval(xv - low[j], coef[j])
    return out


@pytest.fixture(scope="module")
def eng(engine_lib):
    from j_presto_b200 import engine
    return engine


@pytest.mark.parametrize("nwindow", [1, 3])
def test_exact_polynomial_is_recovered(eng, nwindow):
    """A global polynomial of the fitted degree satisfies every continuity condition and has
    zero residual, so every window must reproduce it."""
    rng = np.random.default_rng(3)
    x = np.sort(rng.uniform(0.0, 1.0, 240))
    c = np.array([1.5, -2.0, 0.7, 3.0, -1.2, 0.4])
    y = np.polynomial.polynomial.polyval(x, c)
    w = rng.uniform(0.5, 3.0, len(x))
    for fit in (lambda: eng.lstsq_windows(x, y, w, nwindow, 5)[:3],
                lambda: ora.lstsquare_final(nwindow, 5, 0.0, 1.0, x, y, w)[:3]):
        coef, low, high = fit()
        np.testing.assert_allclose(poly_eval(coef, low, high, x), y, rtol=0, atol=1e-8)


def test_lstsq_windows_matches_oracle(eng):
    rng = np.random.default_rng(5)
    x = np.sort(rng.uniform(0.0, 1.0, 300))
    y = 1.0 / (R_KCAL * (280.0 + 420.0 * x)) + 0.02 * rng.normal(size=len(x))
    w = np.sqrt(rng.integers(1, 400, len(x)).astype(float))
    coef, low, high, res = eng.lstsq_windows(x, y, w, 3, 8)
    co, lo, hi, ro = ora.lstsquare_final(3, 8, 0.0, 1.0, x, y, w)
    np.testing.assert_array_equal(low, lo)
    np.testing.assert_array_equal(high, hi)
    np.testing.assert_allclose(poly_eval(coef, low, high, x), poly_eval(co, lo, hi, x), rtol=1e-12)
    np.testing.assert_allclose(res[0], ro[0], rtol=1e-12)


def _mcmd_histogram(old, emin, emax, nbin, nbor, t_lo=280.0, t_hi=700.0, nsamp=2.0e6):
    """Expected counts of a McMD run: P(E) ~ n(E) exp(-W(E)), with d ln n/dE = 1/(R T(E)),
    T linear on [emin, emax], sampled with the weight `old` (its d W/dE = P_old)."""
    de = (emax - emin) / nbin
    e = emin - de * nbor + de * (np.arange(nbin + 2 * nbor) + 0.5)
    fine = np.linspace(e[0], e[-1], 20001)
    xt = np.clip((fine - emin) / (emax - emin), 0.0, 1.0)
    dlnn = 1.0 / (R_KCAL * (t_lo + (t_hi - t_lo) * xt))
    xo = (fine - old["celw"]) / (old["ceup"] - old["celw"])
    dw = np.array([ora.poly_old(old, v) for v in xo])
    g = np.concatenate([[0.0], np.cumsum(0.5 * (dlnn[1:] + dlnn[:-1] - dw[1:] - dw[:-1]) * np.diff(fine))])
    lnp = np.interp(e, fine, g)
    p = np.exp(lnp - lnp.max())
    return np.round(nsamp * p / p.sum())


def test_ge_fit_matches_oracle_and_converges(eng):
    emin, emax, nbin, nbor = -1000.0, 2000.0, 150, 10
    old = systems.mcmd_weight(emin, emax, ndeg=8, t_lo=330.0, t_hi=620.0)
    hist = _mcmd_histogram(old, emin, emax, nbin, nbor)
    args = (hist, old, emin, emax, nbin, nbor, emin, emax, 300.0, 2, 8)
    nf, res = eng.ge_fit(*args)
    nfo, reso = ora.ge_fit(*args)
    x = np.linspace(0.0, 1.0, 101)
    f = poly_eval(nf["coef"], nf["low"], nf["high"], x)
    np.testing.assert_allclose(f, poly_eval(nfo["coef"], nfo["low"], nfo["high"], x), rtol=1e-12)
    for k in ("alphalw", "alphaup"):
        np.testing.assert_allclose(nf[k], nfo[k], rtol=1e-12)
    assert (nf["celw"], nf["ceup"], nf["tempce"]) == (emin, emax, 300.0)
    # where the run sampled (>= 100 counts), one iteration moves the weight from the guess
    # (330-620 K) to the true 280-700 K law; outside it the reference method extrapolates
    X, _, W = ora.dlnn_data(hist, old, emin, emax, nbin, nbor, emin, emax)
    xs = X[(W >= 10.0) & (X >= 0.0) & (X <= 1.0)]
    assert len(xs) > 20
    true = 1.0 / (R_KCAL * (280.0 + 420.0 * xs))
    new_err = np.abs(poly_eval(nf["coef"], nf["low"], nf["high"], xs) - true).max()
    old_err = np.abs(poly_eval(old["coef"], old["low"], old["high"], xs) - true).max()
    assert new_err < 0.1 * old_err


def test_flat_histogram_is_a_fixed_point(eng):
    """A converged (flat) multicanonical histogram leaves the weight where it was."""
    emin, emax, nbin, nbor = -500.0, 500.0, 120, 0
    old = systems.mcmd_weight(emin, emax, ndeg=6)
    hist = np.full(nbin, 5000.0)
    nf, _ = eng.ge_fit(hist, old, emin, emax, nbin, nbor, emin, emax, 300.0, 1, 6)
    x = np.linspace(0.02, 0.98, 50)
    np.testing.assert_allclose(poly_eval(nf["coef"], nf["low"], nf["high"], x),
                               poly_eval(old["coef"], old["low"], old["high"], x), rtol=2e-4)


def test_ge_fit_rejects_bad_input(eng):
    old = systems.mcmd_weight(0.0, 1.0)
    with pytest.raises(eng.JpError):
        eng.ge_fit(np.zeros(20), old, 0.0, 1.0, 20, 0, 0.0, 1.0, 300.0, 1, 4)   # empty histogram
    with pytest.raises(eng.JpError):
        eng.ge_fit(np.ones(20), old, 0.0, 1.0, 20, 0, 0.0, 1.0, 300.0, 20, 15)  # too few points
