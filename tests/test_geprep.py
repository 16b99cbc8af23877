"""GEprep's McMD distribution step on the host (j_presto_b200/geprep.py, distrib_MULT.f90).

* with one run, run weight 1 and no acceleration it is the library's jp_ge_dlnn / jp_ge_fit
  (fit data equal, fitted weight equal to 1e-12);
* the flatness and the per-set quantities against values worked out by hand: run weights
  fw, flatness acceleration P = sum over sets of tP / flatness^accrat, the energy ranges of
  the sampled bins and of the bins with ln P >= -1.5, the TTPdist counts;
* a histogram sampled with exactly the right weight (flat) reproduces the weight, so `.et`
  recovers the weight's temperatures (280 K at E_min, 700 K at E_max to the polynomial's
  accuracy), and every output file is written in the reference's layout.
No GPU needed: the fit is the library's host function.
"""
import os

import numpy as np
import pytest

from j_presto_b200 import geprep, systems


@pytest.fixture(scope="module")
def eng(engine_lib):
    from j_presto_b200 import engine
    return engine


def _hist(rng, nab):
    h = rng.integers(0, 400, nab).astype(float)
    h[:3] = 0.0
    h[-2:] = 0.0
    return h


def test_one_run_equals_the_library_fit(eng):
    rng = np.random.default_rng(7)
    emin, emax, nbin, nbor = -1000.0, -600.0, 80, 4
    h = _hist(rng, nbin + 2 * nbor)
    old = systems.mcmd_weight(-1050.0, -550.0)
    res = geprep.iterate([h], old, emin, emax, nbin, nbor, -1020.0, -580.0, 300.0, nwindow=2, ndeg=6)
    x, y, w = eng.ge_dlnn(h, old, emin, emax, nbin, nbor, -1020.0, -580.0)
    X, Y, W = res["data"]
    np.testing.assert_array_equal(X, x)
    np.testing.assert_array_equal(Y, y)
    np.testing.assert_array_equal(W, w)
    nf, _ = eng.ge_fit(h, old, emin, emax, nbin, nbor, -1020.0, -580.0, 300.0, 2, 6)
    xs = np.linspace(0.0, 1.0, 57)
    a = [geprep._poly(res["nf"], v) for v in xs]
    b = [geprep._poly(nf, v) for v in xs]
    np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-12)
    assert res["nf"]["alphaup"] == pytest.approx(nf["alphaup"], rel=1e-12)


def test_flatness_weights_and_acceleration():
    # nBIN = 4, nBOR = 1: bins 0 and 5 are border bins
    c1 = np.array([0.0, 8.0, 4.0, 1.0, 1.0, 0.0])
    c2 = np.array([0.0, 0.0, 8.0, 8.0, 4.0, 1.0])
    d = geprep.distribution([c1, c2], 0.0, 4.0, 4, 1, fw=[1.0, 0.5], sets=[0, 1], accele=True,
                            accrat=1.0)
    # set flatness: exp(ln(c/max)) over the 4 inner bins, in percent
    f1 = (1 + 0.5 + 0.125 + 0.125) / 4 * 100
    f2 = (0 + 1 + 1 + 0.5) / 4 * 100
    np.testing.assert_allclose(d["flt"], [f1, f2])
    np.testing.assert_allclose(d["rP"], c1 + c2)
    np.testing.assert_allclose(d["P"], c1 / f1 + 0.5 * c2 / f2)
    rp = c1 + c2
    inner = rp[1:5] / rp.max()
    assert d["flat"] == pytest.approx(inner.sum() / 4 * 100)
    # energy ranges: EE = -0.5, 0.5, ..., 4.5 (bin width 1)
    np.testing.assert_allclose(d["erange"][0], [4.0, 2.0])   # bins 1-4; ln P >= -1.5 in 1-2
    np.testing.assert_allclose(d["erange"][1], [4.0, 3.0])   # bins 2-5; ln P >= -1.5 in 2-4
    assert d["fwflg"]
    # TTPdist: sets whose ln P <= 0, >= -1.5, >= -0.5 in each bin
    np.testing.assert_array_equal(d["ttpdist"][2], [2, 2, 1])
    np.testing.assert_array_equal(d["ttpdist"][5], [1, 0, 0])


def test_flat_histogram_reproduces_the_weight_and_writes_files(eng, tmp_path):
    emin, emax, nbin, nbor = -2000.0, -1000.0, 100, 5
    old = systems.mcmd_weight(emin, emax)
    h = np.full(nbin + 2 * nbor, 500.0)
    prefix = os.path.join(tmp_path, "run")
    res = geprep.iterate([h], old, emin, emax, nbin, nbor, emin, emax, 300.0, ndeg=8, prefix=prefix,
                         smp_temp=300.0, neglect_low=True, neglect_high=True)
    assert res["dist"]["flat"] == pytest.approx(100.0)
    xs = np.linspace(0.0, 1.0, 41)
    np.testing.assert_allclose([geprep._poly(res["nf"], v) for v in xs],
                               [geprep._poly(old, v) for v in xs], rtol=1e-6)
    et = np.loadtxt(prefix + ".et")
    assert et.shape == (nbin + 2, 2)
    assert et[0, 1] == pytest.approx(280.0, rel=2e-3)
    assert et[-1, 1] == pytest.approx(700.0, rel=2e-3)
    for ext in (".dist", ".bar", ".dlnN", ".TTPdist", ".sph", "_300.cdist", "_300.prob"):
        assert os.path.getsize(prefix + ext) > 0, ext
    prob = open(prefix + "_300.prob").read().split("\n")
    assert prob[0] == "MULT" and int(prob[1]) == nbin
    cd = np.loadtxt(prefix + "_300.cdist")
    assert cd.shape == (nbin, 2) and cd[:, 1].max() == 0.0


def test_alsd_mean_force_and_fit(eng):
    """distrib_ALSD on histograms with a known mean force: dE/dlambda summed to
    counts * (a + b lambda) in every bin gives F = -(a + b lambda) / (R T) exactly, and the
    lstsquare_final fit on [lmin, lmax] in lambda recovers that line; run weights and the
    flatness-accelerated sums leave F unchanged when every run has the same mean force."""
    lmin, lmax, nbin, nbor, T = 0.6, 1.0, 20, 2, 300.0
    EE, _ = geprep.bin_centres(lmin, lmax, nbin, nbor)
    rng = np.random.default_rng(3)
    a, b = -120.0, 40.0
    runs_c = rng.integers(50, 400, (3, len(EE))).astype(float)
    runs_f = runs_c * (a + b * EE)
    d = geprep.alsd_distribution(runs_c, runs_f, lmin, lmax, nbin, nbor, T, fw=[1.0, 0.5, 2.0],
                                 accele=True, accrat=0.5)
    rt = 1.0 / (geprep.R_GAS * T)
    np.testing.assert_allclose(d["F"], -(a + b * EE) * rt, rtol=1e-12)
    np.testing.assert_allclose(d["rF"], -(a + b * EE) * rt, rtol=1e-12)
    inner = runs_c.sum(0)[nbor:nbor + nbin]
    assert d["maxmin"] == pytest.approx(inner.max() / inner.min())
    nf, resid, _ = geprep.alsd_fit(d, lmin, lmax, T, 2, 3, 15.0, 25.0)
    lam = np.linspace(lmin, lmax, 17)
    np.testing.assert_allclose([geprep._poly(nf, v) for v in lam], -(a + b * lam) * rt, rtol=1e-9, atol=1e-9)
    assert nf["lower"] == -15.0 and nf["upper"] == 25.0 and nf["celw"] == lmin


def test_alsd_network_data():
    """(E, lambda) training data: the lambda target is the cell's mean force, the E target the
    canonical d ln(visits)/dE + 1/(R T) of the lambda column."""
    T = 300.0
    rt = 1.0 / (geprep.R_GAS * T)
    ne, nbin, nbor = 6, 4, 0
    c2 = np.zeros((ne, nbin))
    c2[1:5, 1] = [10.0, 20.0, 40.0, 80.0]    # ln visits rises by ln 2 per E bin
    f2 = c2 * -50.0
    X, Y, W = geprep.alsd_net_data(c2, f2, -100.0, -40.0, 0.6, 1.0, nbin, nbor, T)
    assert len(X) == 4
    np.testing.assert_allclose(Y[:, 0], 50.0 * rt)
    np.testing.assert_allclose(Y[:, 1], np.log(2.0) / 10.0 + rt)
    np.testing.assert_allclose(W, np.sqrt([10.0, 20.0, 40.0, 80.0]))
    np.testing.assert_allclose(X[:, 1], 0.75)
