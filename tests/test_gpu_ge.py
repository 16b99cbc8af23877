"""McMD iteration on the device: the per-step energy histogram and the in-place weight
update, through the C ABI."""
import numpy as np
import pytest

import oracle
from j_presto_b200 import abi, systems

pytestmark = pytest.mark.gpu

MIXED = abi.JP_PREC_MIXED


@pytest.fixture(scope="module")
def eng_mod(engine_lib):
    from j_presto_b200 import engine
    return engine


@pytest.fixture(scope="module")
def poly_ge():
    top = dict(systems.solvated_polymer(20, 1500, seed=7))
    e0 = oracle.Oracle(top, method=abi.JP_METHOD_MICR).energy_grad()[0][0]
    top["ge"] = systems.mcmd_weight(e0 - 400.0, e0 + 2600.0)
    return top, e0


def distrib_bins(E, emin, emax, nbin, nbor):
    """distrib_MULT.f90:91-97 binning: k = int((E - minEc)/EbinSZ) + 1 (truncation)."""
    de = (emax - emin) / nbin
    n = nbin + 2 * nbor
    h = np.zeros(n)
    for e in E:
        u = (e - (emin - de * nbor)) / de
        k = int(u)
        if u > -1.0 and 0 <= k < n:
            h[k] += 1
    return h


def test_energy_histogram_matches_step_energies(eng_mod, poly_ge):
    top, e0 = poly_ge
    with eng_mod.Engine(top, precision=MIXED, method=abi.JP_METHOD_GE) as e:
        W, _ = e.step(20)                 # past the initial relaxation
        ec = W[-1, 0, 0]
        # the synthetic system is still relaxing (~40 kcal/mol per step): a wide range
        emin, emax, nbin, nbor = ec - 8000.0, ec + 1000.0, 450, 4
        e.ge_hist_setup(emin, emax, nbin, nbor)
        E, _ = e.step(60)
        h = e.ge_hist_get(0)
        h2 = e.ge_hist_get(0, clear=True)
        h3 = e.ge_hist_get(0)
    ref = distrib_bins(E[:, 0, 0], emin, emax, nbin, nbor)
    assert ref.sum() == 60           # every step's energy falls in the range
    np.testing.assert_array_equal(h, ref)
    np.testing.assert_array_equal(h2, ref)
    assert not h3.any()


def test_weight_update_equals_weight_at_create(eng_mod, poly_ge):
    top, e0 = poly_ge
    nf_b = systems.mcmd_weight(e0 - 300.0, e0 + 1500.0, t_lo=260.0, t_hi=600.0)
    top_b = dict(top, ge=nf_b)
    def run(t, switch_to=None):
        with eng_mod.Engine(t, precision=MIXED, method=abi.JP_METHOD_GE) as e:
            e.step(1)        # the step graphs are captured here
            e.set_state(0, top["cord"], top["vel"])
            if switch_to is not None:
                e.ge_set(switch_to)
            e.rebuild()
            e.step(15)
            return e.get_state()[0]
    xb = run(top_b)                 # weight B from the start
    xs = run(top, switch_to=nf_b)   # weight A, replaced by B after capture
    xa = run(top)                   # weight A throughout
    np.testing.assert_array_equal(xs, xb)   # mixed path: bit-reproducible
    assert np.abs(xa - xb).max() > 1e-6     # the weights differ in effect


def test_mcmd_iteration_closes(eng_mod, poly_ge):
    """run -> device histogram -> jp_ge_fit -> jp_ge_set -> run, without leaving the engine."""
    top, e0 = poly_ge
    old = top["ge"]
    with eng_mod.Engine(top, precision=MIXED, method=abi.JP_METHOD_GE) as e:
        W, _ = e.step(20)
        ec = W[-1, 0, 0]
        emin, emax, nbin, nbor = ec - 12000.0, ec + 1000.0, 260, 5
        e.ge_hist_setup(emin, emax, nbin, nbor)
        S, _ = e.step(200)
        h = e.ge_hist_get(0, clear=True)
        # the new weight covers the energies this run visited
        lo, hi = S[:, 0, 0].min(), S[:, 0, 0].max()
        nf, res = eng_mod.ge_fit(h, old, emin, emax, nbin, nbor, lo, hi, 300.0, 1, 4)
        x = np.linspace(0.0, 1.0, 11)
        assert (np.polynomial.polynomial.polyval(x, nf["coef"][0]) > 0.0).all()
        e.ge_set(nf)
        E, _ = e.step(20)
    assert np.isfinite(res).all() and np.isfinite(E).all()
