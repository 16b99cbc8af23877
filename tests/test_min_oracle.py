"""The oracle's steepest descent (steep.f90 steep / linsrd, calrsf.f90, mksrdg) against the
same iteration written out in numpy from single-point energies, and its stop conditions
(no GPU).
"""
import numpy as np
import pytest

import oracle
from j_presto_b200 import abi, systems

CANO, NOSHAKE = abi.JP_METHOD_CANO, abi.JP_SHAKE_NONE


@pytest.fixture(scope="module")
def poly():
    return dict(systems.solvated_polymer(8, 300, seed=3))


def test_iterations_written_out(poly):
    """Three iterations without list rebuilds: x <- x - stp g/|g|, stp0 = ISTEPL sqrt(N),
    stp times 1.2 after a lower energy, 0.6 otherwise."""
    o = oracle.Oracle(poly, method=CANO, shake_method=NOSHAKE)
    ref = oracle.Oracle(poly, method=CANO, shake_method=NOSHAKE)
    x = np.asarray(poly["cord"], float).copy()
    n = len(x)
    e, g = ref.energy_grad(x)
    stp = 0.01 * np.sqrt(n)
    for _ in range(3):
        eold = e[0]
        x = x - stp * g / np.sqrt((g * g).sum())
        e, g = ref.energy_grad(x)
        stp *= 1.2 if e[0] < eold else 0.6
    ier, it, ene, rmsf, st = o.minimize(max_loop=3, update=0, convgr=0.0)
    assert (ier, it, st) == (0, 3, 0)
    xm = o.get_state()[0]
    np.testing.assert_allclose(xm, x, rtol=0, atol=1e-12)
    np.testing.assert_allclose(ene, e, rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(rmsf, np.sqrt((g * g).sum() / n), rtol=1e-12)


def test_converges_and_reports_the_final_gradient(poly):
    o = oracle.Oracle(poly, method=CANO, shake_method=NOSHAKE)
    e0 = o.energy_grad()[0][0]
    ier, it, ene, rmsf, st = o.minimize(max_loop=2000, convgr=3.0)
    assert (ier, st) == (0, 1) and it < 2000
    e, g = o.energy_grad()
    assert rmsf <= 3.0
    np.testing.assert_allclose(rmsf, np.sqrt((g * g).sum() / len(g)), rtol=1e-10)
    np.testing.assert_allclose(ene[0], e[0], rtol=1e-10)
    assert e[0] < e0 - 500.0


def test_shake_keeps_the_constraints(poly):
    o = oracle.Oracle(poly, method=CANO)
    ier, it, _, _, _ = o.minimize(max_loop=40)
    assert ier == 0 and it == 40
    x = o.get_state()[0]
    for g, na, d in zip(poly["shake_atoms"], poly["shake_n"], poly["shake_dist"]):
        pairs = [(0, 1), (1, 2), (2, 0), (3, 0), (2, 3), (1, 3)]
        for (p, q), d0 in zip(pairs, d):
            if p < na and q < na and d0 > 0:
                r2 = ((x[g[p]] - x[g[q]]) ** 2).sum()
                assert abs(r2 - d0 * d0) <= 2e-6 * d0 * d0


def test_vanishing_step_length_stops(poly):
    """A first step far too long raises the energy; with DOWN = 1e-12 the step length falls
    below 1e-10 A per degree of freedom at once (steep.f90:235-243, ier = -2)."""
    o = oracle.Oracle(poly, method=CANO, shake_method=NOSHAKE)
    ier, it, _, _, st = o.minimize(max_loop=10, step0=3.0, down=1e-12, convgr=0.0)
    assert (ier, it, st) == (-2, 1, 2)


def test_conj_first_trial_and_progress(poly):
    """METHOD= CONJ (conj.f90): the first trial point is the steepest-descent step of length
    ISTEPL sqrt(N); over the same number of evaluations it ends lower than STEE; SHAKE is
    refused (ier -1)."""
    ref = oracle.Oracle(poly, method=CANO, shake_method=NOSHAKE)
    x0 = np.asarray(poly["cord"], float)
    _, g0 = ref.energy_grad(x0)
    o = oracle.Oracle(poly, method=CANO, shake_method=NOSHAKE)
    ier, it, _, _, st = o.minimize_conj(max_loop=1, update=0, convgr=0.0)
    assert (ier, it, st) == (0, 1, 0)
    want = x0 - 0.01 * np.sqrt(len(x0)) * g0 / np.sqrt((g0 * g0).sum())
    np.testing.assert_allclose(o.get_state()[0], want, rtol=0, atol=1e-12)
    oc = oracle.Oracle(poly, method=CANO, shake_method=NOSHAKE)
    os_ = oracle.Oracle(poly, method=CANO, shake_method=NOSHAKE)
    ec = oc.minimize_conj(max_loop=150, convgr=0.0)[2][0]
    es = os_.minimize(max_loop=150, convgr=0.0)[2][0]
    assert ec < es
    e1, g1 = oc.energy_grad()
    np.testing.assert_allclose(e1[0], ec, rtol=1e-10)
    assert oracle.Oracle(poly, method=CANO).minimize_conj(max_loop=5)[0] == -1


def test_conj_converges(poly):
    o = oracle.Oracle(poly, method=CANO, shake_method=NOSHAKE)
    ier, it, ene, rmsf, st = o.minimize_conj(max_loop=3000, convgr=1.0)
    assert (ier, st) == (0, 1) and rmsf <= 1.0 and it < 3000
