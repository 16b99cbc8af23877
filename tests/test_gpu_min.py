"""Steepest-descent minimisation (jp_minimize: steep.f90) on the GPU against the oracle:
FP64 iterations with and without SHAKE across list rebuilds, restraints in the energy,
convergence, replicas minimised together equal to each alone, MD continuing from the
minimised state, the stop on a vanishing step and the parameter checks.

Tolerances: FP64 positions within 1e-8 A and energies 1e-8 relative of the oracle after the
same number of iterations (with SHAKE, its convergence tolerance: 1e-6 A, energies 1e-6
relative); the step-length decisions compare energies, which agree to far better than the
differences between successive iterations.
"""
import numpy as np
import pytest

import oracle
from j_presto_b200 import abi, systems

pytestmark = pytest.mark.gpu

FP64, MIXED = abi.JP_PREC_FP64, abi.JP_PREC_MIXED
CANO, NOSHAKE = abi.JP_METHOD_CANO, abi.JP_SHAKE_NONE


@pytest.fixture(scope="module")
def eng_mod(engine_lib):
    from j_presto_b200 import engine
    return engine


@pytest.fixture(scope="module")
def poly():
    return dict(systems.solvated_polymer(20, 1500, seed=7))


def _pair(eng_mod, top, nloop, prm=None, **kw):
    o = oracle.Oracle(top, method=CANO, **kw)
    ier, it, eo, ro, so = o.minimize(max_loop=nloop, update=5, convgr=0.0, **(prm or {}))
    assert ier == 0 and it == nloop
    with eng_mod.Engine(top, precision=FP64, method=CANO, **kw) as e:
        its, ene, rm, st = e.minimize(max_loop=nloop, update=5, convgr=0.0, **(prm or {}))
        x = e.get_state()[0]
    assert its[0] == nloop and st[0] == 0
    return o.get_state()[0], eo, ro, x, ene[0], rm[0]


@pytest.mark.parametrize("shake", [abi.JP_SHAKE_NONE, abi.JP_SHAKE_HBON])
def test_fp64_iterations_vs_oracle(eng_mod, poly, shake):
    """ISTEPL 0.002: with the default 0.01 the step length grows to moves that the SHAKE of
    the reference cannot follow on this unrelaxed system (the exact two-atom solution has
    no real root), in the engine and the oracle alike."""
    xo, eo, ro, x, ene, rm = _pair(eng_mod, poly, 25, prm=dict(step0=0.002), shake_method=shake)
    # with SHAKE each iteration's constraint solution is exact only to COVSHK (1e-6 of d0^2),
    # and the iterative 3-atom solutions may stop one iteration apart: 1e-6 A
    exact = shake == abi.JP_SHAKE_NONE
    assert np.abs(x - xo).max() < (1e-8 if exact else 1e-6)
    np.testing.assert_allclose(ene, eo, rtol=1e-8 if exact else 1e-6, atol=1e-7 if exact else 1e-4)
    np.testing.assert_allclose(rm, ro, rtol=1e-8 if exact else 1e-5)


def test_restraints_enter_the_minimisation(eng_mod, poly):
    top = systems.with_restraints(poly)
    xo, eo, ro, x, ene, rm = _pair(eng_mod, top, 20, shake_method=NOSHAKE)
    assert np.abs(x - xo).max() < 1e-8
    np.testing.assert_allclose(ene, eo, rtol=1e-8, atol=1e-7)


def test_converges_then_md_continues(eng_mod, poly):
    """Minimise to convergence, then 5 MD steps: the engine leaves zero accumulators and a
    list built at the minimised positions, as the oracle's rebuild does.  Without SHAKE:
    steepest descent does not project the constraint forces out of the gradient, so with
    SHAKE the RMS gradient stalls well above this threshold."""
    o = oracle.Oracle(poly, method=CANO, shake_method=NOSHAKE)
    ier, it, eo, ro, so = o.minimize(max_loop=400, convgr=8.0)
    assert ier == 0 and so == 1
    assert o.run(5)[0] == 0
    xo = o.get_state()[0]
    with eng_mod.Engine(poly, precision=FP64, method=CANO, shake_method=NOSHAKE) as e:
        its, ene, rm, st = e.minimize(max_loop=400, convgr=8.0)
        assert its[0] == it and st[0] == 1 and rm[0] <= 8.0
        e.step(5)
        x = e.get_state()[0]
    assert np.abs(x - xo).max() < 1e-7


def test_replicas_minimise_independently(eng_mod, poly):
    other = dict(systems.solvated_polymer(20, 1500, seed=11))
    kw = dict(max_loop=15, update=5, convgr=0.0, step0=0.002)
    singles = []
    for t in (poly, other):
        with eng_mod.Engine(t, precision=FP64, method=CANO) as e:
            its, ene, _, _ = e.minimize(**kw)
            singles.append((e.get_state()[0], ene[0]))
    with eng_mod.Engine([poly, other], precision=FP64, method=CANO) as e:
        its, ene, _, st = e.minimize(**kw)
        for r in range(2):
            assert its[r] == 15 and st[r] == 0
            assert np.abs(e.get_state(rep=r)[0] - singles[r][0]).max() < 1e-9
            np.testing.assert_allclose(ene[r], singles[r][1], rtol=1e-10, atol=1e-8)


def test_mixed_path_lowers_the_energy(eng_mod, poly):
    o = oracle.Oracle(poly, method=CANO)
    e0 = o.energy_grad()[0][0]
    ier, it, eo, _, _ = o.minimize(max_loop=60, step0=0.002)
    assert ier == 0
    with eng_mod.Engine(poly, precision=MIXED, method=CANO) as e:
        its, ene, rm, st = e.minimize(max_loop=60, step0=0.002)
    assert its[0] == 60 and st[0] == 0
    assert ene[0][0] < e0 - 0.5 * (e0 - eo[0])


def test_vanishing_step_and_bad_parameters(eng_mod, poly):
    with eng_mod.Engine(poly, precision=FP64, method=CANO, shake_method=NOSHAKE) as e:
        with pytest.raises(eng_mod.JpError) as ex:
            e.minimize(max_loop=10, step0=0.1, down=1e-12, convgr=0.0)   # E rises 2.8e3 -> 2.2e4
        assert ex.value.code == abi.JP_E_MIN_STEP
        for bad in (dict(max_loop=0), dict(step0=0.0), dict(convgr=-1.0), dict(method=3),
                    dict(method=abi.JP_MIN_CONJ, line_max=0)):
            with pytest.raises(eng_mod.JpError) as ex:
                e.minimize(**bad)
            assert ex.value.code == abi.JP_E_INVALID


def test_conj_vs_oracle(eng_mod, poly):
    """METHOD= CONJ: 40 evaluations through list rebuilds, the direction and line-search
    decisions the same as the oracle's."""
    kw = dict(method=CANO, shake_method=NOSHAKE)
    o = oracle.Oracle(poly, **kw)
    ier, it, eo, ro, so = o.minimize_conj(max_loop=40, update=5, convgr=0.0)
    assert ier == 0 and it == 40
    with eng_mod.Engine(poly, precision=FP64, **kw) as e:
        its, ene, rm, st = e.minimize(method=abi.JP_MIN_CONJ, max_loop=40, update=5, convgr=0.0)
        x = e.get_state()[0]
        assert its[0] == 40 and st[0] == 0
        # and MD runs on from the minimised state
        e.step(3)
    assert np.abs(x - o.get_state()[0]).max() < 1e-7
    np.testing.assert_allclose(ene[0], eo, rtol=1e-8, atol=1e-6)
    np.testing.assert_allclose(rm[0], ro, rtol=1e-6)


def test_conj_refuses_shake(eng_mod, poly):
    with eng_mod.Engine(poly, precision=MIXED, method=CANO) as e:
        with pytest.raises(eng_mod.JpError) as ex:
            e.minimize(method=abi.JP_MIN_CONJ, max_loop=5)
        assert ex.value.code == abi.JP_E_INVALID
