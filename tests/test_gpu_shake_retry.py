"""verlethe's SHAKE failure handling (verlethe.f90:552-574, :745-752) in the engine.

md_run redoes a step whose SHAKE failed: the state goes back to the start of the step, the
time step is halved (jshk and ishk doubled) and the step is completed in sub-steps; two
completed halves merge back into one.  Below 1 % of dt it stops with ier = -9999.  The
oracle restates the same loop, so engine and oracle take the same path:

* LIMSHK = 3 makes some groups of the small solvated polymer miss the tolerance at the full
  time step but not at half of it: the FP64 trajectory equals the oracle's to 1e-8 A and
  differs from the LIMSHK = 1000 trajectory (so the redo path ran);
* two replicas in one context each equal their own oracle run, and every replica's energy
  histogram counts one energy per step;
* a water whose O-H bond starts 0.3 A long cannot be constrained in one SHAKE iteration at
  any time step: the step ends with JP_E_SHAKE_ABORT, as the oracle's -9999.
"""
import numpy as np
import pytest

import oracle
from j_presto_b200 import abi, systems

pytestmark = pytest.mark.gpu

FP64, MIXED = abi.JP_PREC_FP64, abi.JP_PREC_MIXED
CANO = abi.JP_METHOD_CANO
NSTEP = 6


@pytest.fixture(scope="module")
def eng_mod(engine_lib):
    from j_presto_b200 import engine
    return engine


@pytest.fixture(scope="module")
def tops():
    return [systems.solvated_polymer(6, 300, seed=11), systems.solvated_polymer(6, 300, seed=12)]


def _oracle_run(top, maxit, nsteps=NSTEP):
    o = oracle.Oracle(top, method=CANO, shake_maxit=maxit)
    ier, E, _ = o.run(nsteps)
    x, v = o.get_state()
    return ier, E, x, v


def test_retry_matches_oracle(eng_mod, tops):
    top = tops[0]
    ier, Eo, xo, vo = _oracle_run(top, 3)
    assert ier == 0
    _, _, xf, _ = _oracle_run(top, 1000)
    assert np.abs(xo - xf).max() > 1e-4          # the halved steps changed the trajectory
    with eng_mod.Engine(top, precision=FP64, method=CANO, shake_maxit=3) as e:
        E, _ = e.step(NSTEP)
        x, v = e.get_state()
    assert np.abs(x - xo).max() < 1e-8
    assert np.abs(v - vo).max() < 1e-8
    np.testing.assert_allclose(E[:, 0, 0], Eo[:, 0], rtol=1e-8, atol=1e-6)


def test_retry_in_a_replica_batch(eng_mod, tops):
    ref = [_oracle_run(t, 3) for t in tops]
    assert all(r[0] == 0 for r in ref)
    with eng_mod.Engine(tops, precision=FP64, method=CANO, shake_maxit=3) as e:
        e.ge_hist_setup(-1.0e6, 1.0e6, 100, 0)
        E, _ = e.step(NSTEP)
        for r, (_, Eo, xo, _) in enumerate(ref):
            x, _ = e.get_state(rep=r)
            assert np.abs(x - xo).max() < 1e-8
            np.testing.assert_allclose(E[:, r, 0], Eo[:, 0], rtol=1e-8, atol=1e-6)
            assert e.ge_hist_get(rep=r).sum() == NSTEP


def test_retry_on_the_mixed_path(eng_mod, tops):
    top = tops[0]
    _, _, xo, _ = _oracle_run(top, 3)
    with eng_mod.Engine(top, precision=MIXED, method=CANO, shake_maxit=3) as e:
        e.step(NSTEP)
        x, _ = e.get_state()
    assert np.abs(x - xo).max() < 1e-3


def test_abort_below_one_percent_of_dt(eng_mod, tops):
    top = dict(tops[0])
    x = top["cord"].copy()
    a = int(np.flatnonzero(top["atype"] == systems.T_OW)[3])
    d = x[a + 1] - x[a]
    x[a + 1] += 0.3 * d / np.linalg.norm(d)
    top["cord"] = x
    ier, _, _, _ = _oracle_run(top, 1, nsteps=1)
    assert ier == abi.JP_E_SHAKE_ABORT
    with eng_mod.Engine(top, precision=FP64, method=CANO, shake_maxit=1) as e:
        with pytest.raises(eng_mod.JpError) as ex:
            e.step(1)
        assert ex.value.code == abi.JP_E_SHAKE_ABORT
