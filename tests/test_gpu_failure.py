"""Failure detection through the C ABI, made on the host so that no GPU faults.

* a grid-barrier wait of the integration kernel bounded at one SM cycle: the step returns
  JP_E_TIMEOUT, and after the state is restored the context steps like the oracle;
* a NaN coordinate: the step returns JP_E_NONFINITE;
* two oxygens 0.1 A apart: the force and energy terms leave the 64-bit fixed-point range
  and the evaluation returns JP_E_FIXED_OVERFLOW instead of a wrapped sum (md_run's
  overflow `ier` codes, cutoff.f90:30-46 and celpar.f90 ier=28, are the model: stop with a
  code rather than continue with damaged lists or sums).
Tolerance of the recovered trajectory: the FP64 path's 1e-8 A.
"""
import numpy as np
import pytest

import oracle
from j_presto_b200 import abi, systems

pytestmark = pytest.mark.gpu

FP64, MIXED = abi.JP_PREC_FP64, abi.JP_PREC_MIXED


@pytest.fixture(scope="module")
def eng_mod(engine_lib):
    from j_presto_b200 import engine
    return engine


@pytest.fixture(scope="module")
def water():
    return systems.config_c1_prime()


def test_barrier_timeout_is_reported_and_the_context_recovers(eng_mod, water):
    o = oracle.Oracle(water, method=abi.JP_METHOD_CANO)
    ier, _, _ = o.run(5)
    assert ier == 0
    xo, vo = o.get_state()
    with eng_mod.Engine(water, precision=FP64, method=abi.JP_METHOD_CANO) as e:
        x0, v0 = e.get_state()
        e.set_wait_limit(1)    # the first block at a barrier gives up at once
        with pytest.raises(eng_mod.JpError) as ex:
            e.step(1)
        assert ex.value.code == abi.JP_E_TIMEOUT
        e.set_wait_limit(0)
        e.set_state(cord=x0, vel=v0)
        e.step(5)
        x, v = e.get_state()
    assert np.abs(x - xo).max() < 1e-8
    assert np.abs(v - vo).max() < 1e-8


@pytest.mark.parametrize("prec", [FP64, MIXED])
def test_nan_coordinate_is_reported(eng_mod, water, prec):
    with eng_mod.Engine(water, precision=prec, method=abi.JP_METHOD_MICR) as e:
        x, v = e.get_state()
        bad = x.copy()
        bad[4, 1] = np.nan
        e.set_state(cord=bad)
        with pytest.raises(eng_mod.JpError) as ex:
            e.step(1)
        assert ex.value.code == abi.JP_E_NONFINITE
        # the context is still usable: the original state gives the original energies
        e.set_state(cord=x, vel=v)
        e.rebuild()
        ene, g = e.energy_grad()
        assert np.isfinite(ene).all() and np.isfinite(g).all()


@pytest.mark.parametrize("prec", [FP64, MIXED])
def test_fixed_point_overflow_is_reported(eng_mod, water, prec):
    x = water["cord"].copy()
    ow = np.flatnonzero(water["atype"] == systems.T_OW)
    a, b = int(ow[0]), int(ow[1])
    shift = x[a] + np.array([0.1, 0.0, 0.0]) - x[b]
    x[b:b + 3] += shift               # move water b rigidly next to water a's oxygen
    with eng_mod.Engine(water, precision=prec, method=abi.JP_METHOD_MICR) as e:
        e0, g0 = e.energy_grad()
        e.set_state(cord=x)
        e.rebuild()
        with pytest.raises(eng_mod.JpError) as ex:
            e.energy_grad()
        assert ex.value.code == abi.JP_E_FIXED_OVERFLOW
        e.set_state(cord=water["cord"])
        e.rebuild()
        e1, g1 = e.energy_grad()
    np.testing.assert_allclose(e1, e0, rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(g1, g0, rtol=1e-12, atol=1e-9)
