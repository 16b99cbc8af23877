"""Atom cut-off (CAL15M= ATOM) and free boundary (BOUNDA= NO) on the GPU against the oracle.

The engine runs BOUNDA= NO in a periodic container in which minimum image is the identity;
the droplet's own box (28 A) is deliberately too small for it, so a wrong (periodic) answer
cannot pass.  Tolerances as the other parity tests: FP64 gradient RMS relative 1e-12 and
energies 1e-8 relative; mixed path gradient RMS relative 1e-5; 15-step FP64 trajectories
within 1e-8 A.
"""
import numpy as np
import pytest

import oracle
from j_presto_b200 import abi, systems
from tests._util import rms_rel

pytestmark = pytest.mark.gpu

FP64, MIXED = abi.JP_PREC_FP64, abi.JP_PREC_MIXED
ZD, ATOM = abi.JP_CAL15M_ZD, abi.JP_CAL15M_ATOM
PBC, NONE = abi.JP_BOUND_PBC, abi.JP_BOUND_NONE


@pytest.fixture(scope="module")
def eng_mod(engine_lib):
    from j_presto_b200 import engine
    return engine


@pytest.fixture(scope="module")
def drop():
    return dict(systems.droplet(12, 1200, seed=9), box=np.full(3, 28.0))


@pytest.fixture(scope="module")
def poly():
    return dict(systems.solvated_polymer(20, 1500, seed=7))


@pytest.mark.parametrize("sysname,cal,bnd", [("drop", ZD, NONE), ("drop", ATOM, NONE),
                                             ("poly", ATOM, PBC)])
def test_energy_grad_vs_oracle(eng_mod, request, sysname, cal, bnd):
    top = request.getfixturevalue(sysname)
    kw = dict(method=abi.JP_METHOD_CANO, cal15m=cal, bounda=bnd)
    eo, go = oracle.Oracle(top, **kw).energy_grad()
    for prec, gtol, etol in ((FP64, 1e-12, 1e-8), (MIXED, 1e-5, 1e-5)):
        with eng_mod.Engine(top, precision=prec, **kw) as e:
            ene, g = e.energy_grad()
        assert rms_rel(g, go) < gtol
        np.testing.assert_allclose(ene, eo, rtol=etol, atol=1e-7 if prec == FP64 else 1e-2)


@pytest.mark.parametrize("cal", [ZD, ATOM])
def test_trajectory_vs_oracle(eng_mod, drop, cal):
    kw = dict(method=abi.JP_METHOD_CANO, cal15m=cal, bounda=NONE, update=5)
    o = oracle.Oracle(drop, **kw)
    ier, _, _ = o.run(15)
    assert ier == 0
    xo, vo = o.get_state()
    with eng_mod.Engine(drop, precision=FP64, **kw) as e:
        e.step(15)
        x, v = e.get_state()
    assert np.abs(x - xo).max() < 1e-8
    assert np.abs(v - vo).max() < 1e-8


def test_leaving_the_window_is_reported(eng_mod, drop):
    """An atom moved far outside the droplet is caught at the next list rebuild."""
    with eng_mod.Engine(drop, precision=MIXED, method=abi.JP_METHOD_CANO, bounda=NONE) as e:
        x, v = e.get_state()
        x = x.copy()
        x[0] += 500.0
        e.set_state(0, x, v)
        with pytest.raises(eng_mod.JpError) as ex:
            e.rebuild()
        assert ex.value.code == abi.JP_E_FREE_WINDOW


def test_cmm_needs_the_free_boundary(eng_mod, drop):
    with pytest.raises(eng_mod.JpError) as ex:
        eng_mod.Engine(dict(drop, box=np.full(3, 80.0)), precision=MIXED, cal15m=abi.JP_CAL15M_CMM,
                       bounda=PBC)
    assert ex.value.code == abi.JP_E_INVALID
