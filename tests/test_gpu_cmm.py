"""Cell multipole method (CAL15M= CMM, BOUNDA= NO) on the GPU against the oracle: the near
field (neighbouring level-1 cells without cut-off, LJ-only pairs out to CUTLEN) in the tile
kernels, multipoles at each rebuild, the far field every CMMUPD steps and reused between.

Tolerances as the other parity tests: FP64 gradient RMS relative 1e-12 (1e-11 with the far
field, whose cell sums are FP64 atomics), energies 1e-8 relative; mixed path gradient RMS
relative 1e-5; 12-step FP64 trajectories (far field at steps 1, 6, 11, a rebuild after
step 10) within 1e-8 A.
"""
import numpy as np
import pytest

import oracle
from j_presto_b200 import abi, systems
from tests._util import rms_rel

pytestmark = pytest.mark.gpu

FP64, MIXED = abi.JP_PREC_FP64, abi.JP_PREC_MIXED
CMM = dict(method=abi.JP_METHOD_CANO, cal15m=abi.JP_CAL15M_CMM, bounda=abi.JP_BOUND_NONE)


@pytest.fixture(scope="module")
def eng_mod(engine_lib):
    from j_presto_b200 import engine
    return engine


@pytest.fixture(scope="module")
def drop():
    return dict(systems.droplet(12, 1200, seed=9), box=np.full(3, 28.0))


@pytest.mark.parametrize("cell", [6.0, 4.0])
def test_energy_grad_vs_oracle(eng_mod, drop, cell):
    kw = dict(CMM, cmm_cell=cell)
    o = oracle.Oracle(drop, **kw)
    eo, go = o.energy_grad()
    ef, _ = o.cmm_far()
    assert abs(ef) > 1.0   # the far field is there
    for prec, gtol, etol in ((FP64, 1e-11, 1e-8), (MIXED, 1e-5, 1e-5)):
        with eng_mod.Engine(drop, precision=prec, **kw) as e:
            ene, g = e.energy_grad()
        assert rms_rel(g, go) < gtol
        np.testing.assert_allclose(ene, eo, rtol=etol, atol=1e-6 if prec == FP64 else 1e-2)


def test_trajectory_vs_oracle(eng_mod, drop):
    kw = dict(CMM, cmm_update=5, update=10)
    o = oracle.Oracle(drop, **kw)
    ier, Eo, _ = o.run(12)
    assert ier == 0
    xo, vo = o.get_state()
    with eng_mod.Engine(drop, precision=FP64, **kw) as e:
        E, _ = e.step(12)
        x, v = e.get_state()
    assert np.abs(x - xo).max() < 1e-8
    assert np.abs(v - vo).max() < 1e-8
    np.testing.assert_allclose(np.asarray(E)[:, 0, :], Eo, rtol=1e-8, atol=1e-6)


def test_mixed_trajectory_tracks_fp64(eng_mod, drop):
    kw = dict(CMM, cmm_update=5, update=10)
    with eng_mod.Engine(drop, precision=FP64, **kw) as e:
        e.step(20)
        x64, _ = e.get_state()
    with eng_mod.Engine(drop, precision=MIXED, **kw) as e:
        e.step(20)
        x32, _ = e.get_state()
    assert np.abs(x32 - x64).max() < 1e-3


@pytest.mark.parametrize("kw", [dict(alsd=abi.JP_ALSD_LMD), dict(update=7, cmm_update=5),
                                dict(cmm_cell=0.0)])
def test_invalid_cmm_parameters(eng_mod, drop, kw):
    with pytest.raises(eng_mod.JpError) as ex:
        eng_mod.Engine(drop, precision=MIXED, **dict(CMM, **kw))
    assert ex.value.code == abi.JP_E_INVALID


def _celres(top):
    """Every water (O, H, H) and every 10-atom stretch of the chain as a CELRES residue."""
    t = np.asarray(top["atype"])
    ow = np.flatnonzero(t == systems.T_OW)
    res = [(o, o + 2) for o in ow]
    nsol = int(ow.min()) if len(ow) else int(top["natom"])
    res += [(a, min(a + 9, nsol - 1)) for a in range(0, nsol, 10)]
    return dict(top, celres=np.array(res, np.int32))


def test_celres_vs_oracle(eng_mod, drop):
    """CELRES: atoms take the cell of their residue's centre (celpar.f90:131-153), which
    moves near/far boundaries; energies, gradients and a 12-step trajectory as the oracle."""
    top = _celres(drop)
    kw = dict(CMM, cmm_update=5, update=10)
    o = oracle.Oracle(top, **kw)
    eo, go = o.energy_grad()
    e_plain = oracle.Oracle(drop, **kw).energy_grad()[0]
    assert abs(eo[abi.JP_E_ELE15] - e_plain[abi.JP_E_ELE15]) > 1e-3   # the cells changed
    for prec, gtol, etol in ((FP64, 1e-11, 1e-8), (MIXED, 1e-5, 1e-5)):
        with eng_mod.Engine(top, precision=prec, **kw) as e:
            ene, g = e.energy_grad()
        assert rms_rel(g, go) < gtol
        np.testing.assert_allclose(ene, eo, rtol=etol, atol=1e-6 if prec == FP64 else 1e-2)
    ier, Eo, _ = o.run(12)
    assert ier == 0
    xo, _ = o.get_state()
    with eng_mod.Engine(top, precision=FP64, **kw) as e:
        e.step(12)
        x, _ = e.get_state()
    assert np.abs(x - xo).max() < 1e-8


def test_celres_needs_cmm(eng_mod, drop):
    with pytest.raises(eng_mod.JpError) as ex:
        eng_mod.Engine(_celres(drop), precision=MIXED, method=abi.JP_METHOD_CANO)
    assert ex.value.code == abi.JP_E_INVALID
