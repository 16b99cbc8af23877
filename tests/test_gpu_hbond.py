"""The hydrogen-bond 10-12 pairs (iyppid = 2, enear.f90:330-516) on the GPU against the
oracle: energies with the JP_E_HBOND slot and gradients for ZD and atom cut-off, periodic
and free boundary, FP64 and mixed; 15-step trajectories across list rebuilds; ALSD class
energies; two replicas in one context; and the parameter checks.

The marked type pairs (donor H -- acceptor O, water H -- water O included) give thousands
of H-bond pairs.  Tolerances as the other parity tests: FP64 gradient RMS relative 1e-12
and energies 1e-8 relative; mixed path gradient RMS relative 1e-5; 15-step FP64
trajectories within 1e-8 A.
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
HB = abi.JP_E_HBOND
PAIRS = systems.HBOND_PAIRS + ((systems.T_HW, systems.T_OW),)


@pytest.fixture(scope="module")
def eng_mod(engine_lib):
    from j_presto_b200 import engine
    return engine


@pytest.fixture(scope="module")
def poly():
    return systems.with_hbond(dict(systems.solvated_polymer(20, 1500, seed=7)), pairs=PAIRS)


@pytest.fixture(scope="module")
def drop():
    return systems.with_hbond(dict(systems.droplet(12, 1200, seed=9), box=np.full(3, 28.0)), pairs=PAIRS)


def _check(eng_mod, top, kw, precs=(FP64, MIXED)):
    eo, go = oracle.Oracle(top, **kw).energy_grad()
    assert eo[HB] < -50.0
    for prec, gtol, etol in ((FP64, 1e-12, 1e-8), (MIXED, 1e-5, 1e-5)):
        if prec not in precs:
            continue
        with eng_mod.Engine(top, precision=prec, **kw) as e:
            ene, g = e.energy_grad()
        assert rms_rel(g, go) < gtol
        np.testing.assert_allclose(ene, eo, rtol=etol, atol=1e-7 if prec == FP64 else 1e-2)


@pytest.mark.parametrize("sysname,cal,bnd", [("poly", ZD, PBC), ("poly", ATOM, PBC),
                                             ("drop", ZD, NONE), ("drop", ATOM, NONE)])
def test_energy_grad_vs_oracle(eng_mod, request, sysname, cal, bnd):
    top = request.getfixturevalue(sysname)
    _check(eng_mod, top, dict(method=abi.JP_METHOD_CANO, cal15m=cal, bounda=bnd))


@pytest.mark.parametrize("method", [abi.JP_METHOD_MICR, abi.JP_METHOD_CANO])
def test_trajectory_vs_oracle(eng_mod, poly, method):
    """UPDATE= 5: the H-bond list is rebuilt twice inside the 15 steps."""
    kw = dict(method=method, update=5)
    o = oracle.Oracle(poly, **kw)
    ier, eh, _ = o.run(15)
    assert ier == 0
    xo, vo = o.get_state()
    with eng_mod.Engine(poly, precision=FP64, **kw) as e:
        ene, _ = e.step(15)
        x, v = e.get_state()
    assert np.abs(x - xo).max() < 1e-8
    assert np.abs(v - vo).max() < 1e-8
    np.testing.assert_allclose(ene[:, 0, HB], np.asarray(eh)[:, HB], rtol=1e-7, atol=1e-5)


def test_mixed_path_follows_the_oracle(eng_mod, poly):
    """10 steps through a rebuild; the fixed-point sums make the run bit-reproducible."""
    kw = dict(method=abi.JP_METHOD_CANO, update=5)
    o = oracle.Oracle(poly, **kw)
    ier, eh, _ = o.run(10)
    assert ier == 0
    out = []
    for _ in range(2):
        with eng_mod.Engine(poly, precision=MIXED, **kw) as e:
            ene, _ = e.step(10)
            out.append(e.get_state()[0])
        np.testing.assert_allclose(ene[:, 0, HB], np.asarray(eh)[:, HB], rtol=1e-3, atol=0.05)
    assert np.array_equal(out[0], out[1])


def test_alsd_class_energies_vs_oracle(eng_mod, poly):
    top = dict(poly)
    cl = np.zeros(top["natom"], np.int32)
    cl[:60] = 1
    for g, na in zip(top["shake_atoms"], top["shake_n"]):
        if cl[g[:na]].any():
            cl[g[:na]] = 1
    top["cluster"] = cl
    kw = dict(method=abi.JP_METHOD_CANO, alsd=abi.JP_ALSD_LMD, lambda0=0.8)
    o = oracle.Oracle(top, **kw)
    eo, go = o.energy_grad()
    _, eco = o.get_lambda()
    for prec, gtol, etol in ((FP64, 1e-12, 1e-8), (MIXED, 1e-5, 1e-5)):
        with eng_mod.Engine(top, precision=prec, **kw) as e:
            ene, g = e.energy_grad()
            _, ec = e.get_lambda()
        assert rms_rel(g, go) < gtol
        np.testing.assert_allclose(ene, eo, rtol=etol, atol=1e-7 if prec == FP64 else 1e-2)
        np.testing.assert_allclose(ec, eco, rtol=etol, atol=1e-7 if prec == FP64 else 1e-2)
    # 15 steps of atoms and lambda
    o = oracle.Oracle(top, **kw)
    assert o.run(15)[0] == 0
    xo, _ = o.get_state()
    (lo, lvo), _ = o.get_lambda()
    with eng_mod.Engine(top, precision=FP64, **kw) as e:
        e.step(15)
        x, _ = e.get_state()
        (lam, lv), _ = e.get_lambda()
    assert np.abs(x - xo).max() < 1e-8
    assert abs(lam - lo) < 1e-9 and abs(lv - lvo) < 1e-9


def test_two_replicas_in_one_context(eng_mod, poly):
    other = systems.with_hbond(dict(systems.solvated_polymer(20, 1500, seed=11)), pairs=PAIRS)
    kw = dict(method=abi.JP_METHOD_CANO)
    want = [oracle.Oracle(t, **kw).energy_grad() for t in (poly, other)]
    with eng_mod.Engine([poly, other], precision=MIXED, **kw) as e:
        for r, (eo, go) in enumerate(want):
            ene, g = e.energy_grad(rep=r)
            assert rms_rel(g, go) < 1e-5
            np.testing.assert_allclose(ene[HB], eo[HB], rtol=1e-5, atol=1e-2)


def test_invalid_tables_are_rejected(eng_mod, poly, drop):
    asym = dict(poly, hbond=np.triu(poly["hbond"]))
    bad = (
        (asym, {}),
        (dict(poly, c10=None), {}),
        (dict(drop, box=np.full(3, 80.0)), dict(cal15m=abi.JP_CAL15M_CMM, bounda=NONE)),
    )
    for top, kw in bad:
        with pytest.raises(eng_mod.JpError) as ex:
            eng_mod.Engine(top, precision=MIXED, **kw)
        assert ex.value.code == abi.JP_E_INVALID
    plain = {k: v for k, v in poly.items() if k not in ("hbond", "c10", "c12h")}
    with pytest.raises(eng_mod.JpError) as ex:   # the tables must agree between replicas
        eng_mod.Engine([poly, plain], precision=MIXED)
    assert ex.value.code == abi.JP_E_INVALID
