"""Restraints (POSITI, DISTAN, DIHEDR: dneres.f90) and the CAP (SETBOU sphere, box and
ellipsoid: dnecap.f90) on the GPU against the oracle: energies in their four slots and gradients, FP64 and mixed,
periodic (restraints) and free boundary (restraints + CAP); 15-step FP64 trajectories;
ALSD class energies (the restraints belong to class BB, unscaled); the parameter checks.

Tolerances as the other parity tests: FP64 gradient RMS relative 1e-12 and energies 1e-8
relative; mixed path gradient RMS relative 1e-5; 15-step FP64 trajectories within 1e-8 A.
"""
import numpy as np
import pytest

import oracle
from j_presto_b200 import abi, systems
from tests._util import rms_rel

pytestmark = pytest.mark.gpu

FP64, MIXED = abi.JP_PREC_FP64, abi.JP_PREC_MIXED
PBC, NONE = abi.JP_BOUND_PBC, abi.JP_BOUND_NONE
SLOTS = [abi.JP_E_POSRES, abi.JP_E_DISTRES, abi.JP_E_DIHERES, abi.JP_E_CAP]


@pytest.fixture(scope="module")
def eng_mod(engine_lib):
    from j_presto_b200 import engine
    return engine


@pytest.fixture(scope="module")
def poly():
    return systems.with_restraints(dict(systems.solvated_polymer(20, 1500, seed=7)))


@pytest.fixture(scope="module")
def drop():
    return systems.with_restraints(dict(systems.droplet(12, 1200, seed=9), box=np.full(3, 28.0)), cap=True)


@pytest.mark.parametrize("sysname,bnd", [("poly", PBC), ("drop", NONE)])
def test_energy_grad_vs_oracle(eng_mod, request, sysname, bnd):
    top = request.getfixturevalue(sysname)
    kw = dict(method=abi.JP_METHOD_CANO, bounda=bnd)
    eo, go = oracle.Oracle(top, **kw).energy_grad()
    assert (eo[SLOTS[:3]] > 1.0).all()
    for prec, gtol, etol in ((FP64, 1e-12, 1e-8), (MIXED, 1e-5, 1e-5)):
        with eng_mod.Engine(top, precision=prec, **kw) as e:
            ene, g = e.energy_grad()
        assert rms_rel(g, go) < gtol
        np.testing.assert_allclose(ene, eo, rtol=etol, atol=1e-7 if prec == FP64 else 1e-2)
        np.testing.assert_allclose(ene[SLOTS], eo[SLOTS], rtol=1e-9, atol=1e-8)   # FP64 on both paths


@pytest.mark.parametrize("sysname,bnd,method", [("poly", PBC, abi.JP_METHOD_MICR),
                                                ("drop", NONE, abi.JP_METHOD_CANO)])
def test_trajectory_vs_oracle(eng_mod, request, sysname, bnd, method):
    top = request.getfixturevalue(sysname)
    kw = dict(method=method, bounda=bnd, update=5)
    o = oracle.Oracle(top, **kw)
    ier, eh, _ = o.run(15)
    assert ier == 0
    xo, vo = o.get_state()
    with eng_mod.Engine(top, precision=FP64, **kw) as e:
        ene, _ = e.step(15)
        x, v = e.get_state()
    assert np.abs(x - xo).max() < 1e-8
    assert np.abs(v - vo).max() < 1e-8
    np.testing.assert_allclose(ene[:, 0][:, SLOTS], np.asarray(eh)[:, SLOTS], rtol=1e-7, atol=1e-6)


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


def test_one_more_launch_per_step(eng_mod, poly):
    plain = {k: v for k, v in poly.items() if k != "restraints"}
    with eng_mod.Engine(plain, precision=MIXED) as e:
        n0 = e.launch_counts()[0]
    with eng_mod.Engine(poly, precision=MIXED) as e:
        n1 = e.launch_counts()[0]
    assert n1 == n0 + 1


def test_invalid_restraints_are_rejected(eng_mod, poly, drop):
    rd = poly["restraints"]
    ig, jg, lo, up, klo, kup = rd["dist"]
    overlap = dict(rd, dist=([[ig[0][0]]] + ig[1:], [[ig[0][0]]] + jg[1:], lo, up, klo, kup))
    swapped = dict(rd, dist=(ig, jg, up, lo, klo, kup))
    atoms, k, ref = rd["pos"]
    bad_atom = dict(rd, pos=(np.append(atoms[:-1], poly["natom"]).astype(np.int32), k, ref))
    cases = [(dict(poly, restraints=overlap), {}), (dict(poly, restraints=swapped), {}),
             (dict(poly, restraints=bad_atom), {}),
             (drop, dict(bounda=PBC))]   # the CAP belongs to BOUNDA= NO
    for top, kw in cases:
        with pytest.raises(eng_mod.JpError) as ex:
            eng_mod.Engine(top, precision=MIXED, **kw)
        assert ex.value.code == abi.JP_E_INVALID


@pytest.mark.parametrize("shape", [abi.JP_CAP_BOX, abi.JP_CAP_ELLIPSOID])
def test_cap_shapes_vs_oracle(eng_mod, drop, shape):
    """SETBOU box and ellipsoid shapes (dnecap.f90:123-250) on the droplet's groups and atoms."""
    from tests.test_restraint_oracle import _shaped
    top = _shaped(drop, shape)
    kw = dict(method=abi.JP_METHOD_CANO, bounda=NONE)
    eo, go = oracle.Oracle(top, **kw).energy_grad()
    assert eo[abi.JP_E_CAP] > 1.0
    for prec, gtol, etol in ((FP64, 1e-12, 1e-8), (MIXED, 1e-5, 1e-5)):
        with eng_mod.Engine(top, precision=prec, **kw) as e:
            ene, g = e.energy_grad()
        assert rms_rel(g, go) < gtol
        np.testing.assert_allclose(ene, eo, rtol=etol, atol=1e-7 if prec == FP64 else 1e-2)
        np.testing.assert_allclose(ene[abi.JP_E_CAP], eo[abi.JP_E_CAP], rtol=1e-9)


def test_biquadratic_cap_vs_oracle(eng_mod, drop):
    cap = dict(drop["restraints"]["cap"], function=abi.JP_CAP_BIQUADRATIC)
    top = dict(drop, restraints=dict(drop["restraints"], cap=cap))
    kw = dict(method=abi.JP_METHOD_CANO, bounda=NONE)
    eo, go = oracle.Oracle(top, **kw).energy_grad()
    assert eo[abi.JP_E_CAP] > 1.0
    for prec, gtol in ((FP64, 1e-12), (MIXED, 1e-5)):
        with eng_mod.Engine(top, precision=prec, **kw) as e:
            ene, g = e.energy_grad()
        assert rms_rel(g, go) < gtol
        np.testing.assert_allclose(ene[abi.JP_E_CAP], eo[abi.JP_E_CAP], rtol=1e-9)
    bad = dict(cap, shape=abi.JP_CAP_BOX, wall=np.zeros(6), atom_wall=np.zeros(6))
    with pytest.raises(eng_mod.JpError) as ex:   # function 2 belongs to the sphere
        eng_mod.Engine(dict(top, restraints=dict(cap=bad)), precision=MIXED, **kw)
    assert ex.value.code == abi.JP_E_INVALID
