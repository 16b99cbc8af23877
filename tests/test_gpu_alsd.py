"""ALSD (adaptive lambda square dynamics, CLSTMETHOD= LMD / LMD2) on the GPU against the
oracle: class energies, the lambda-weighted gradient, and trajectories of atoms and lambda
for METHOD= CANO and GE, with lambda thermostatted or free, one or per-sub-system
temperatures.

Tolerances as the other parity tests: FP64 gradient RMS relative 1e-12, energies 1e-8
relative; 15-step trajectories 1e-8 A (FP64), lambda and its velocity 1e-9; mixed path
gradient RMS relative 1e-5.
"""
import numpy as np
import pytest

import oracle
from j_presto_b200 import abi, systems
from tests._util import rms_rel

pytestmark = pytest.mark.gpu

FP64, MIXED = abi.JP_PREC_FP64, abi.JP_PREC_MIXED
ALL_TERMS = abi.JP_SCALE_BOND | abi.JP_SCALE_ANGLE | abi.JP_SCALE_TORS | abi.JP_SCALE_IMPR


@pytest.fixture(scope="module")
def eng_mod(engine_lib):
    from j_presto_b200 import engine
    return engine


@pytest.fixture(scope="module")
def clustered():
    top = dict(systems.solvated_polymer(20, 1500, seed=7))
    cl = np.zeros(top["natom"], np.int32)
    cl[:60] = 1                      # the first residues of the chain ...
    for g, na in zip(top["shake_atoms"], top["shake_n"]):   # ... with whole SHAKE groups,
        if cl[g[:na]].any():                                 # as residue lists give
            cl[g[:na]] = 1
    top["cluster"] = cl
    # McMD weight in lambda (GE): d lnP/dlambda linear on [0.6, 1.0], walls outside
    top["ge"] = dict(coef=np.array([[40.0, -30.0]]), low=np.array([0.0]), high=np.array([2.0]),
                     alphalw=0.0, alphaup=0.0, celw=0.6, ceup=1.0, tempce=300.0, lower=20.0,
                     upper=20.0)
    return top


@pytest.mark.parametrize("mode", [abi.JP_ALSD_LMD, abi.JP_ALSD_LMD2])
def test_alsd_energy_grad_vs_oracle(eng_mod, clustered, mode):
    kw = dict(method=abi.JP_METHOD_CANO, alsd=mode, lambda0=0.8, scale_terms=ALL_TERMS)
    o = oracle.Oracle(clustered, **kw)
    eo, go = o.energy_grad()
    _, eco = o.get_lambda()
    for prec, gtol in ((FP64, 1e-12), (MIXED, 1e-5)):
        with eng_mod.Engine(clustered, precision=prec, **kw) as e:
            ene, g = e.energy_grad()
            (lam, _), ec = e.get_lambda()
        assert lam == 0.8
        assert rms_rel(g, go) < gtol
        etol = 1e-8 if prec == FP64 else 1e-5
        np.testing.assert_allclose(ene, eo, rtol=etol, atol=1e-7 if prec == FP64 else 1e-2)
        np.testing.assert_allclose(ec, eco, rtol=etol, atol=1e-7 if prec == FP64 else 1e-2)
    np.testing.assert_allclose(eco.sum(), eo[0], rtol=1e-10)


@pytest.mark.parametrize("method,tempco,tc,mode,grid", [
    (abi.JP_METHOD_GE, 1, 1, abi.JP_ALSD_LMD, 0),
    (abi.JP_METHOD_GE, 2, 1, abi.JP_ALSD_LMD, 0),
    (abi.JP_METHOD_GE, 2, 0, abi.JP_ALSD_LMD2, 0),
    (abi.JP_METHOD_CANO, 1, 0, abi.JP_ALSD_LMD, 0),
    # per-phase launches (forced by a two-block cooperative grid): lambda's state of the
    # step is carried between the launches
    (abi.JP_METHOD_GE, 2, 1, abi.JP_ALSD_LMD, 2),
    (abi.JP_METHOD_GE, 1, 0, abi.JP_ALSD_LMD2, 2),
])
def test_alsd_trajectory_vs_oracle(eng_mod, clustered, method, tempco, tc, mode, grid):
    kw = dict(method=method, alsd=mode, lambda0=0.8, scale_terms=abi.JP_SCALE_TORS, tempco=tempco,
              lambda_temp_control=tc)
    o = oracle.Oracle(clustered, **kw)
    ier, Eo, To = o.run(15)
    assert ier == 0
    xo, _ = o.get_state()
    lo, _ = o.get_lambda()
    with eng_mod.Engine(clustered, precision=FP64, **kw) as e:
        if grid:
            e.set_grid_limit(grid)
        E, T = e.step(15)
        x, _ = e.get_state()
        l2, _ = e.get_lambda()
    assert np.abs(x - xo).max() < 1e-8
    np.testing.assert_allclose(l2, lo, rtol=0, atol=1e-9)
    if method == abi.JP_METHOD_GE:
        assert abs(l2[0] - 0.8) > 1e-6          # lambda moved


def test_alsd_needs_verlethe(eng_mod, clustered):
    with pytest.raises(eng_mod.JpError):
        eng_mod.Engine(clustered, precision=MIXED, method=abi.JP_METHOD_MICR, alsd=abi.JP_ALSD_LMD)


def test_shake_group_across_subsystems_is_rejected(eng_mod, clustered):
    """With per-sub-system temperatures every SHAKE group must lie in one sub-system."""
    bad = dict(clustered)
    cl = clustered["cluster"].copy()
    g = next(g for g, na in zip(clustered["shake_atoms"], clustered["shake_n"]) if na >= 2)
    cl[g[0]], cl[g[1]] = 1, 0
    bad["cluster"] = cl
    with pytest.raises(eng_mod.JpError) as ex:
        eng_mod.Engine(bad, precision=MIXED, method=abi.JP_METHOD_CANO, alsd=abi.JP_ALSD_LMD, tempco=2)
    assert ex.value.code == abi.JP_E_INVALID


def test_peptide_torsions_stay_unscaled_vs_oracle(eng_mod, clustered):
    """SCALET's peptide-bond exemption: every other torsion marked in tors_unscaled stays in
    class BB with the torsion bit set; energies, class energies and gradients as the oracle."""
    top = dict(clustered, tors_unscaled=(np.arange(len(clustered["tors"])) % 2).astype(np.int32))
    kw = dict(method=abi.JP_METHOD_CANO, alsd=abi.JP_ALSD_LMD, lambda0=0.8, scale_terms=ALL_TERMS)
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
