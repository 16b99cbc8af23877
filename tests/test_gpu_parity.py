"""CUDA engine (through the C ABI) against the oracle and the golden vectors.

Tolerances: FP64 path -- forces RMS relative 1e-12, energies 1e-8 relative; mixed path
(FP32 pair arithmetic, 64-bit fixed-point accumulation) -- forces RMS relative 1e-5,
the accuracy bar the engine is specified to.
"""
import numpy as np
import pytest

import oracle
from j_presto_b200 import abi, systems
from tests._util import golden_top, load_golden, rms_rel

pytestmark = pytest.mark.gpu

FP64, MIXED = abi.JP_PREC_FP64, abi.JP_PREC_MIXED
GOLD = load_golden()
CASES = [k for k in GOLD if not k.startswith("_")]


@pytest.fixture(scope="module")
def eng_mod(engine_lib):
    from j_presto_b200 import engine
    return engine


@pytest.fixture(scope="module")
def water():
    return systems.config_c1_prime()


@pytest.fixture(scope="module")
def poly():
    return systems.solvated_polymer(20, 1500, seed=7)


@pytest.mark.parametrize("prec", [FP64, MIXED])
@pytest.mark.parametrize("name", CASES)
def test_golden_energy_grad(eng_mod, name, prec):
    g = GOLD[name]
    top = golden_top(g["system"])
    with eng_mod.Engine(top, precision=prec, method=abi.JP_METHOD_MICR,
                        shake_method=abi.JP_SHAKE_NONE, cutoff=g["cutoff"]) as e:
        ene, grad = e.energy_grad()
    gold_g = np.array(g["grad"])
    if prec == FP64:
        np.testing.assert_allclose(ene, g["energy"], rtol=1e-9, atol=1e-8)
        np.testing.assert_allclose(grad, gold_g, rtol=1e-5, atol=1e-5)
    else:
        np.testing.assert_allclose(ene, g["energy"], rtol=1e-5, atol=1e-4)
        np.testing.assert_allclose(grad, gold_g, rtol=1e-4, atol=1e-4)


@pytest.mark.parametrize("sysname", ["water", "poly"])
def test_energy_grad_vs_oracle(eng_mod, request, sysname):
    top = request.getfixturevalue(sysname)
    o = oracle.Oracle(top, method=abi.JP_METHOD_MICR)
    eo, go = o.energy_grad()
    for prec in (FP64, MIXED):
        with eng_mod.Engine(top, precision=prec, method=abi.JP_METHOD_MICR) as e:
            ene, g = e.energy_grad()
            assert e.pair_count() == o.npairs_cut
            ntile, nlisted, _ = e.list_stats()
            assert nlisted == o.npairs_listed
        if prec == FP64:
            assert rms_rel(g, go) < 1e-12
            np.testing.assert_allclose(ene, eo, rtol=1e-8, atol=1e-7)
        else:
            assert rms_rel(g, go) < 1e-5
            np.testing.assert_allclose(ene, eo, rtol=1e-5, atol=1e-2)


@pytest.mark.parametrize("method", [abi.JP_METHOD_MICR, abi.JP_METHOD_CANO])
def test_trajectory_vs_oracle(eng_mod, poly, method):
    """20 steps through two pair-list rebuilds (UPDATE=10)."""
    o = oracle.Oracle(poly, method=method)
    ier, Eo, To = o.run(20)
    assert ier == 0
    xo, vo = o.get_state()
    for prec, tol in ((FP64, 1e-8), (MIXED, 1e-4)):
        with eng_mod.Engine(poly, precision=prec, method=method) as e:
            E, T = e.step(20)
            x, v = e.get_state()
        assert np.abs(x - xo).max() < tol
        np.testing.assert_allclose(E[:, 0, 0], Eo[:, 0], rtol=1e-6 if prec == FP64 else 1e-4,
                                   atol=1e-3 if prec == FP64 else 0.5)


def test_mixed_is_bit_reproducible(eng_mod, poly):
    out = []
    for _ in range(2):
        with eng_mod.Engine(poly, precision=MIXED, method=abi.JP_METHOD_CANO) as e:
            e.step(15)
            out.append(e.get_state()[0])
    assert np.array_equal(out[0], out[1])


def test_replica_batch_equals_single(eng_mod, poly, water):
    p2 = systems.solvated_polymer(8, 900, seed=3)
    tops = [poly, water, p2]
    singles = []
    for t in tops:
        with eng_mod.Engine(t, precision=MIXED, method=abi.JP_METHOD_MICR) as e:
            singles.append(e.energy_grad())
    with eng_mod.Engine(tops, precision=MIXED, method=abi.JP_METHOD_MICR) as e:
        for r, (es, gs) in enumerate(singles):
            eb, gb = e.energy_grad(rep=r)
            assert np.array_equal(gb, gs)
            np.testing.assert_allclose(eb, es, rtol=1e-9, atol=1e-6)


def test_shake_hook_vs_oracle(eng_mod, poly):
    rng = np.random.default_rng(3)
    x0 = poly["cord"]
    x1 = x0 + rng.normal(0.0, 0.01, size=x0.shape)
    o = oracle.Oracle(poly, method=abi.JP_METHOD_MICR)
    ier, ro = o.shake(x1, x0)
    with eng_mod.Engine(poly, precision=FP64, method=abi.JP_METHOD_MICR) as e:
        code, rg = e.shake(x1, x0)
    assert ier == 0 and code == 0
    assert np.abs(rg - ro).max() < 1e-10


def test_mcmd_steps_vs_oracle(eng_mod, poly):
    top = dict(poly)
    o0 = oracle.Oracle(poly, method=abi.JP_METHOD_MICR)
    e0 = o0.energy_grad()[0][0]
    top["ge"] = systems.mcmd_weight(e0 - 400.0, e0 + 2600.0)
    o = oracle.Oracle(top, method=abi.JP_METHOD_GE)
    ier, Eo, _ = o.run(10)
    assert ier == 0
    xo, _ = o.get_state()
    with eng_mod.Engine(top, precision=FP64, method=abi.JP_METHOD_GE) as e:
        E, _ = e.step(10)
        x, _ = e.get_state()
    assert np.abs(x - xo).max() < 1e-8


def test_heating_ramp_vs_oracle(eng_mod, poly):
    kw = dict(method=abi.JP_METHOD_CANO, temp_start=100.0, heat_loop=50, tempco=1)
    o = oracle.Oracle(poly, **kw)
    ier, Eo, To = o.run(12)
    xo, _ = o.get_state()
    with eng_mod.Engine(poly, precision=FP64, **kw) as e:
        E, T = e.step(12)
        x, _ = e.get_state()
    assert np.abs(x - xo).max() < 1e-8


def test_invalid_topology_is_rejected(eng_mod, poly):
    bad = dict(poly)
    bad["bond"] = poly["bond"].copy()
    bad["bond"][0, 0] = poly["natom"] + 5
    with pytest.raises(eng_mod.JpError) as ex:
        eng_mod.Engine(bad, precision=MIXED)
    assert ex.value.code == abi.JP_E_INVALID
    with pytest.raises(eng_mod.JpError):
        eng_mod.Engine(poly, precision=MIXED, method=abi.JP_METHOD_GE)   # GE needs a weight


def test_shake_nonconvergence_is_reported(eng_mod, poly):
    """LIMSHK too small: the step returns md_run's ier = 1 warning, nothing faults."""
    with eng_mod.Engine(poly, precision=FP64, method=abi.JP_METHOD_MICR,
                        shake_method=abi.JP_SHAKE_ALLB, shake_maxit=1) as e:
        e.step(1, warn_ok=True)
        assert e.last_code == abi.JP_W_SHAKE_NOT_CONVERGED
