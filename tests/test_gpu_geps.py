"""Partial McMD (GEPSME= AND / OR / XOR) and dnergy's per-class outputs on the GPU, against
the oracle.

* Per-class energies and gradients (jp_energy_grad_cls): FP64 path -- gradients RMS
  relative to the whole gradient 1e-12, class energies 1e-8 of the total; mixed path --
  1e-5 and 1e-5.  ALSD replicas give their three classes (weights set one class at a time).
* 15-step trajectories with the class-1 forces scaled by the McMD weight of the class-1
  energy (METHOD= GE) or by SETTEM / PSETMP (METHOD= CANO): FP64 within 1e-8 A of the
  oracle, mixed within 1e-4 A.
* A replica with regions next to one without in one context equals each run alone (the
  former to 1e-9 A; the latter alone runs the kernels without classes, so to 1e-4 A).
* Refused: partial McMD with nothing to scale the classes (md_run would integrate class 2
  alone), region B with ALSD, the minimiser on a partial-McMD context.
"""
import numpy as np
import pytest

import oracle
from j_presto_b200 import abi, systems
from tests._util import rms_rel

pytestmark = pytest.mark.gpu

FP64, MIXED = abi.JP_PREC_FP64, abi.JP_PREC_MIXED
AND, OR, XOR = abi.JP_GEPS_AND, abi.JP_GEPS_OR, abi.JP_GEPS_XOR
TOL = {FP64: (1e-12, 1e-8), MIXED: (1e-5, 1e-5)}


@pytest.fixture(scope="module")
def eng_mod(engine_lib):
    from j_presto_b200 import engine
    return engine


@pytest.fixture(scope="module")
def chain():
    top = dict(systems.solvated_polymer(12, 900, seed=21))
    res = top["residues"]
    a = np.zeros(top["natom"], np.int32)
    for r in (2, 3, 4):
        a[res[r]] = 1
    ab = a.copy()
    for r in (8, 9):
        ab[res[r]] = 2
    return top, a, ab


def _ge(top, cluster, method):
    t = dict(top, cluster=cluster)
    e1 = oracle.Oracle(t, method=abi.JP_METHOD_MICR, alsd=method).energy_grad_cls()[1][0]
    t["ge"] = systems.mcmd_weight(e1 - 60.0, e1 + 240.0)
    return t


@pytest.mark.parametrize("prec", [FP64, MIXED])
@pytest.mark.parametrize("method,regions", [(AND, "a"), (OR, "a"), (XOR, "a"), (AND, "ab"), (OR, "ab"),
                                            (XOR, "ab")])
def test_class_outputs_vs_oracle(eng_mod, chain, prec, method, regions):
    top, a, ab = chain
    t = dict(top, cluster=a if regions == "a" else ab)
    kw = dict(method=abi.JP_METHOD_CANO, alsd=method, psetmp=600.0, scale_terms=abi.JP_SCALE_TORS)
    eo, eco, go = oracle.Oracle(t, **kw).energy_grad_cls()
    with eng_mod.Engine(t, precision=prec, **kw) as e:
        ee, ec, g = e.energy_grad_cls()
        e2, gt = e.energy_grad()
    gtol, etol = TOL[prec]
    assert len(ec) == 2
    scale = np.sqrt((go.sum(0) ** 2).sum())
    for q in range(2):
        assert np.sqrt(((g[q] - go[q]) ** 2).sum()) < gtol * scale, q
        assert abs(ec[q] - eco[q]) < etol * abs(eo[0]) + 1e-6, (q, ec[q], eco[q])
    assert rms_rel(gt, go.sum(0)) < gtol          # jp_energy_grad: both classes
    assert abs(e2[0] - eo[0]) < etol * abs(eo[0])


@pytest.mark.parametrize("prec", [FP64, MIXED])
def test_alsd_class_outputs_vs_oracle(eng_mod, chain, prec):
    top, a, _ = chain
    t = dict(top, cluster=a)
    kw = dict(method=abi.JP_METHOD_CANO, alsd=abi.JP_ALSD_LMD, lambda0=0.8, scale_terms=abi.JP_SCALE_TORS)
    o = oracle.Oracle(t, **kw)
    eo, eco, go = o.energy_grad_cls()
    with eng_mod.Engine(t, precision=prec, **kw) as e:
        ee, ec, g = e.energy_grad_cls()
        lam, ecl = e.get_lambda()
        _, gt = e.energy_grad()                  # lambda weights back after the per-class call
    gtol, etol = TOL[prec]
    assert len(ec) == 3
    scale = np.sqrt((go.sum(0) ** 2).sum())
    for q in range(3):
        assert np.sqrt(((g[q] - go[q]) ** 2).sum()) < gtol * scale, q
        assert abs(ec[q] - eco[q]) < etol * abs(eo[0]) + 1e-6, q
    w = np.array([0.8 * 0.8, 0.8, 1.0])
    np.testing.assert_allclose(gt, np.tensordot(w, g, 1), rtol=0, atol=10 * gtol * np.abs(gt).max())


@pytest.mark.parametrize("prec", [FP64, MIXED])
@pytest.mark.parametrize("method", [AND, XOR])
def test_ge_trajectory_vs_oracle(eng_mod, chain, prec, method):
    top, a, ab = chain
    t = _ge(top, a if method == AND else ab, method)
    kw = dict(method=abi.JP_METHOD_GE, alsd=method, scale_terms=abi.JP_SCALE_TORS)
    o = oracle.Oracle(t, **kw)
    ier, Eo, To = o.run(15)
    assert ier == 0
    xo, vo = o.get_state()
    with eng_mod.Engine(t, precision=prec, **kw) as e:
        E, T = e.step(15)
        x, v = e.get_state()
    tol = 1e-8 if prec == FP64 else 1e-4
    assert np.abs(x - xo).max() < tol
    np.testing.assert_allclose(E[:, 0, 0], Eo[:, 0], rtol=1e-8 if prec == FP64 else 1e-5, atol=1e-6)


def test_pseudo_temperature_trajectory_vs_oracle(eng_mod, chain):
    top, a, _ = chain
    t = dict(top, cluster=a)
    kw = dict(method=abi.JP_METHOD_CANO, alsd=OR, psetmp=450.0, scale_terms=abi.JP_SCALE_TORS)
    o = oracle.Oracle(t, **kw)
    ier, Eo, To = o.run(15)
    assert ier == 0
    xo, _ = o.get_state()
    with eng_mod.Engine(t, precision=FP64, **kw) as e:
        e.step(15)
        x, _ = e.get_state()
    assert np.abs(x - xo).max() < 1e-8


def test_batch_equals_single(eng_mod, chain):
    top, a, _ = chain
    t1 = _ge(top, a, OR)
    t2 = dict(systems.solvated_polymer(6, 500, seed=23))
    t2["ge"] = systems.mcmd_weight(-5000.0, 5000.0)
    kw = dict(method=abi.JP_METHOD_GE, alsd=OR, precision=MIXED)
    with eng_mod.Engine([t1, t2], **kw) as e:
        e.step(12)
        xb = [e.get_state(r)[0] for r in range(2)]
    with eng_mod.Engine(t1, **kw) as e:   # the same kernels alone
        e.step(12)
        assert np.abs(e.get_state()[0] - xb[0]).max() < 1e-9
    with eng_mod.Engine(t2, **kw) as e:   # alone it takes the kernels without classes
        e.step(12)
        assert np.abs(e.get_state()[0] - xb[1]).max() < 1e-4


def test_refused(eng_mod, chain):
    top, a, ab = chain
    bad = [
        (dict(top, cluster=a), dict(method=abi.JP_METHOD_CANO, alsd=AND)),   # nothing scales class 1
        (dict(top, cluster=a), dict(method=abi.JP_METHOD_MICR, alsd=XOR)),
        (dict(top, cluster=ab), dict(method=abi.JP_METHOD_CANO, alsd=abi.JP_ALSD_LMD, lambda0=0.8)),
    ]
    for t, kw in bad:
        with pytest.raises(eng_mod.JpError) as ei:
            eng_mod.Engine(t, precision=FP64, **kw)
        assert ei.value.code == abi.JP_E_INVALID
    with eng_mod.Engine(dict(top, cluster=a), precision=FP64, method=abi.JP_METHOD_CANO, alsd=AND,
                        psetmp=600.0) as e:
        with pytest.raises(eng_mod.JpError) as ei:
            e.minimize(max_loop=3)
        assert ei.value.code == abi.JP_E_INVALID
