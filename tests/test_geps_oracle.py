"""The oracle's partial McMD (GEPSME= AND / OR / XOR, nfrg = 2) pinned without a GPU.

The region classes follow n_matrix (inpcls.f90:298-325): with region A alone, AND keeps the
A-A terms in class 1, XOR the A-rest terms, OR both, so E1(OR) = E1(AND) + E1(XOR) term for
term; with regions A and B, AND = A-A + B-B, OR = A-A + A-B, XOR = A-B.  The classes sum to
the whole energy and gradient, each class gradient is the derivative of its class energy
(central differences), and the force of the step is dew(E1) grad1 + grad2 with dew the
McMD weight of the class-1 energy (verlethe.f90:196-238) or SETTEM / PSETMP.
"""
import numpy as np
import pytest

import oracle
from j_presto_b200 import abi, systems

AND, OR, XOR = abi.JP_GEPS_AND, abi.JP_GEPS_OR, abi.JP_GEPS_XOR


@pytest.fixture(scope="module")
def chain():
    top = dict(systems.solvated_polymer(6, 250, seed=3))
    res = top["residues"]
    a = np.zeros(top["natom"], np.int32)
    a[res[1]] = 1
    a[res[2]] = 1
    ab = a.copy()
    ab[res[4]] = 2
    return top, a, ab


def cls(top, cluster, method, **kw):
    t = dict(top, cluster=cluster)
    kw.setdefault("psetmp", 600.0)
    kw.setdefault("scale_terms", abi.JP_SCALE_TORS)
    o = oracle.Oracle(t, method=abi.JP_METHOD_CANO, alsd=method, **kw)
    return o, o.energy_grad_cls()


@pytest.mark.parametrize("method", [AND, OR, XOR])
@pytest.mark.parametrize("regions", ["a", "ab"])
def test_classes_sum_to_the_whole(chain, method, regions):
    top, a, ab = chain
    o, (e, ec, g) = cls(top, a if regions == "a" else ab, method)
    assert len(ec) == 2 and g.shape == (2, top["natom"], 3)
    e0, g0 = o.energy_grad()
    assert abs(ec.sum() - e0[0]) < 1e-9 * max(1.0, abs(e0[0]))
    np.testing.assert_allclose(g.sum(0), g0, rtol=0, atol=1e-9)
    assert abs(ec[0]) > 1e-3 and np.abs(g[0]).max() > 1e-3   # both classes populated


def test_or_is_and_plus_xor(chain):
    top, a, ab = chain
    _, (_, e_and, g_and) = cls(top, a, AND)
    _, (_, e_or, g_or) = cls(top, a, OR)
    _, (_, e_xor, g_xor) = cls(top, a, XOR)
    assert abs(e_or[0] - e_and[0] - e_xor[0]) < 1e-9 * max(1.0, abs(e_or[0]))
    np.testing.assert_allclose(g_or[0], g_and[0] + g_xor[0], rtol=0, atol=1e-9)
    # with B: AND = AA + BB, OR = AA + AB, XOR = AB
    b_as_a = (ab == 2).astype(np.int32)
    _, (_, e_aa, g_aa) = cls(top, a, AND)
    _, (_, e_bb, g_bb) = cls(top, b_as_a, AND)
    _, (_, e_and2, g_and2) = cls(top, ab, AND)
    _, (_, e_or2, g_or2) = cls(top, ab, OR)
    _, (_, e_xor2, g_xor2) = cls(top, ab, XOR)
    assert abs(e_and2[0] - e_aa[0] - e_bb[0]) < 1e-9 * max(1.0, abs(e_and2[0]))
    assert abs(e_or2[0] - e_aa[0] - e_xor2[0]) < 1e-9 * max(1.0, abs(e_or2[0]))
    np.testing.assert_allclose(g_and2[0], g_aa[0] + g_bb[0], rtol=0, atol=1e-9)
    np.testing.assert_allclose(g_or2[0], g_aa[0] + g_xor2[0], rtol=0, atol=1e-9)


def test_everything_in_region_a(chain):
    top = chain[0]
    every = np.ones(top["natom"], np.int32)
    scaled = abi.JP_SCALE_BOND | abi.JP_SCALE_ANGLE | abi.JP_SCALE_TORS | abi.JP_SCALE_IMPR
    o, (e, ec, g) = cls(top, every, AND, scale_terms=scaled)   # every term A-A: all class 1
    assert abs(ec[1]) < 1e-12 and np.abs(g[1]).max() < 1e-12
    _, (_, ec2, _) = cls(top, every, AND)      # bonded terms SCALET leaves out: class 2
    assert abs(ec2[1]) > 1e-3
    _, (_, ex, gx) = cls(top, every, XOR, scale_terms=scaled)  # no A-rest term: class 1 empty
    assert abs(ex[0]) < 1e-12 and np.abs(gx[0]).max() < 1e-12
    no = np.zeros(top["natom"], np.int32)      # no region atoms: one class (nfrg = 1)
    _, (_, e1, g1) = cls(top, no, AND)
    assert len(e1) == 1


@pytest.mark.parametrize("method", [AND, XOR])
def test_class_gradient_is_the_class_energy_derivative(chain, method):
    top, a, _ = chain
    o, (_, ec, g) = cls(top, a, method)
    x0 = np.asarray(top["cord"], float).reshape(-1, 3)
    h = 1e-5
    for atom in np.flatnonzero(a)[:3].tolist() + [int(np.flatnonzero(a == 0)[0])]:
        for k in range(3):
            xp, xm = x0.copy(), x0.copy()
            xp[atom, k] += h
            xm[atom, k] -= h
            ep = o.energy_grad_cls(xp)[1]
            em = o.energy_grad_cls(xm)[1]
            fd = (ep - em) / (2 * h)
            np.testing.assert_allclose(fd, g[:, atom, k], rtol=1e-5, atol=1e-5)
    o.energy_grad_cls(x0)


def test_step_force_scales_class_one(chain):
    top, a, _ = chain
    t = dict(top, cluster=a)
    e_cls = oracle.Oracle(t, method=abi.JP_METHOD_MICR, alsd=OR).energy_grad_cls()[1]
    t["ge"] = systems.mcmd_weight(e_cls[0] - 50.0, e_cls[0] + 150.0)
    o = oracle.Oracle(t, method=abi.JP_METHOD_GE, alsd=OR)
    _, ec, g = o.energy_grad_cls()
    dew = o.mcmd_scale(ec[0])
    assert abs(dew - 1.0) > 1e-3
    _, _, gf = o.first_force()
    np.testing.assert_allclose(gf, dew * g[0] + g[1], rtol=0, atol=1e-9)
    # the pseudo temperature scales class 1 by SETTEM / PSETMP
    o2 = oracle.Oracle(dict(top, cluster=a), method=abi.JP_METHOD_CANO, alsd=XOR, psetmp=500.0)
    _, ec2, g2 = o2.energy_grad_cls()
    _, _, gf2 = o2.first_force()
    np.testing.assert_allclose(gf2, (300.0 / 500.0) * g2[0] + g2[1], rtol=0, atol=1e-9)
