"""The CPU oracle against the closed-form known-answer vectors (tests/golden/kat.json)
and analytic identities.  Pins the oracle before it is used to check the CUDA engine."""
import numpy as np
import pytest

import oracle
from j_presto_b200 import abi, systems
from tests._util import golden_top, load_golden, rms_rel

GOLD = load_golden()
CASES = [k for k in GOLD if not k.startswith("_")]


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_golden(name):
    g = GOLD[name]
    top = golden_top(g["system"])
    o = oracle.Oracle(top, method=abi.JP_METHOD_MICR, shake_method=abi.JP_SHAKE_NONE,
                      cutoff=g["cutoff"])
    e, grad = o.energy_grad()
    np.testing.assert_allclose(e, g["energy"], rtol=1e-10, atol=1e-9)
    np.testing.assert_allclose(grad, np.array(g["grad"]), rtol=1e-5, atol=1e-5)


def test_cutoff_edge_pair_counts():
    """r == rc interacts (co = 1 at equality); rc < r <= rc+1.5 is listed but contributes
    nothing; r > rc+1.5 is not listed (cutoff.f90 `dd .le. rlim2`, enear.f90:134)."""
    g = GOLD["cutoff_edge"]
    o = oracle.Oracle(golden_top(g["system"]), method=abi.JP_METHOD_MICR,
                      shake_method=abi.JP_SHAKE_NONE, cutoff=12.0)
    o.energy_grad()
    # pairs: (0,1) 12.0 A in, (0,2) 12.5 A listed only, (0,3) 14 A not listed,
    # (1,2),(1,3),(2,3) beyond the list radius
    assert o.npairs_listed == 2
    assert o.npairs_cut == 1


def test_mcmd_weight_golden():
    m = GOLD["_mcmd"]
    top = golden_top(GOLD["zd_pair"]["system"])
    top["ge"] = m["ge"]
    o = oracle.Oracle(top, method=abi.JP_METHOD_GE, shake_method=abi.JP_SHAKE_NONE)
    got = [o.mcmd_scale(e) for e in m["energies"]]
    np.testing.assert_allclose(got, m["scale"], rtol=1e-13)


def test_dself_neutral_molecule_is_zero():
    g = GOLD["water"]
    o = oracle.Oracle(golden_top(g["system"]), method=abi.JP_METHOD_MICR,
                      shake_method=abi.JP_SHAKE_NONE)
    assert abs(o.dself) < 1e-12


@pytest.fixture(scope="module")
def poly():
    return systems.solvated_polymer(6, 700, seed=11)


def test_oracle_gradient_is_energy_derivative(poly):
    o = oracle.Oracle(poly, method=abi.JP_METHOD_CANO)
    x = poly["cord"].copy()
    e, g = o.energy_grad(x)
    rng = np.random.default_rng(0)
    for i in rng.choice(poly["natom"], 10, replace=False):
        for k in range(3):
            h = 1e-6
            xp, xm = x.copy(), x.copy()
            xp[i, k] += h
            xm[i, k] -= h
            fd = (o.energy_grad(xp)[0][0] - o.energy_grad(xm)[0][0]) / (2 * h)
            assert abs(fd - g[i, k]) < 1e-4 * max(1.0, abs(g[i, k]))


def test_oracle_shake_restores_constraints(poly):
    o = oracle.Oracle(poly, method=abi.JP_METHOD_MICR)
    rng = np.random.default_rng(1)
    x0 = poly["cord"]
    x1 = x0 + rng.normal(0.0, 0.01, size=x0.shape)
    ier, r = o.shake(x1, x0)
    assert ier == 0
    pairs = [(0, 1), (1, 2), (2, 0), (3, 0), (2, 3), (1, 3)]
    for n, a, d in zip(poly["shake_n"], poly["shake_atoms"], poly["shake_dist"]):
        for q in range(n * (n - 1) // 2):
            i, j = a[pairs[q][0]], a[pairs[q][1]]
            dd = np.sum((r[i] - r[j]) ** 2)
            assert abs(dd - d[q] ** 2) < 1e-6 * d[q] ** 2


def test_oracle_nve_energy_conservation():
    """Leap-frog NVE on an equilibrated small water box: total energy drifts little."""
    top = systems.water_box(300, 28.0, seed=5)
    o = oracle.Oracle(top, method=abi.JP_METHOD_CANO, dt=1.0)
    ier, _, _ = o.run(200)
    assert ier == 0
    x, v = o.get_state()
    m = oracle.Oracle(top, method=abi.JP_METHOD_MICR, dt=1.0)
    m.set_state(x, v)
    m.rebuild()
    ier, E, T = m.run(200)
    assert ier == 0
    # total = potential + kinetic (KE from T and DOF: ek = T*R*ndf/2 kcal/mol)
    ek = T * 8.31451e-3 / 4.184 * m.dof / 2.0
    tot = E[:, 0] + ek
    assert np.std(tot[20:]) < 0.05 * np.std(E[20:, 0]) + 1.0
