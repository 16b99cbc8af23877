"""The oracle's hydrogen-bond 10-12 pairs (iyppid = 2: cutoff.f90:98-154 splits them off,
enear.f90:330-516 evaluates them) against closed forms and a brute-force sum (no GPU).

A marked type pair keeps its Coulomb term, loses its 12-6 term and gets
E = C12h/r^12 - C10/r^10 for r <= CUTLEN in the JP_E_HBOND slot; 1-4 pairs of those types
keep the 12-6 term (dnergv.f90:490).
"""
import numpy as np
import pytest

import oracle
from j_presto_b200 import abi, systems
from tests._util import golden_top, load_golden

GOLD = load_golden()
HB = abi.JP_E_HBOND


def _mark(top, pairs, c10=1800.0, c12h=5400.0):
    nt = int(top["ntype"])
    hb = np.zeros((nt, nt), np.int32)
    a10 = np.zeros((nt, nt))
    a12 = np.zeros((nt, nt))
    for i, j in pairs:
        hb[i, j] = hb[j, i] = 1
        a10[i, j] = a10[j, i] = c10
        a12[i, j] = a12[j, i] = c12h
    return dict(top, hbond=hb, c10=a10, c12h=a12)


@pytest.mark.parametrize("cal", [abi.JP_CAL15M_ZD, abi.JP_CAL15M_ATOM])
@pytest.mark.parametrize("r", [1.7, 2.4, 11.9, 12.4])
def test_pair_closed_form(cal, r):
    top = golden_top(GOLD["zd_pair"]["system"])
    top["cord"] = np.array([[5.0, 5.0, 5.0], [5.0 + r, 5.0, 5.0]])
    hb = _mark(top, [(0, 0)])
    kw = dict(method=abi.JP_METHOD_MICR, shake_method=abi.JP_SHAKE_NONE, cal15m=cal, cutoff=12.0)
    e0, g0 = oracle.Oracle(top, **kw).energy_grad()
    e1, g1 = oracle.Oracle(hb, **kw).energy_grad()
    want = 5400.0 / r ** 12 - 1800.0 / r ** 10 if r <= 12.0 else 0.0
    dwant = -12.0 * 5400.0 / r ** 13 + 10.0 * 1800.0 / r ** 11 if r <= 12.0 else 0.0   # dE/dr
    np.testing.assert_allclose(e1[HB], want, rtol=1e-12, atol=1e-15)
    assert e1[abi.JP_E_VDW15] == 0.0
    np.testing.assert_allclose(e1[abi.JP_E_ELE15], e0[abi.JP_E_ELE15], rtol=1e-14)
    # the Coulomb part of the gradient is the same; the 10-12 part is dE/dr along x
    g_coul = g0.copy()
    if r <= 12.0:
        lj = -12.0 * np.ravel(top["c12"])[0] / r ** 13 + 6.0 * np.ravel(top["c6"])[0] / r ** 7
        g_coul[1, 0] -= lj
        g_coul[0, 0] += lj
    np.testing.assert_allclose(g1[1, 0] - g_coul[1, 0], dwant, rtol=1e-10, atol=1e-14)
    np.testing.assert_allclose(g1.sum(0), 0.0, atol=1e-12)


def test_one_four_pairs_keep_the_12_6_term():
    top = golden_top(GOLD["bonded_chain"]["system"])
    kw = dict(method=abi.JP_METHOD_MICR, shake_method=abi.JP_SHAKE_NONE, cutoff=12.0)
    e0, g0 = oracle.Oracle(top, **kw).energy_grad()
    e1, g1 = oracle.Oracle(_mark(top, [(1, 1), (0, 1)]), **kw).energy_grad()
    # all four atoms exclude each other: no 1-5 pair, so nothing changes
    np.testing.assert_array_equal(e1, e0)
    np.testing.assert_array_equal(g1, g0)
    assert e0[abi.JP_E_VDW14] != 0.0


def _brute_hbond(top, cutoff):
    """Sum of C12h/r^12 - C10/r^10 and its gradient over the non-excluded marked pairs
    within the cut-off, minimum image."""
    x = np.asarray(top["cord"], float)
    n = len(x)
    t = np.asarray(top["atype"])
    hb, c10, c12h = top["hbond"], top["c10"], top["c12h"]
    box = np.asarray(top["box"], float)
    ptr, idx = top["excl_ptr"], top["excl_idx"]
    e, g = 0.0, np.zeros_like(x)
    for i in range(n):
        js = np.arange(i + 1, n)
        js = js[hb[t[i], t[js]] != 0]
        js = js[~np.isin(js, idx[ptr[i]:ptr[i + 1]])]
        d = x[i] - x[js]
        d -= box * np.round(d / box)
        r2 = (d * d).sum(1)
        ok = r2 <= cutoff * cutoff
        js, d, r2 = js[ok], d[ok], r2[ok]
        v1 = c10[t[i], t[js]] / r2 ** 5
        v2 = c12h[t[i], t[js]] / r2 ** 6
        e += (v2 - v1).sum()
        f = ((-12.0 * v2 + 10.0 * v1) / r2)[:, None] * d   # dE/dxi per pair
        g[i] += f.sum(0)
        np.add.at(g, js, -f)
    return e, g


@pytest.mark.parametrize("cal", [abi.JP_CAL15M_ZD, abi.JP_CAL15M_ATOM])
def test_system_matches_brute_force(cal):
    top = dict(systems.solvated_polymer(8, 300, seed=3))
    hb = systems.with_hbond(top, pairs=systems.HBOND_PAIRS + ((systems.T_HW, systems.T_OW),))
    marked = hb["hbond"] != 0
    # the same system with the 12-6 term of the marked type pairs removed everywhere
    nolj = dict(top, c6=np.where(marked, 0.0, top["c6"]), c12=np.where(marked, 0.0, top["c12"]))
    kw = dict(method=abi.JP_METHOD_CANO, cal15m=cal)
    e1, g1 = oracle.Oracle(hb, **kw).energy_grad()
    e0, g0 = oracle.Oracle(nolj, **kw).energy_grad()
    e14 = oracle.Oracle(top, **kw).energy_grad()[0][abi.JP_E_VDW14]
    eb, gb = _brute_hbond(hb, 12.0)
    assert eb < -10.0
    np.testing.assert_allclose(e1[HB], eb, rtol=1e-11)
    np.testing.assert_allclose(e1[abi.JP_E_ELE15], e0[abi.JP_E_ELE15], rtol=1e-13)
    np.testing.assert_allclose(e1[abi.JP_E_VDW15], e0[abi.JP_E_VDW15], rtol=1e-12)
    np.testing.assert_allclose(e1[abi.JP_E_VDW14], e14, rtol=1e-14)   # 1-4 keeps 12-6
    np.testing.assert_allclose(e1[0], e0[0] + eb + e14 - e0[abi.JP_E_VDW14], rtol=1e-11)
    # gradients: apart from the atoms of 1-4 pairs (whose 12-6 term differs between the
    # two runs) the difference is the brute-force 10-12 gradient
    tors = np.asarray(hb["tors"])[np.asarray(hb["tors_nbf"]) == 1]
    others = np.setdiff1d(np.arange(hb["natom"]), np.unique(tors[:, [0, 3]]))
    np.testing.assert_allclose((g1 - g0)[others], gb[others], rtol=0, atol=1e-9)


def test_cmm_is_refused():
    top = systems.with_hbond(dict(systems.droplet(4, 100, seed=9)))
    with pytest.raises(ValueError):
        oracle.Oracle(top, cal15m=abi.JP_CAL15M_CMM, bounda=abi.JP_BOUND_NONE)
