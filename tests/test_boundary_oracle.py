"""The oracle's atom cut-off (CAL15M= ATOM, enear_ACT_*) and free boundary (BOUNDA= NO,
*_CB variants) against closed forms and identities (no GPU).

ATOM: E = 332.06378/eps q1 q2 / r for r <= CUTLEN, nothing beyond, no self or excess term.
NO: no minimum image -- a droplet in a box too small for it has no image interactions, and
matches the periodic result in a box so large that images never come near.
"""
import numpy as np
import pytest

import oracle
from j_presto_b200 import abi, systems
from tests._util import golden_top, load_golden

GOLD = load_golden()
CCOEF = 332.06378   # eekcal of md_run


@pytest.mark.parametrize("r", [3.0, 11.9, 12.0, 12.4])
def test_atom_cutoff_pair_closed_form(r):
    top = golden_top(GOLD["zd_pair"]["system"])
    top["cord"] = np.array([[5.0, 5.0, 5.0], [5.0 + r, 5.0, 5.0]])
    o = oracle.Oracle(top, method=abi.JP_METHOD_MICR, shake_method=abi.JP_SHAKE_NONE,
                      cal15m=abi.JP_CAL15M_ATOM, cutoff=12.0)
    e, g = o.energy_grad()
    q1, q2 = top["charge"]
    want = CCOEF * q1 * q2 / r if r <= 12.0 else 0.0
    np.testing.assert_allclose(e[abi.JP_E_ELE15], want, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(g[1, 0], -want / r, rtol=1e-12, atol=1e-14)   # dE/dx2 = -q q / r^2
    assert o.dself == 0.0


def test_atom_cutoff_has_no_excess_term():
    top = golden_top(GOLD["bonded_chain"]["system"])
    kw = dict(method=abi.JP_METHOD_MICR, shake_method=abi.JP_SHAKE_NONE, cutoff=12.0)
    ezd = oracle.Oracle(top, **kw).energy_grad()[0]
    eat = oracle.Oracle(top, cal15m=abi.JP_CAL15M_ATOM, **kw).energy_grad()[0]
    # bonded and 1-4 terms are the same; all four atoms exclude each other, so the ZD self
    # and excess terms are the whole of ELE15 there, and nothing is left without ZD
    np.testing.assert_allclose(eat[1:7], ezd[1:7], rtol=1e-14)
    assert abs(ezd[abi.JP_E_ELE15]) > 1e-3 and eat[abi.JP_E_ELE15] == 0.0


@pytest.fixture(scope="module")
def drop():
    return dict(systems.droplet(6, 400, seed=9))


@pytest.mark.parametrize("cal", [abi.JP_CAL15M_ZD, abi.JP_CAL15M_ATOM])
def test_free_boundary_equals_isolated_periodic(drop, cal):
    x = np.asarray(drop["cord"])
    span = (x.max(0) - x.min(0)).max()
    small = dict(drop, box=np.full(3, 28.0))         # too small: images would interact
    huge = dict(drop, box=np.full(3, 2.0 * span + 40.0))
    kw = dict(method=abi.JP_METHOD_CANO, cal15m=cal)
    e_free, g_free = oracle.Oracle(small, bounda=abi.JP_BOUND_NONE, **kw).energy_grad()
    e_huge, g_huge = oracle.Oracle(huge, **kw).energy_grad()
    e_pbc, _ = oracle.Oracle(small, **kw).energy_grad()
    np.testing.assert_allclose(e_free, e_huge, rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(g_free, g_huge, rtol=1e-12, atol=1e-9)
    assert abs(e_pbc[abi.JP_E_ELE15] - e_free[abi.JP_E_ELE15]) > 1.0
