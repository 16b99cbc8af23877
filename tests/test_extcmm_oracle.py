"""The oracle's external CMM environment (EXTCMM=, enear_extCMM.f90) against closed forms
(no GPU): one atom of charge q beside one occupied external cell holding a point charge Q.

Beyond 1.5 cell sizes from the cell centre the term is the Coulomb energy 332.06378 q Q / r
(the multipole expansion of a monopole is exact), times md_run's factor 0.5; inside, the
value on that sphere is blended towards the centre by a cubic in r, continuous in energy
and force with the outside at the sphere.
"""
import numpy as np
import pytest

import oracle
from j_presto_b200 import abi

CCOEF = 332.06378
CELL, NLEV = 6.0, 4
NV = 4 << (NLEV - 1)        # 32 level-1 cells per axis


def _one_atom(x, q=0.6):
    return dict(natom=1, box=np.full(3, 60.0), cord=np.array([x], float), vel=np.zeros((1, 3)),
                mass=np.array([12.0]), charge=np.array([q]), atype=np.zeros(1, np.int32),
                molecule=np.zeros(1, np.int32), ntype=1, c6=np.zeros((1, 1)), c12=np.zeros((1, 1)),
                s14_vdw=np.full(1, 0.5), s14_ele=np.full(1, 1 / 1.2),
                excl_ptr=np.zeros(2, np.int32), excl_idx=np.zeros(0, np.int32),
                bond=np.zeros((0, 2), np.int32), bond_k=np.zeros(0), bond_r0=np.zeros(0),
                angle=np.zeros((0, 3), np.int32), angle_k=np.zeros(0), angle_theta0=np.zeros(0),
                tors=np.zeros((0, 4), np.int32), tors_k=np.zeros(0), tors_nrot=np.zeros(0),
                tors_phase=np.zeros(0), tors_div=np.zeros(0, np.int32), tors_nbf=np.zeros(0, np.int32),
                impr=np.zeros((0, 4), np.int32), impr_k=np.zeros(0), impr_nrot=np.zeros(0),
                impr_phase=np.zeros(0), impr_div=np.zeros(0, np.int32),
                shake_n=np.zeros(0, np.int32), shake_atoms=np.zeros((0, 4), np.int32),
                shake_dist=np.zeros((0, 6)))


def _env(Q=-0.8, cell=(16, 16, 16)):
    """A grid centred at the origin with one occupied cell holding Q at its centre."""
    flag = np.zeros((NV, NV, NV), np.uint8)
    pot = np.zeros((NV, NV, NV, 13))
    ix, iy, iz = cell                                    # 0-based, x fastest in memory
    flag[iz, iy, ix] = 1
    pot[iz, iy, ix, 0] = Q
    centre = np.array([CELL * (i + 1 - 0.5 * (NV + 1)) for i in cell])
    return dict(nlev=NLEV, cell=CELL, center=np.zeros(3), flag=flag, pot=pot), centre


def _energy_grad(x, env):
    top = dict(_one_atom(x), ext_cmm=env)
    o = oracle.Oracle(top, method=abi.JP_METHOD_MICR, shake_method=abi.JP_SHAKE_NONE,
                      cal15m=abi.JP_CAL15M_CMM, bounda=abi.JP_BOUND_NONE, cmm_levels=NLEV,
                      cmm_cell=CELL)
    e, g = o.energy_grad()
    return e[abi.JP_E_ELE15], g[0]


@pytest.mark.parametrize("r", [9.5, 11.0, 14.0])
def test_outside_the_sphere_is_coulomb(r):
    env, c = _env()
    u = np.array([1.0, -1.0, 1.0]) / np.sqrt(3.0)   # along a diagonal: still a neighbour cell
    e, g = _energy_grad(c + r * u, env)
    want = 0.5 * CCOEF * 0.6 * -0.8 / r
    np.testing.assert_allclose(e, want, rtol=1e-13)
    np.testing.assert_allclose(g, -2.0 * want / r * u, rtol=1e-12, atol=1e-14)   # ccoef q Q d / r^3


def test_blend_is_continuous_and_closed_form():
    """Energy and force meet the Coulomb values at r = 1.5 cells; inside, for a monopole Q:
    with E0 = Q/R, F0 = Q/R^2, t = r/R and B = F0 r, E = (2E0 + B) t^3 - (3E0 + B) t^2 + 2E0
    and the force is the sphere's field times r/R^3 (6E0 (r - R) + B (3r - 2R)) / F0
    (enear_extCMM.f90:80-125)."""
    env, c = _env(Q=-0.8)
    R = 1.5 * CELL
    u = np.array([0.6, 0.0, 0.8])
    e_in, g_in = _energy_grad(c + R * (1 - 1e-10) * u, env)
    e_out, g_out = _energy_grad(c + R * (1 + 1e-10) * u, env)
    np.testing.assert_allclose(e_in, e_out, rtol=1e-8)
    np.testing.assert_allclose(g_in, g_out, rtol=1e-8)
    Q, q = -0.8, 0.6
    for r in (2.0, 5.0, 8.0):
        e, g = _energy_grad(c + r * u, env)
        E0, F0 = Q / R, abs(Q) / R ** 2
        B, t = F0 * r, r / R
        E = (2 * E0 + B) * t ** 3 - (3 * E0 + B) * t ** 2 + 2 * E0
        np.testing.assert_allclose(e, 0.5 * CCOEF * q * E, rtol=1e-12)
        sf = r / R ** 3 * (6 * E0 * (r - R) + B * (3 * r - 2 * R)) / F0
        np.testing.assert_allclose(g, CCOEF * q * (-Q * u / R ** 2) * sf, rtol=1e-12, atol=1e-14)


def test_cells_beyond_the_neighbours_are_not_seen():
    env, c = _env()
    e, g = _energy_grad(c + np.array([2.5 * CELL, 0.0, 0.0]), env)   # two cells away
    assert e == 0.0 and not g.any()
