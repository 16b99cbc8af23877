"""External CMM environment (EXTCMM=) on the GPU against the oracle: a droplet inside a shell
of frozen point charges, binned into level-1 multipoles on the run's own 4-level grid.

Tolerances as the other CMM tests: FP64 gradient RMS relative 1e-11, energies 1e-8
relative; mixed gradient 1e-5; a 12-step FP64 trajectory within 1e-8 A.
"""
import numpy as np
import pytest

import oracle
from j_presto_b200 import abi, systems
from tests._util import rms_rel

pytestmark = pytest.mark.gpu

FP64, MIXED = abi.JP_PREC_FP64, abi.JP_PREC_MIXED
CELL, NLEV = 4.0, 4
NV = 4 << (NLEV - 1)


@pytest.fixture(scope="module")
def eng_mod(engine_lib):
    from j_presto_b200 import engine
    return engine


def _environment(centre, rng, n=3000, r0=23.0, r1=28.0):
    """Point charges in a shell around `centre`, as level-1 multipoles about the cell centres
    of the grid centred at `centre` (engine layout: q, p, Q_kk/2, Q_kk, Q_xy, Q_yz, Q_zx)."""
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1)[:, None]
    pos = centre + u * rng.uniform(r0, r1, n)[:, None]
    q = rng.choice([-0.5, 0.5], n)
    org = centre - 0.5 * NV * CELL
    m = np.floor((pos - org) / CELL).astype(int)
    flag = np.zeros((NV, NV, NV), np.uint8)
    pot = np.zeros((NV, NV, NV, 13))
    for (ix, iy, iz), qi, p in zip(m, q, pos):
        c = org + CELL * (np.array([ix, iy, iz]) + 0.5)
        d = p - c
        flag[iz, iy, ix] = 1
        P = pot[iz, iy, ix]
        P[0] += qi
        P[1:4] += qi * d
        R = np.array([qi * (3 * d[k] ** 2 - d @ d) for k in range(3)])
        P[4:7] += R / 2
        P[7:10] += R
        P[10:13] += 3 * qi * np.array([d[0] * d[1], d[1] * d[2], d[2] * d[0]])
    return dict(nlev=NLEV, cell=CELL, center=centre, flag=flag, pot=pot)


@pytest.fixture(scope="module")
def drop():
    d = dict(systems.droplet(12, 1200, seed=9), box=np.full(3, 28.0))
    centre = np.round(np.asarray(d["cord"]).mean(0), 1)
    d["ext_cmm"] = _environment(centre, np.random.default_rng(3))
    return d


KW = dict(method=abi.JP_METHOD_CANO, cal15m=abi.JP_CAL15M_CMM, bounda=abi.JP_BOUND_NONE,
          cmm_levels=NLEV, cmm_cell=CELL)


def test_energy_grad_vs_oracle(eng_mod, drop):
    eo, go = oracle.Oracle(drop, **KW).energy_grad()
    e_none, _ = oracle.Oracle(dict(drop, ext_cmm=None), **KW).energy_grad()
    assert abs(eo[abi.JP_E_ELE15] - e_none[abi.JP_E_ELE15]) > 1.0   # the environment acts
    for prec, gtol, etol in ((FP64, 1e-11, 1e-8), (MIXED, 1e-5, 1e-5)):
        with eng_mod.Engine(drop, precision=prec, **KW) as e:
            ene, g = e.energy_grad()
        assert rms_rel(g, go) < gtol
        np.testing.assert_allclose(ene, eo, rtol=etol, atol=1e-6 if prec == FP64 else 1e-2)


def test_trajectory_vs_oracle(eng_mod, drop):
    kw = dict(KW, cmm_update=5, update=10)
    o = oracle.Oracle(drop, **kw)
    ier, Eo, _ = o.run(12)
    assert ier == 0
    xo, vo = o.get_state()
    with eng_mod.Engine(drop, precision=FP64, **kw) as e:
        E, _ = e.step(12)
        x, v = e.get_state()
    assert np.abs(x - xo).max() < 1e-8
    np.testing.assert_allclose(np.asarray(E)[:, 0, :], Eo, rtol=1e-8, atol=1e-6)


def test_environment_needs_four_levels_and_the_cell_size(eng_mod, drop):
    for kw in (dict(KW, cmm_cell=5.0), dict(KW, cmm_levels=3), dict(KW, cal15m=abi.JP_CAL15M_ZD)):
        with pytest.raises(eng_mod.JpError) as ex:
            eng_mod.Engine(drop, precision=MIXED, **kw)
        assert ex.value.code == abi.JP_E_INVALID
