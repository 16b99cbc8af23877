"""The oracle's cell multipole method (CAL15M= CMM, BOUNDA= NO) against independent
restatements and physics (no GPU).

* celpol: the multipoles of every cell at every level equal the moments of the charges in
  it about the cell centre (monopole, dipole, traceless quadrupole in md_run's storage:
  [q, p, Q_kk/2, Q_kk, Q_xy, Q_yz, Q_zx]); level-to-level translation is exact to this order.
* cmmdo / mk_cm: the far field (energy and gradient) equals a numpy sum of the Cartesian
  multipole expansion of every non-empty far cell -- the children of the parent's
  neighbours minus the own neighbours, every non-neighbour at the top level.
* near + far approximates the direct Coulomb sum (gradient within a few percent).
"""
import numpy as np
import pytest

import oracle
from j_presto_b200 import abi, systems

CCOEF = 332.06378
CMM = dict(method=abi.JP_METHOD_CANO, cal15m=abi.JP_CAL15M_CMM, bounda=abi.JP_BOUND_NONE)


@pytest.fixture(scope="module")
def drop():
    d = dict(systems.droplet(8, 500, seed=4))
    return dict(d, c6=np.zeros_like(d["c6"]), c12=np.zeros_like(d["c12"]))   # Coulomb only


def _cells(o, x):
    lv = o.cmm_levels()
    cen1 = lv[0][2]
    siz1 = cen1[1, 0] - cen1[0, 0]
    m = np.floor((x - (cen1[0] - 0.5 * siz1)) / siz1).astype(int)   # 0-based, all in range
    return lv, m


def test_multipoles_are_the_cell_moments(drop):
    o = oracle.Oracle(drop, cmm_cell=4.0, **CMM)
    o.energy_grad()
    x, q = np.asarray(drop["cord"]), np.asarray(drop["charge"])
    lv, m = _cells(o, x)
    assert len(lv) >= 3
    for L, (pot, pop, cen) in enumerate(lv):
        nv = len(cen)
        mm = m // (2 ** L)
        for cid in np.nonzero(pop)[0]:
            ix, iy, iz = cid % nv, (cid // nv) % nv, cid // (nv * nv)
            sel = (mm[:, 0] == ix) & (mm[:, 1] == iy) & (mm[:, 2] == iz)
            d = x[sel] - np.array([cen[ix, 0], cen[iy, 1], cen[iz, 2]])
            qq = q[sel]
            R = [(qq * (2 * d[:, k] ** 2 - d[:, (k + 1) % 3] ** 2 - d[:, (k + 2) % 3] ** 2)).sum()
                 for k in range(3)]
            want = np.r_[qq.sum(), (qq[:, None] * d).sum(0), np.array(R) / 2, R,
                         [3 * (qq * d[:, k] * d[:, (k + 1) % 3]).sum() for k in range(3)]]
            assert pop[cid] == sel.sum()
            np.testing.assert_allclose(pot[cid], want, rtol=1e-11, atol=1e-11)


def _far_numpy(o, x, q):
    lv, m = _cells(o, x)
    nlev = len(lv)
    e = 0.0
    g = np.zeros_like(x)
    for L, (pot, pop, cen) in enumerate(lv):
        nv = len(cen)
        a = m // (2 ** L)
        for i in range(len(x)):
            if L < nlev - 1:   # children of the parent's neighbours
                p = a[i] // 2
                lo = np.maximum(p - 1, 0) * 2
                hi = np.minimum(p + 1, nv // 2 - 1) * 2 + 1
            else:
                lo, hi = np.zeros(3, int), np.full(3, nv - 1)
            rng = [np.arange(lo[k], hi[k] + 1) for k in range(3)]
            KZ, KY, KX = np.meshgrid(rng[2], rng[1], rng[0], indexing="ij")
            kx, ky, kz = KX.ravel(), KY.ravel(), KZ.ravel()
            near = (np.abs(kx - a[i, 0]) <= 1) & (np.abs(ky - a[i, 1]) <= 1) & (np.abs(kz - a[i, 2]) <= 1)
            cid = ((kz * nv + ky) * nv + kx)[~near]
            cid = cid[pop[cid] > 0]
            Q = pot[cid]
            d = x[i] - np.stack([cen[cid % nv, 0], cen[(cid // nv) % nv, 1], cen[cid // (nv * nv), 2]], 1)
            r2 = (d * d).sum(1)
            r = np.sqrt(r2)
            # potential of monopole + dipole + traceless quadrupole and its gradient
            quad = (Q[:, 4] * d[:, 0] ** 2 + Q[:, 5] * d[:, 1] ** 2 + Q[:, 6] * d[:, 2] ** 2 +
                    Q[:, 10] * d[:, 0] * d[:, 1] + Q[:, 11] * d[:, 1] * d[:, 2] + Q[:, 12] * d[:, 2] * d[:, 0])
            dip = (Q[:, 1:4] * d).sum(1)
            phi = Q[:, 0] / r + dip / r ** 3 + quad / r ** 5
            gq = np.stack([2 * Q[:, 4] * d[:, 0] + Q[:, 10] * d[:, 1] + Q[:, 12] * d[:, 2],
                           2 * Q[:, 5] * d[:, 1] + Q[:, 10] * d[:, 0] + Q[:, 11] * d[:, 2],
                           2 * Q[:, 6] * d[:, 2] + Q[:, 11] * d[:, 1] + Q[:, 12] * d[:, 0]], 1)
            gphi = (-Q[:, 0:1] * d / r[:, None] ** 3 + Q[:, 1:4] / r[:, None] ** 3 -
                    3 * dip[:, None] * d / r[:, None] ** 5 + gq / r[:, None] ** 5 -
                    5 * quad[:, None] * d / r[:, None] ** 7)
            e += 0.5 * CCOEF * q[i] * phi.sum()
            g[i] += CCOEF * q[i] * gphi.sum(0)
    return e, g


def test_far_field_equals_multipole_expansion_sum(drop):
    o = oracle.Oracle(drop, cmm_cell=4.0, **CMM)
    o.energy_grad()
    ef, gf = o.cmm_far()
    x, q = np.asarray(drop["cord"]), np.asarray(drop["charge"])
    e, g = _far_numpy(o, x, q)
    np.testing.assert_allclose(ef, e, rtol=1e-10)
    np.testing.assert_allclose(gf, g, rtol=1e-9, atol=1e-9 * np.abs(g).max())


def test_cmm_approximates_direct_coulomb(drop):
    _, g = oracle.Oracle(drop, **CMM).energy_grad()
    _, gd = oracle.Oracle(drop, method=abi.JP_METHOD_CANO, cal15m=abi.JP_CAL15M_ATOM,
                          bounda=abi.JP_BOUND_NONE, cutoff=500.0).energy_grad()
    assert np.sqrt(((g - gd) ** 2).sum() / (gd ** 2).sum()) < 0.03


def test_far_field_cadence(drop):
    """The far field is evaluated at steps 1, 1 + CMMUPD, ... and reused in between
    (md.f90:680-684): energies of steps 2-5 carry the far field of step 1."""
    o = oracle.Oracle(drop, cmm_update=5, update=10, **CMM)
    ier, e, _ = o.run(6)
    assert ier == 0
    ef1 = o.cmm_far()[0]   # the far field of step 6 (recomputed there)
    o2 = oracle.Oracle(drop, cmm_update=5, update=10, **CMM)
    o2.run(1)
    ef0 = o2.cmm_far()[0]
    o2.run(4)
    assert o2.cmm_far()[0] == ef0     # steps 2-5 reuse it
    assert ef1 != ef0


def test_celres_cells_follow_the_residue_centre():
    """CELRES (celpar.f90:131-153): the level-1 populations are those of the residues'
    geometric centres, every atom of a residue counted in its residue's cell."""
    top = dict(systems.droplet(6, 400, seed=9))
    t = np.asarray(top["atype"])
    ow = np.flatnonzero(t == systems.T_OW)
    res = np.array([(o, o + 2) for o in ow], np.int32)
    kw = dict(method=abi.JP_METHOD_CANO, cal15m=abi.JP_CAL15M_CMM, bounda=abi.JP_BOUND_NONE)
    o = oracle.Oracle(dict(top, celres=res), **kw)
    o.energy_grad()
    _, pop, cen = o.cmm_levels()[0]
    x = np.asarray(top["cord"], float)
    pos = x.copy()
    for f, l in res:
        pos[f:l + 1] = x[f:l + 1].mean(0)
    siz = cen[1, 0] - cen[0, 0]
    org = cen[0] - 0.5 * siz
    m = np.floor((pos - org) / siz).astype(int)   # all inside: floor = int() here
    nv = len(cen)
    want = np.zeros(nv ** 3, int)
    np.add.at(want, (m[:, 2] * nv + m[:, 1]) * nv + m[:, 0], 1)
    np.testing.assert_array_equal(pop, want)
    plain = oracle.Oracle(top, **kw)
    plain.energy_grad()
    assert not np.array_equal(plain.cmm_levels()[0][1], pop)
