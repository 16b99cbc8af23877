"""The oracle's restraints (dneres.f90: dposc, ddistc, dcdihe) and CAP (dnecap.f90 iufcap 1:
sphere, box and ellipsoid shapes) against closed forms written independently in numpy,
finite differences of their energies, and the ALSD class rules (no GPU).
"""
import numpy as np
import pytest

import oracle
from j_presto_b200 import abi, systems

SLOTS = [abi.JP_E_POSRES, abi.JP_E_DISTRES, abi.JP_E_DIHERES, abi.JP_E_CAP]
CANO, NONE = abi.JP_METHOD_CANO, abi.JP_BOUND_NONE


@pytest.fixture(scope="module")
def poly():
    return systems.with_restraints(dict(systems.solvated_polymer(8, 300, seed=3)))


@pytest.fixture(scope="module")
def drop():
    return systems.with_restraints(dict(systems.droplet(6, 400, seed=9)), cap=True)


def _plain(top):
    return {k: v for k, v in top.items() if k != "restraints"}


def _image(d, box, pbc):
    return d - box * np.round(d / box) if pbc else d


def _dihedral(x, q):
    b1, b2, b3 = x[q[1]] - x[q[0]], x[q[2]] - x[q[1]], x[q[3]] - x[q[2]]
    n1, n2 = np.cross(b1, b2), np.cross(b2, b3)
    return np.arctan2(np.dot(np.cross(n1, n2), b2) / np.linalg.norm(b2), np.dot(n1, n2)) % (2 * np.pi)


def _numpy_energies(top, pbc):
    """The four restraint energies from the documented formulas."""
    x = np.asarray(top["cord"], float)
    box = np.asarray(top["box"], float)
    rd = top["restraints"]
    atoms, k, ref = rd["pos"]
    d = _image(x[atoms] - ref, box, pbc)
    epos = 0.5 * (k * (d * d).sum(1)).sum()
    edist = 0.0
    for gi, gj, lo, up, klo, kup in zip(*rd["dist"]):
        r = np.array([np.linalg.norm(_image(x[a] - x[b], box, pbc)) for a in gi for b in gj])
        R = np.mean(r ** -6.0) ** (-1.0 / 6.0)
        if R > up:
            edist += kup * (R * R - up * up) ** 2
        elif R < lo:
            edist += klo * (R * R - lo * lo) ** 2
    edihe = 0.0
    for q, lo, up, klo, kup in zip(*rd["dihe"]):
        phi = _dihedral(x, q)
        if lo <= phi <= up:
            continue
        to_up, to_lo = (phi - up) % (2 * np.pi), (lo - phi) % (2 * np.pi)
        edihe += kup * to_up ** 2 if to_up < to_lo else klo * to_lo ** 2
    ecap = 0.0
    cap = rd.get("cap")
    if cap is not None:
        m = np.asarray(top["mass"], float)
        for f, l in cap["groups"]:
            c = (m[f:l + 1, None] * x[f:l + 1]).sum(0) / m[f:l + 1].sum() - cap["center"]
            ecap += 0.5 * cap["k"] * max(np.linalg.norm(c) - cap["radius"], 0.0) ** 2
        for a in cap["atoms"]:
            ecap += 0.5 * cap["atom_k"] * max(np.linalg.norm(x[a] - cap["center"]) - cap["atom_radius"], 0.0) ** 2
    return np.array([epos, edist, edihe, ecap])


@pytest.mark.parametrize("name,bnd", [("poly", abi.JP_BOUND_PBC), ("drop", NONE)])
def test_energies_match_closed_forms(request, name, bnd):
    top = request.getfixturevalue(name)
    e, _ = oracle.Oracle(top, method=CANO, bounda=bnd).energy_grad()
    want = _numpy_energies(top, bnd == abi.JP_BOUND_PBC)
    np.testing.assert_allclose(e[SLOTS], want, rtol=1e-11, atol=1e-12)
    assert (want[:3] > 1.0).all()
    if name == "drop":
        assert want[3] > 1.0
    e0, _ = oracle.Oracle(_plain(top), method=CANO, bounda=bnd).energy_grad()
    np.testing.assert_allclose(e[0] - e0[0], want.sum(), rtol=1e-10)


@pytest.mark.parametrize("name,bnd", [("poly", abi.JP_BOUND_PBC), ("drop", NONE)])
def test_gradient_is_the_derivative(request, name, bnd):
    top = request.getfixturevalue(name)
    x0 = np.asarray(top["cord"], float)
    kw = dict(method=CANO, bounda=bnd)
    o = oracle.Oracle(top, **kw)
    o0 = oracle.Oracle(_plain(top), **kw)
    g = o.energy_grad()[1] - o0.energy_grad()[1]
    rd = top["restraints"]
    atoms = set(int(a) for a in rd["pos"][0])
    for gi, gj in zip(rd["dist"][0], rd["dist"][1]):
        atoms.update(int(a) for a in gi + gj)
    atoms.update(int(a) for a in np.ravel(rd["dihe"][0]))
    if "cap" in rd:
        atoms.update(int(a) for a in rd["cap"]["atoms"][:10])
        atoms.update(int(f) + k for f, _ in rd["cap"]["groups"][-20:] for k in range(3))
    h = 1e-5

    def eres(x):
        return o.energy_grad(x)[0][SLOTS].sum()

    for a in sorted(atoms):
        for k in range(3):
            xp, xm = x0.copy(), x0.copy()
            xp[a, k] += h
            xm[a, k] -= h
            fd = (eres(xp) - eres(xm)) / (2 * h)
            assert abs(fd - g[a, k]) < 1e-5 * max(1.0, abs(g[a, k])), (a, k, fd, g[a, k])


def test_position_reference_under_minimum_image(poly):
    moved = dict(poly)
    atoms, k, ref = poly["restraints"]["pos"]
    ref2 = ref.copy()
    ref2[0] += np.asarray(poly["box"]) * np.array([1, -1, 2])
    moved["restraints"] = dict(poly["restraints"], pos=(atoms, k, ref2))
    e1 = oracle.Oracle(poly, method=CANO).energy_grad()[0]
    e2 = oracle.Oracle(moved, method=CANO).energy_grad()[0]
    np.testing.assert_allclose(e2[abi.JP_E_POSRES], e1[abi.JP_E_POSRES], rtol=1e-12)


def test_dihedral_walls_across_two_pi():
    """phi near 350 deg with the window [40, 80] deg: the lower wall, 50 deg away across
    2 pi, is nearer than the upper one (270 deg)."""
    top = dict(systems.solvated_polymer(8, 300, seed=3))
    x = np.asarray(top["cord"], float)
    heavy = np.flatnonzero(np.isin(np.asarray(top["atype"]), (systems.T_C, systems.T_N, systems.T_O)))
    q = heavy[:4]
    phi = _dihedral(x, q)
    lo, up = (phi + np.radians(50.0)) % (2 * np.pi), (phi + np.radians(90.0)) % (2 * np.pi)
    if up < lo:   # keep 0 <= lo <= up < 2 pi by moving phi's window the other way
        lo, up = (phi - np.radians(90.0)) % (2 * np.pi), (phi - np.radians(50.0)) % (2 * np.pi)
    rd = dict(dihe=(np.array([q], np.int32), np.array([lo]), np.array([up]), np.array([3.0]),
                    np.array([7.0])))
    e = oracle.Oracle(dict(top, restraints=rd), method=CANO).energy_grad()[0]
    to_up, to_lo = (phi - up) % (2 * np.pi), (lo - phi) % (2 * np.pi)
    want = 7.0 * to_up ** 2 if to_up < to_lo else 3.0 * to_lo ** 2
    np.testing.assert_allclose(e[abi.JP_E_DIHERES], want, rtol=1e-12)
    np.testing.assert_allclose(min(to_up, to_lo), np.radians(50.0), rtol=1e-9)


def test_alsd_restraints_are_class_bb_and_unscaled(poly):
    top = dict(poly)
    cl = np.zeros(top["natom"], np.int32)
    cl[:40] = 1
    for g, na in zip(top["shake_atoms"], top["shake_n"]):
        if cl[g[:na]].any():
            cl[g[:na]] = 1
    top["cluster"] = cl
    kw = dict(method=CANO, alsd=abi.JP_ALSD_LMD, lambda0=0.7)
    o1, o0 = oracle.Oracle(top, **kw), oracle.Oracle(_plain(top), **kw)
    e1, g1 = o1.energy_grad()
    e0, g0 = o0.energy_grad()
    ec1, ec0 = o1.get_lambda()[1], o0.get_lambda()[1]
    eres = e1[SLOTS].sum()
    np.testing.assert_allclose(ec1 - ec0, [0.0, 0.0, eres], atol=1e-9)
    p1 = oracle.Oracle(poly, method=CANO).energy_grad()[1]
    p0 = oracle.Oracle(_plain(poly), method=CANO).energy_grad()[1]
    np.testing.assert_allclose(g1 - g0, p1 - p0, rtol=0, atol=1e-10)


def _shaped(drop, shape):
    """The droplet's CAP as a box or an ellipsoid around the same centre."""
    rd = dict(drop["restraints"])
    cap = dict(rd["cap"], shape=shape)
    x = np.asarray(drop["cord"], float)
    h = np.abs(x - cap["center"]).max(0)
    cap["wall"] = np.ravel([(-0.8 * v, 0.8 * v) for v in h])                 # relative to the centre
    cap["atom_wall"] = np.ravel([(c - 0.8 * v + 3.0, c + 0.8 * v - 3.0)      # absolute
                                 for c, v in zip(cap["center"], h)])
    cap["ellipse"] = 1.0 / (0.8 * h) ** 2
    cap["atom_ellipse"] = 1.0 / (0.8 * h - 3.0) ** 2
    rd["cap"] = cap
    return dict(drop, restraints=rd)


def _numpy_cap(top):
    """Energy and the gradient dnecap.f90 writes for the box (capshp 2) and ellipsoid
    (capshp 3) shapes."""
    x = np.asarray(top["cord"], float)
    m = np.asarray(top["mass"], float)
    cap = top["restraints"]["cap"]
    e, g = 0.0, np.zeros_like(x)

    def term(T, Tb, k, wall, ell):
        if cap["shape"] == abi.JP_CAP_BOX:
            lo, hi = np.asarray(wall)[0::2], np.asarray(wall)[1::2]
            over = np.where(Tb < lo, Tb - lo, np.where(Tb > hi, Tb - hi, 0.0))
            return 0.5 * k * (over ** 2).sum(), k * over
        s = (T * T * ell).sum()
        if s <= 1.0:
            return 0.0, np.zeros(3)
        rt = 1.0 - np.sqrt(1.0 / s)
        return 0.5 * k * (np.linalg.norm(T) * rt) ** 2, T * rt * k

    for f, l in cap["groups"]:
        C = (m[f:l + 1, None] * x[f:l + 1]).sum(0) / m[f:l + 1].sum() - cap["center"]
        de, dg = term(C, C, cap["k"], cap["wall"], cap["ellipse"])
        e += de
        g[f:l + 1] += dg * (m[f:l + 1, None] / m[f:l + 1].sum())
    for a in cap["atoms"]:
        de, dg = term(x[a] - cap["center"], x[a], cap["atom_k"], cap["atom_wall"], cap["atom_ellipse"])
        e += de
        g[a] += dg
    return e, g


@pytest.mark.parametrize("shape", [abi.JP_CAP_BOX, abi.JP_CAP_ELLIPSOID])
def test_cap_shapes_closed_form(drop, shape):
    top = _shaped(drop, shape)
    rd = top["restraints"]
    only = dict(top, restraints=dict(cap=rd["cap"]))
    kw = dict(method=CANO, bounda=NONE)
    e1, g1 = oracle.Oracle(only, **kw).energy_grad()
    e0, g0 = oracle.Oracle(_plain(top), **kw).energy_grad()
    ew, gw = _numpy_cap(only)
    assert ew > 1.0
    np.testing.assert_allclose(e1[abi.JP_E_CAP], ew, rtol=1e-11)
    np.testing.assert_allclose(g1 - g0, gw, rtol=0, atol=1e-10)


def test_box_cap_gradient_is_the_derivative(drop):
    top = _shaped(drop, abi.JP_CAP_BOX)
    only = dict(top, restraints=dict(cap=top["restraints"]["cap"]))
    o = oracle.Oracle(only, method=CANO, bounda=NONE)
    o0 = oracle.Oracle(_plain(top), method=CANO, bounda=NONE)
    g = o.energy_grad()[1] - o0.energy_grad()[1]
    x0 = np.asarray(top["cord"], float)
    moved = np.flatnonzero(np.abs(g).sum(1) > 1e-6)[:30]
    assert len(moved) > 5
    h = 1e-6
    for a in moved:
        for k in range(3):
            xp, xm = x0.copy(), x0.copy()
            xp[a, k] += h
            xm[a, k] -= h
            fd = (o.energy_grad(xp)[0][abi.JP_E_CAP] - o.energy_grad(xm)[0][abi.JP_E_CAP]) / (2 * h)
            assert abs(fd - g[a, k]) < 1e-5 * max(1.0, abs(g[a, k]))


def test_biquadratic_cap(drop):
    """CAP function 2 (dnecap.f90:253-281): 1/4 k R^2 ((d^2 - R^2) / R^2)^2 outside the sphere,
    for group centres and atoms; its gradient is the derivative."""
    cap = dict(drop["restraints"]["cap"], function=abi.JP_CAP_BIQUADRATIC)
    top = dict(drop, restraints=dict(cap=cap))
    kw = dict(method=CANO, bounda=NONE)
    o = oracle.Oracle(top, **kw)
    e1, g1 = o.energy_grad()
    g0 = oracle.Oracle(_plain(top), **kw).energy_grad()[1]
    x = np.asarray(top["cord"], float)
    m = np.asarray(top["mass"], float)
    want = 0.0
    for f, l in cap["groups"]:
        c = (m[f:l + 1, None] * x[f:l + 1]).sum(0) / m[f:l + 1].sum() - cap["center"]
        s = max(((c * c).sum() - cap["radius"] ** 2) / cap["radius"] ** 2, 0.0)
        want += 0.25 * cap["k"] * cap["radius"] ** 2 * s * s
    for a in cap["atoms"]:
        c = x[a] - cap["center"]
        s = max(((c * c).sum() - cap["atom_radius"] ** 2) / cap["atom_radius"] ** 2, 0.0)
        want += 0.25 * cap["atom_k"] * cap["atom_radius"] ** 2 * s * s
    assert want > 1.0
    np.testing.assert_allclose(e1[abi.JP_E_CAP], want, rtol=1e-11)
    g = g1 - g0
    moved = np.flatnonzero(np.abs(g).sum(1) > 1e-6)[:20]
    h = 1e-6
    for a in moved:
        for k in range(3):
            xp, xm = x.copy(), x.copy()
            xp[a, k] += h
            xm[a, k] -= h
            fd = (o.energy_grad(xp)[0][abi.JP_E_CAP] - o.energy_grad(xm)[0][abi.JP_E_CAP]) / (2 * h)
            assert abs(fd - g[a, k]) < 1e-5 * max(1.0, abs(g[a, k]))
