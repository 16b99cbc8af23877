"""The oracle's centre-of-mass stop (remotv), Berendsen scaling (METHOD= CONS, scalet) and
their degrees of freedom, against analytic answers (no GPU).

remotv must remove exactly a rigid translation V and rotation W x (x - centre) added to
velocities that carry no momentum and no angular momentum; scalet multiplies the new
velocities by sqrt(1 + dt/taut (T0/T - 1)), at most 2, T the temperature of v(t-dt/2).
"""
import numpy as np
import pytest

import oracle
from j_presto_b200 import abi, systems


@pytest.fixture(scope="module")
def poly():
    return dict(systems.solvated_polymer(8, 300, seed=3))


def _first_molecule(top):
    mol = np.asarray(top["molecule"])
    return int(np.argmax(mol != mol[0]))


def _internal_velocities(x, m, rng):
    """Random velocities with zero momentum and zero angular momentum about the centre."""
    v = rng.normal(size=x.shape)
    c = (m[:, None] * x).sum(0) / m.sum()
    d = x - c
    v -= (m[:, None] * v).sum(0) / m.sum()
    inertia = np.einsum("i,ij->", m, d * d) * np.eye(3) - np.einsum("i,ij,ik->jk", m, d, d)
    w = np.linalg.solve(inertia, (m[:, None] * np.cross(d, v)).sum(0))
    return v - np.cross(w, d)


@pytest.mark.parametrize("mode", [abi.JP_STOP_TRANS, abi.JP_STOP_ROT, abi.JP_STOP_BOTH])
def test_remotv_removes_rigid_motion(poly, mode):
    rng = np.random.default_rng(5)
    n0 = _first_molecule(poly)
    o = oracle.Oracle(poly, method=abi.JP_METHOD_MICR, stop_center=mode)
    x = np.asarray(poly["cord"], np.float64)
    m = np.asarray(poly["mass"], np.float64)
    vint = _internal_velocities(x[:n0], m[:n0], rng)
    c = (m[:n0, None] * x[:n0]).sum(0) / m[:n0].sum()
    V = np.array([0.003, -0.002, 0.001])
    W = np.array([1e-4, 3e-4, -2e-4])
    vel = rng.normal(size=x.shape) * 0.01          # atoms past the molecule stay as they are
    vel[:n0] = vint + V + np.cross(W, x[:n0] - c)
    ier, out = o.remotv(x, vel)
    assert ier == 0
    want = vel.copy()
    if mode in (abi.JP_STOP_TRANS, abi.JP_STOP_BOTH):
        want[:n0] -= V
    if mode in (abi.JP_STOP_ROT, abi.JP_STOP_BOTH):
        want[:n0] -= np.cross(W, x[:n0] - c)
    np.testing.assert_allclose(out, want, rtol=0, atol=1e-13)
    np.testing.assert_array_equal(out[n0:], vel[n0:])


def test_stop_natom_selects_the_atoms(poly):
    x = np.asarray(poly["cord"], np.float64)
    m = np.asarray(poly["mass"], np.float64)
    vel = np.random.default_rng(2).normal(size=x.shape) * 0.01
    o = oracle.Oracle(poly, method=abi.JP_METHOD_MICR, stop_center=abi.JP_STOP_TRANS, stop_natom=10)
    ier, out = o.remotv(x, vel)
    assert ier == 0
    np.testing.assert_allclose((m[:10, None] * out[:10]).sum(0), 0.0, atol=1e-15)
    np.testing.assert_array_equal(out[10:], vel[10:])


def test_stop_degrees_of_freedom(poly):
    base = oracle.Oracle(poly, method=abi.JP_METHOD_CANO, tempco=2)
    nf0 = base.nfrmol()
    for mode, drop in ((abi.JP_STOP_TRANS, 3), (abi.JP_STOP_ROT, 3), (abi.JP_STOP_BOTH, 6)):
        o = oracle.Oracle(poly, method=abi.JP_METHOD_CANO, tempco=2, stop_center=mode)
        assert o.dof == base.dof - drop
        nf = o.nfrmol()
        assert nf[0] == nf0[0] - drop                # the first molecule is sub-system 0
        np.testing.assert_array_equal(nf[1:], nf0[1:])


def test_stop_dof_split_over_cluster_subsystems(poly):
    """A first molecule split into its cluster and non-cluster sub-systems (ALSD) loses the
    degrees of freedom in proportion to theirs (md.f90:197-211)."""
    top = dict(poly)
    cl = np.zeros(top["natom"], np.int32)
    cl[:12] = 1
    for g, na in zip(top["shake_atoms"], top["shake_n"]):
        if cl[g[:na]].any():
            cl[g[:na]] = 1
    top["cluster"] = cl
    kw = dict(method=abi.JP_METHOD_CANO, tempco=2, alsd=abi.JP_ALSD_LMD, lambda0=0.9)
    nf0 = oracle.Oracle(top, **kw).nfrmol()
    nf = oracle.Oracle(top, stop_center=abi.JP_STOP_BOTH, **kw).nfrmol()
    ratio = nf0[:2] / nf0[:2].sum()
    np.testing.assert_allclose(nf[:2], nf0[:2] - 6.0 * ratio, rtol=1e-15)
    np.testing.assert_array_equal(nf[2:], nf0[2:])


def _one_step(top, vel, method, **kw):
    o = oracle.Oracle(top, method=method, shake_method=abi.JP_SHAKE_NONE, **kw)
    o.set_state(top["cord"], vel)
    ier, _, _ = o.run(1)
    assert ier == 0
    return o, o.get_state()[0]


@pytest.mark.parametrize("tscale", [1.0, 1e-3, 0.0])
def test_scalet_factor(poly, tscale):
    """CONS step = MICR step with the new velocity scaled by the Berendsen factor (capped at
    2 for a cold start; no scaling at zero temperature)."""
    x0 = np.asarray(poly["cord"], np.float64)
    vel = np.asarray(poly["vel"], np.float64) * tscale
    om, xm = _one_step(poly, vel, abi.JP_METHOD_MICR)
    oc, xc = _one_step(poly, vel, abi.JP_METHOD_CONS, taut=40.0, temp=300.0)
    t = oc.temperature(vel)
    lam = 1.0 if t <= 0.0 else min(2.0, np.sqrt(1.0 + 2.0 / 40.0 * (300.0 / t - 1.0)))
    if tscale == 1e-3:
        assert lam == 2.0
    np.testing.assert_allclose(xc - x0, lam * (xm - x0), rtol=1e-12, atol=1e-13)   # ulp of x


def _clustered(top, n=40):
    top = dict(top)
    cl = np.zeros(top["natom"], np.int32)
    cl[:n] = 1
    for g, na in zip(top["shake_atoms"], top["shake_n"]):
        if cl[g[:na]].any():
            cl[g[:na]] = 1
    top["cluster"] = cl
    return top


def test_scalet_peptide_exemption(poly):
    """SCALET's peptide-bond exemption (scale_tor 2/3, incel.f90:846-866): a marked torsion
    stays in class BB.  All marked = the torsion bit off; none marked = the bit on; a subset
    moves only those torsions' energy into BB and leaves the total alone."""
    top = _clustered(poly)
    kw = dict(method=abi.JP_METHOD_CANO, alsd=abi.JP_ALSD_LMD, lambda0=0.7)
    nt = len(top["tors"])

    def run(scale, mark):
        t = dict(top, tors_unscaled=mark) if mark is not None else top
        o = oracle.Oracle(t, scale_terms=scale, **kw)
        e, g = o.energy_grad()
        return e, g, o.get_lambda()[1]

    on = abi.JP_SCALE_TORS
    e_off, g_off, c_off = run(0, None)
    e_all, g_all, c_all = run(on, np.ones(nt, np.int32))
    np.testing.assert_allclose(g_all, g_off, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(c_all, c_off, rtol=1e-12, atol=1e-10)
    e_on, g_on, c_on = run(on, None)
    e_none, g_none, c_none = run(on, np.zeros(nt, np.int32))
    np.testing.assert_allclose(g_none, g_on, rtol=1e-12, atol=1e-12)
    assert np.abs(c_on - c_off).max() > 1.0          # the bit matters for this cluster
    sub = (np.arange(nt) % 2).astype(np.int32)
    e_sub, g_sub, c_sub = run(on, sub)
    np.testing.assert_allclose(e_sub, e_on, rtol=1e-12, atol=1e-10)
    np.testing.assert_allclose(c_sub.sum(), c_on.sum(), rtol=1e-12)
    assert c_sub[2] > c_on[2] or np.allclose(c_sub, c_on)
