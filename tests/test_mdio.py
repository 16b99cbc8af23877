"""md_run's output records (monmd.f90 outtco / outtve / outten) and PBcord wrapping, as
written by j_presto_b200.mdio (no GPU)."""
import struct

import numpy as np
import pytest

from j_presto_b200 import mdio


@pytest.mark.parametrize("prec,size", [(mdio.REAL4, 4), (mdio.REAL8, 8)])
def test_trajectory_records(tmp_path, prec, size):
    rng = np.random.default_rng(3)
    frames = rng.normal(size=(3, 5, 3))
    p = tmp_path / "t.cod"
    with mdio.TrajectoryWriter(p, prec, atoms=[0, 2, 4]) as w:
        for k, x in enumerate(frames):
            w.write(x, step=10 * k, time=0.02 * k, etot=-1.5, temp=300.0, lam=0.5, n15v=7, n15h=3,
                    epot_cls=(1.0, 2.0, 3.0))
    recs = mdio.read_records(p)
    assert len(recs) == 6
    # header: idloop, 7 reals, 2 integers, rmsd, 3 class energies
    assert len(recs[0]) == 4 + 7 * size + 8 + size + 3 * size
    assert len(recs[1]) == 3 * 3 * size
    heads, got = mdio.read_trajectory(p, prec)
    assert heads[2][0] == 20 and heads[1][8:10] == (7, 3)
    np.testing.assert_allclose(got, frames[:, [0, 2, 4]], rtol=1e-6 if size == 4 else 0)
    raw = p.read_bytes()
    assert struct.unpack("<i", raw[:4])[0] == len(recs[0])   # leading byte count


def test_energy_and_velocity_records(tmp_path):
    p = tmp_path / "e.ene"
    e = np.arange(15.0)
    with mdio.EnergyWriter(p, mdio.REAL8) as w:
        w.write(e, step=1, time=0.002, etot=3.0, ekin=1.0, temp=300.0, rmsf=0.5, n15v=9, n15h=1)
    recs = mdio.read_records(p)
    assert [len(r) for r in recs] == [4 + 16, 3 * 8 + 15 * 8 + 8 + 8 + 8]
    vals = struct.unpack("<ddd" + "d" * 15 + "diid", recs[1])
    assert vals[3:18] == tuple(e) and vals[19:21] == (9, 1)
    pv = tmp_path / "v.vel"
    with mdio.VelocityWriter(pv, mdio.REAL4) as w:
        w.write(np.ones((4, 3)), step=2)
    assert [len(r) for r in mdio.read_records(pv)] == [4 + 7 * 4 + 8 + 4, 4 * 3 * 4]


def test_wrap_chains():
    """PBcord: a chain whose centre left the cell comes back by whole box lengths; its
    shape is kept."""
    box = np.array([10.0, 10.0, 10.0])
    x = np.array([[11.0, 1.0, 1.0], [12.0, 1.0, 1.0], [-3.0, 5.0, 5.0]])
    out = mdio.wrap_chains(x, [(0, 1), (2, 2)], box, wall_lo=np.zeros(3))
    np.testing.assert_allclose(out, [[1.0, 1.0, 1.0], [2.0, 1.0, 1.0], [7.0, 5.0, 5.0]])
    np.testing.assert_allclose(out[1] - out[0], x[1] - x[0])


def test_restart_round_trip(tmp_path):
    """outrst.f90 records: title, natom nvar, step time energies, coordinates, velocities,
    lambda; read back as inprst.f90 reads them."""
    rng = np.random.default_rng(5)
    x, v = rng.normal(size=(6, 3)), rng.normal(size=(6, 3))
    p = tmp_path / "restart.dat"
    mdio.write_restart(p, x, v, step=500, time=1.0, etot=-3.5, ekin=2.0, epot=-5.5, lam=0.8, lam_v=0.01)
    recs = mdio.read_records(p)
    assert [len(r) for r in recs] == [80, 8, 4 + 32, 6 * 24, 6 * 24, 16]
    r = mdio.read_restart(p)
    assert (r["step"], r["time"], r["epot"], r["lam"], r["lam_v"]) == (500, 1.0, -5.5, 0.8, 0.01)
    np.testing.assert_array_equal(r["cord"], x)
    np.testing.assert_array_equal(r["vel"], v)
    assert r["title"].startswith("     VERLET")
