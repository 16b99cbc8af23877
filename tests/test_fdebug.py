"""md_run's FDEBUG force file (1stp_force.bin, verlethe.f90:325-387) written and read by
the oracle's tools, and the oracle's first-step force against its definition (no GPU).
"""
import struct

import numpy as np
import pytest

import oracle
from oracle import fdebug
from j_presto_b200 import abi, systems


@pytest.fixture(scope="module")
def poly():
    top = dict(systems.solvated_polymer(8, 300, seed=3))
    e0 = oracle.Oracle(top, method=abi.JP_METHOD_MICR).energy_grad()[0][0]
    top["ge"] = dict(coef=np.array([[1.2, -0.3]]), low=np.array([0.0]), high=np.array([1.0 + 1e-12]),
                     alphalw=1.2, alphaup=0.9, celw=e0 - 2000.0, ceup=e0 + 2000.0, tempce=300.0)
    return top


def test_record_layout_and_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    e, g = rng.normal(size=15), rng.normal(size=(7, 3))
    p = tmp_path / "1stp_force.bin"
    fdebug.write(p, e, 0.25, g)
    raw = p.read_bytes()
    # three records framed by 4-byte counts: 120, 8 and 24 * natom bytes
    assert len(raw) == (4 + 120 + 4) + (4 + 8 + 4) + (4 + 168 + 4)
    assert struct.unpack("<i", raw[:4])[0] == 120 and struct.unpack("<i", raw[124:128])[0] == 120
    assert struct.unpack("<d", raw[132:140])[0] == 0.25
    e2, lf, g2 = fdebug.read(p)
    np.testing.assert_array_equal(e2, e)
    np.testing.assert_array_equal(g2, g)
    assert lf == 0.25
    # grad(1:3, i) order: atom 0's three components first
    np.testing.assert_array_equal(np.frombuffer(raw[148:172], np.float64), g[0])


def test_compare_follows_the_check(tmp_path):
    rng = np.random.default_rng(2)
    e, g = rng.normal(size=15), rng.normal(size=(5, 3))
    ref = (e, 0.0, g)
    same = fdebug.compare(ref, e, 0.0, g)
    assert same["passed"] and same["max_force_error"] == 0.0
    g2 = g.copy()
    g2[3, 1] += 5e-9
    e2 = e.copy()
    e2[0] += 1.0          # eneval(1), the total, is not part of the energy check
    out = fdebug.compare(ref, e2, 0.0, g2)
    assert not out["passed"] and out["atoms_over"].tolist() == [3]
    np.testing.assert_allclose(out["max_force_error"], 5e-9, rtol=1e-6)
    assert out["max_energy_error"] == 0.0


def test_first_force_is_the_scaled_gradient(poly, tmp_path):
    """CANO: the plain gradient; GE: times the McMD factor of the total energy
    (verlethe.f90:196-238); the file written from it reads back unchanged."""
    o = oracle.Oracle(poly, method=abi.JP_METHOD_CANO)
    e, lf, g = o.first_force()
    e0, g0 = o.energy_grad()
    np.testing.assert_allclose(g, g0, rtol=1e-12, atol=1e-12)   # OpenMP sums: order varies
    assert lf == 0.0
    og = oracle.Oracle(poly, method=abi.JP_METHOD_GE)
    e, lf, g = og.first_force()
    np.testing.assert_allclose(g, g0 * og.mcmd_scale(e[0]), rtol=1e-12, atol=1e-12)
    p = tmp_path / "1stp_force.bin"
    fdebug.write(p, e, lf, g)
    assert fdebug.compare(fdebug.read(p), e, lf, g)["passed"]
