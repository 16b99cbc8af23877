"""md_run's initial-velocity generator (ranun.f90, ranno.f90, setvel.f90, md.f90:1009-1040)
restated for the host (no GPU)."""
import numpy as np

import oracle
from j_presto_b200 import abi, setvel, systems


def test_ranun_sequence():
    """The 30-bit state advances as (a s + c) mod 2^30 (a = 32771, c = 123456781), carried in
    two 15-bit halves; each number is the new state over 2^30 in single precision."""
    x, s = setvel.ranun(5, 12345)
    seq, want = 12345, []
    for _ in range(5):
        seq = (32771 * seq + 123456781) % 2 ** 30
        want.append(np.float32(seq) * np.float32(2.0 ** -30))
    assert s == seq
    np.testing.assert_array_equal(x, np.array(want, np.float32))
    assert ((x > 0) & (x < 1)).all()


def test_ranno_moments_and_odd_counts():
    x, _ = setvel.ranno(20001, 777)
    assert x.dtype == np.float32
    assert abs(float(x.mean())) < 0.03 and abs(float(x.std()) - 1.0) < 0.03
    y, s1 = setvel.ranno(4, 5)
    z, s2 = setvel.ranno(5, 5)
    np.testing.assert_array_equal(y, z[:4])   # the pairs do not depend on the count
    assert s1 != s2                            # the odd count drew one extra pair


def test_initial_velocities_temperature_and_momentum():
    top = dict(systems.solvated_polymer(8, 300, seed=3))
    o = oracle.Oracle(top, method=abi.JP_METHOD_CANO, shake_method=abi.JP_SHAKE_NONE, stop_center=abi.JP_STOP_BOTH)
    v, seed = setvel.initial_velocities(top["mass"], top["cord"], 300.0, 1, o.dof)
    np.testing.assert_allclose(o.temperature(v), 300.0, rtol=1e-10)
    m = np.asarray(top["mass"])[:, None]
    x = np.asarray(top["cord"])
    c = (m * x).sum(0) / m.sum()
    assert np.abs((m * v).sum(0)).max() < 1e-12
    assert np.abs((m * np.cross(x - c, v)).sum(0)).max() < 1e-10
    v2, _ = setvel.initial_velocities(top["mass"], top["cord"], 300.0, 1, o.dof)
    np.testing.assert_array_equal(v, v2)
