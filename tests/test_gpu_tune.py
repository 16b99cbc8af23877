"""The block-shape tuner of jp_create (the role of md_run's SIMD_check.f90 autotuning).

Every replica's list is built with each candidate column grid and the grid needing the
fewest pair records is kept.  Checked: the kept candidate is the minimum of the reported
counts; two contexts on the same input choose the same and report the same counts (the
choice is deterministic); a replica chooses alone as it does in a batch; with tuning off
the unit factor is kept; the forces do not depend on the block shape (FP64 path, RMS
relative 1e-12; the listed pair set is the same).
"""
import numpy as np
import pytest

from j_presto_b200 import abi, systems
from tests._util import rms_rel

pytestmark = pytest.mark.gpu

SCALES = [0.84, 0.92, 1.0, 1.09, 1.19]


@pytest.fixture(scope="module")
def eng_mod(engine_lib):
    from j_presto_b200 import engine
    return engine


@pytest.fixture(scope="module")
def tops():
    return [systems.solvated_polymer(20, 1500, seed=7), systems.config_c1_prime()]


def test_choice_is_the_fewest_tiles_and_deterministic(eng_mod, tops):
    shapes = []
    for _ in range(2):
        with eng_mod.Engine(tops[0], precision=abi.JP_PREC_MIXED, method=abi.JP_METHOD_CANO) as e:
            f, tiles = e.tile_shape()
            nt, nlisted, _ = e.list_stats()
        assert all(t > 0 for t in tiles)
        assert tiles[SCALES.index(f)] == min(tiles) == nt
        shapes.append((f, tiles, nlisted))
    assert shapes[0] == shapes[1]


def test_batch_chooses_as_alone(eng_mod, tops):
    alone = []
    for t in tops:
        with eng_mod.Engine(t, precision=abi.JP_PREC_MIXED, method=abi.JP_METHOD_MICR) as e:
            alone.append(e.tile_shape())
    with eng_mod.Engine(tops, precision=abi.JP_PREC_MIXED, method=abi.JP_METHOD_MICR) as e:
        for r in range(len(tops)):
            assert e.tile_shape(r) == alone[r]


def test_forces_do_not_depend_on_the_shape(eng_mod, tops):
    out = {}
    for tune in (0, 1):
        with eng_mod.Engine(tops[0], precision=abi.JP_PREC_FP64, method=abi.JP_METHOD_MICR,
                            tune_blocks=tune) as e:
            f, tiles = e.tile_shape()
            if not tune:
                assert f == 1.0 and all(t == -1 for t in tiles)
            out[tune] = (e.energy_grad(), e.pair_count(), e.list_stats()[1])
    (e0, g0), p0, l0 = out[0]
    (e1, g1), p1, l1 = out[1]
    assert p0 == p1 and l0 == l1
    assert rms_rel(g1, g0) < 1e-12
    # energies: each pair record's FP64 sum enters in 2^-32 fixed point, and other records
    # round differently (~1e-10 per tile)
    np.testing.assert_allclose(e1, e0, rtol=1e-9, atol=1e-6)
