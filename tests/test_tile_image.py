"""The pair kernels' per-tile image rule, checked on random geometry: where box/2 is at least
rc + 2 h_max + 2 A on every axis, every pair within the cut-off takes the nearest image of
its two blocks' references, so the tile's single shift is exact for it (jp_pair.cu applies
the per-pair minimum image only below that bound).

Blocks: references anywhere in the box, atoms within h of their reference per axis at the
list build, then each atom moved by up to 1 A per axis (2 A between two atoms, the margin
the rule holds for the atoms' motion between builds).
"""
import numpy as np
import pytest


def nearest(d, box):
    return d - box * np.rint(d / box)


@pytest.mark.parametrize("seed", range(4))
def test_tile_image_is_every_listed_pairs_image(seed):
    rng = np.random.default_rng(seed)
    rc, h = 12.0, 4.0
    box = np.full(3, 2.0 * (rc + 2.0 * h + 2.0)) * rng.uniform(1.0, 1.3, 3)
    n_checked = 0
    for _ in range(400):
        ri, rj = rng.uniform(0.0, box, (2, 3))
        xi = ri + rng.uniform(-h, h, (32, 3)) + rng.uniform(-1.0, 1.0, (32, 3))
        xj = rj + rng.uniform(-h, h, (32, 3)) + rng.uniform(-1.0, 1.0, (32, 3))
        shift = nearest(ri - rj, box) - (ri - rj)       # the tile's image (multiples of box)
        d_tile = (xi[:, None, :] - xj[None, :, :]) + shift
        d_min = nearest(xi[:, None, :] - xj[None, :, :], box)
        r_min = np.sqrt((d_min ** 2).sum(-1))
        within = r_min <= rc
        n_checked += int(within.sum())
        np.testing.assert_allclose(d_tile[within], d_min[within], atol=1e-9)
    assert n_checked > 100


def test_rule_is_needed_below_the_bound():
    """with box/2 well below rc + 2 h, some pair within rc has another image than its tile's"""
    rng = np.random.default_rng(5)
    rc, h = 12.0, 4.0
    box = np.full(3, 2.0 * rc)
    found = False
    for _ in range(200):
        ri, rj = rng.uniform(0.0, box, (2, 3))
        xi = ri + rng.uniform(-h, h, (32, 3))
        xj = rj + rng.uniform(-h, h, (32, 3))
        shift = nearest(ri - rj, box) - (ri - rj)
        d_tile = (xi[:, None, :] - xj[None, :, :]) + shift
        d_min = nearest(xi[:, None, :] - xj[None, :, :], box)
        within = np.sqrt((d_min ** 2).sum(-1)) <= rc
        if np.abs(d_tile[within] - d_min[within]).max(initial=0.0) > 1e-6:
            found = True
            break
    assert found
