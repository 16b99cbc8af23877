"""The bit layouts that carry a pair list from the tile scan to the pair kernel, restated in
Python and checked end to end on random tiles: every pair a tile mask lists is met exactly
once by the pair kernel's enumeration of the records built from it, and no other pair is.

Layouts (j_presto_b200/csrc/jp_cells.cu, jp_pair.cu):
* tile row of i atom ri (0-31 of the i block): bit k is j lane (ri + k) & 31;
* a half block h (rows 16 h .. 16 h + 15) lists, per tile, the j lanes some of its rows
  use (the occupancy word); its record entries are those lanes, tile after tile, 32 per
  record (the last record padded);
* record row r (i atom 16 h + r), built by k_ct_emit: bit p is slot p's j lane in its
  tile's row 16 h + r (one warp ballot per row), then each 16-bit half rotated right by r;
* the pair kernel: lane l of the half meets at step k (k < 16) entries a = (l + k) & 15 and
  b = 16 + a, with mask bits k and 16 + k of its row.
"""
import random

import pytest


def rotl(x, s):
    s &= 31
    return ((x << s) | (x >> (32 - s))) & 0xFFFFFFFF if s else x


def tile_rows(pairs):
    """pairs: set of (i, j) in one 32x32 tile -> the 32 stored (rotated) rows"""
    rows = [0] * 32
    for i, j in pairs:
        rows[i] |= 1 << ((j - i) & 31)
    return rows


def occupancy(rows, h):
    occ = 0
    for r in range(16 * h, 16 * h + 16):
        occ |= rotl(rows[r], r)   # unrotated: bit j = j lane j
    return occ


def records(tiles, h):
    """tiles: list of 32-row masks of one i block -> records of half h as lists of
    (entries: [(tile, j lane) or None] * 32, rows: [16 stored words])"""
    entries = []
    for t, rows in enumerate(tiles):
        occ = occupancy(rows, h)
        entries += [(t, j) for j in range(32) if (occ >> j) & 1]
    out = []
    for s0 in range(0, len(entries), 32):
        slots = entries[s0:s0 + 32] + [None] * max(0, s0 + 32 - len(entries))
        words = []
        for r in range(16):
            ri = 16 * h + r
            row = 0
            for p, e in enumerate(slots):   # the ballot: slot p's bit
                if e is not None:
                    t, jl = e
                    row |= ((tiles[t][ri] >> ((jl - ri) & 31)) & 1) << p
            lo, hi = row & 0xFFFF, row >> 16
            rl = ((lo >> r) | (lo << (16 - r))) & 0xFFFF
            rh = ((hi >> r) | (hi << (16 - r))) & 0xFFFF
            words.append(rl | (rh << 16))
        out.append((slots, words))
    return out


def kernel_pairs(recs, h):
    """the (i row, (tile, j lane)) pairs the pair kernel evaluates on the records"""
    met = []
    for slots, words in recs:
        for l in range(16):
            m = words[l]
            for k in range(16):
                a = (l + k) & 15
                for bit, e in ((k, a), (16 + k, 16 + a)):
                    if (m >> bit) & 1:
                        assert slots[e] is not None, "a mask bit on a padding slot"
                        met.append((16 * h + l, slots[e]))
    return met


@pytest.mark.parametrize("seed", range(6))
def test_records_list_every_tile_pair_once(seed):
    rng = random.Random(seed)
    ntile = rng.randint(1, 9)
    want = set()
    tiles = []
    for t in range(ntile):
        dens = rng.choice([0.02, 0.1, 0.4, 0.9])
        pairs = {(i, j) for i in range(32) for j in range(32) if rng.random() < dens}
        tiles.append(tile_rows(pairs))
        want |= {(i, (t, j)) for i, j in pairs}
    got = []
    for h in (0, 1):
        got += kernel_pairs(records(tiles, h), h)
    assert len(got) == len(set(got)), "a pair met twice"
    assert set(got) == want


def test_record_count_is_entries_over_32():
    rng = random.Random(7)
    tiles = [tile_rows({(i, j) for i in range(32) for j in range(32) if rng.random() < 0.3})
             for _ in range(5)]
    for h in (0, 1):
        n = sum(bin(occupancy(rows, h)).count("1") for rows in tiles)
        assert len(records(tiles, h)) == (n + 31) // 32
