"""Two FP32 facts the mixed pair kernel relies on (jp_pair.cu rint2 / rint1, jp_common.cuh
to_fix_f), checked in numpy float32:

* adding then subtracting 1.5 * 2^23 (each a separately rounded FP32 add) gives the nearest
  integer of v, ties to even, for |v| < 2^22 -- the minimum-image multiple on the FMA pipe;
* an FP32 force times 2^32 is exact in FP32, so rounding it to a 64-bit integer gives the
  same fixed-point value as doing the product in FP64.
"""
import numpy as np

F = np.float32


def test_magic_add_rounds_to_nearest_even():
    rng = np.random.default_rng(0)
    v = np.concatenate([
        rng.uniform(-8.0, 8.0, 200000),                     # the minimum-image range
        rng.uniform(-2.0 ** 22, 2.0 ** 22, 100000),
        np.arange(-64, 64) + 0.5,                           # exact ties
        np.nextafter(np.arange(-64, 64) + 0.5, 0.0),
        np.nextafter(np.arange(-64, 64) + 0.5, 100.0),
    ]).astype(F)
    m = F(12582912.0)
    got = (v + m) - m           # two FP32 adds, each rounded
    want = np.rint(v)           # ties to even
    assert np.array_equal(got, want)


def test_force_to_fixed_point_matches_fp64_product():
    rng = np.random.default_rng(1)
    f = np.concatenate([rng.normal(0.0, 1.0, 100000) * 10.0 ** rng.uniform(-6, 4, 100000),
                        [0.0, -0.0, 1e-30, -1e-30, 3.0e4]]).astype(F)
    s32 = (f * F(4294967296.0)).astype(F)                  # the FP32 product
    assert np.array_equal(s32.astype(np.float64), f.astype(np.float64) * 4294967296.0)   # exact
    via32 = np.rint(s32.astype(np.float64)).astype(np.int64)
    via64 = np.rint(f.astype(np.float64) * 4294967296.0).astype(np.int64)
    assert np.array_equal(via32, via64)
