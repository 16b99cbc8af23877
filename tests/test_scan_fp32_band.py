"""The tile scan's FP32 distance test, restated in numpy float32, against its documented
error bound: every squared distance it computes is within a quarter of the uncertainty band
of the exact FP64 value, so a pair decided in FP32 (outside the band) is decided as FP64
decides it, and the list equals the FP64 list (jp_cells.cu tile_row_f32 and the band of
k_tile_scan_chunks).

The FP32 path: i atoms relative to their block's reference, (float)(x - ref_i); j atoms as
their block-local FP32 position plus block j's reference moved into the i block's frame,
(float)(image - (ref_i - ref_j)); d^2 with fused multiply-adds.
"""
import numpy as np
import pytest

F = np.float32


def fma32(a, b, c):
    # a*b is exact in FP64 for FP32 inputs; one rounding to FP32 as the fused operation
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(F)


@pytest.mark.parametrize("seed", range(4))
def test_fp32_distance_within_quarter_band(seed):
    rng = np.random.default_rng(seed)
    rlim, hm = 13.5, 4.0
    box = rng.uniform(60.0, 120.0, 3)
    mb = rlim + 3.0 * hm
    band = 4.0 * 5.9604645e-8 * (17.33 * rlim * mb + 3.0 * rlim * rlim)
    worst = 0.0
    for _ in range(300):
        ref_i = rng.uniform(0.0, box)
        ref_j = ref_i + rng.normal(0.0, 1.0, 3) * (rlim / 2.0)
        ref_j -= box * np.floor(ref_j / box)
        xi = ref_i + rng.uniform(-hm, hm, (32, 3))
        xj = ref_j + rng.uniform(-hm, hm, (32, 3))
        # the scan's inputs
        xf_i = (xi - ref_i).astype(F)
        pos_j = (xj - ref_j).astype(F)
        d = ref_i - ref_j
        cj = (box * np.rint(d / box) - d).astype(F)
        r = pos_j + cj                                   # FP32 add
        dx = xf_i[:, None, :] - r[None, :, :]            # FP32 subtract
        d2f = fma32(dx[..., 0], dx[..., 0], fma32(dx[..., 1], dx[..., 1], dx[..., 2] * dx[..., 2]))
        # exact, in FP64, with the same image
        img = box * np.rint(d / box)
        dd = xi[:, None, :] - (xj[None, :, :] + img)
        d2 = (dd ** 2).sum(-1)
        near = np.abs(d2 - rlim * rlim) < 50.0           # pairs that matter: near the list radius
        if near.any():
            worst = max(worst, float(np.abs(d2f[near].astype(np.float64) - d2[near]).max()))
    assert worst < band / 4.0, (worst, band)
