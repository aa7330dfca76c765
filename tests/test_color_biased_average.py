"""The integer averages of the fused RGB -> YUV / scale kernel (k_fused_rgb_yuv_scale8,
mivisionx_b200/csrc/geometry.cu) run on words 0x4B000000 + v (the bits of the float 2^23 + v
that one round-toward-zero add leaves) instead of on v: the U/V block average
((u0 + u2 + 1) >> 1 + (u1 + u3 + 1) >> 1 + 1) >> 1, the bilinear half-size
((y0 + y1 + 1) >> 1 + (y2 + y3 + 1) >> 1 + 1) >> 1 and the area half-size
(y0 + y1 + y2 + y3 + 2) >> 2, all in uint32 arithmetic (sums wrap modulo 2^32).  The low byte of
each biased result must equal the plain integer result for every input in [0, 255]."""
import numpy as np

K = np.uint32(0x4B000000)


def _avg2(a, b):
    return (a + b + np.uint32(1)) >> np.uint32(1)


def test_biased_block_averages_match_plain_integers():
    rng = np.random.default_rng(7)
    v = np.concatenate([rng.integers(0, 256, (200000, 4)), np.array([[0, 0, 0, 0], [255, 255, 255, 255],
                                                                    [255, 0, 255, 0], [0, 255, 0, 255]])]).astype(np.uint32)
    b = v + K
    with np.errstate(over="ignore"):
        # U / V (rgb_block) and bilinear half-size: two pair averages, then their average
        plain = _avg2(_avg2(v[:, 0], v[:, 2]), _avg2(v[:, 1], v[:, 3]))
        biased = _avg2(_avg2(b[:, 0], b[:, 2]), _avg2(b[:, 1], b[:, 3]))
        assert np.array_equal(biased & np.uint32(0xFF), plain)
        assert np.array_equal(biased, plain + K)
        # area half-size: four terms, the bias 4 * K wraps modulo 2^32 to a multiple of 4
        plain4 = (v.sum(axis=1, dtype=np.uint32) + np.uint32(2)) >> np.uint32(2)
        biased4 = (b[:, 0] + b[:, 1] + b[:, 2] + b[:, 3] + np.uint32(2)) >> np.uint32(2)
        assert np.array_equal(biased4 & np.uint32(0xFF), plain4)
    assert int(4 * int(K)) % (1 << 32) % 4 == 0
