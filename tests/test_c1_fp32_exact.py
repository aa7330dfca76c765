"""The exact-fp32 Sobel / threshold arithmetic of the TMA-staged configuration-1 kernel
(k_fused_c1_tma, mivisionx_b200/csrc/filters.cu), restated in numpy float32 step by step and
compared with the oracle chain (Gaussian3x3 -> SobelMagnitude -> ConvertDepth(SAT) ->
Threshold(BINARY)) for every threshold and shift on noise and on high-contrast frames.

The kernel's claim is that no step rounds: t = 6144 + G/128 is built by dropping the masked
16G lane into the mantissa of 6144, gx / gy are sums of differences of t, and
r = (n_min - 1/2)/16384 - gx^2 - gy^2 is exact, so r < 0 exactly when gx^2 + gy^2 >= n_min.
Each fused multiply-add is checked here to be exact (its float64 value is a float32)."""
import numpy as np
import pytest

import oracle_chains as OC

f32 = np.float32


def _fma(a, b, c):
    r64 = a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)
    r = r64.astype(np.float32)
    assert np.all(r.astype(np.float64) == r64), "a fused multiply-add of the kernel would round"
    return r


def _exact_sub(a, b):
    r = (a - b).astype(np.float32)
    assert np.all(r.astype(np.float64) == a.astype(np.float64) - b.astype(np.float64))
    return r


def _thresholds(shift, thr):
    """c1_thresholds: T for the SIMD body (round) and the scalar tail (truncate)."""
    t = thr & 255
    if t < 255 and ((t + 1) << shift) <= 2048:
        M = (t + 1) << shift
        tr, tt = (M * M - M + 1 - 0.5) / 16384.0, (M * M - 0.5) / 16384.0
        assert float(f32(tr)) == tr and float(f32(tt)) == tt
        return f32(tr), f32(tt)
    return f32(1024.0), f32(1024.0)


def fused_c1_fp32(img, shift, thr):
    H, W = img.shape
    p = img.astype(np.int64)
    pp = np.pad(p, ((0, 0), (1, 1)))
    h = pp[:, :-2] + 2 * pp[:, 1:-1] + pp[:, 2:]               # horizontal [1 2 1] (16-bit lanes)
    g16 = (h[:-2] + 2 * h[1:-1] + h[2:]) & 0xFFF0                # 16 x Gaussian of rows 1 .. H-2
    t = (np.uint32(0x45C00000) | g16.astype(np.uint32)).view(np.float32)
    assert np.all(t.astype(np.float64) == 6144 + g16 / 2048.0)
    d = _exact_sub(t[:, 2:], t[:, :-2])                          # columns 1 .. W-2
    D = (d[:-1] + d[1:]).astype(np.float32)
    gx = (D[:-1] + D[1:]).astype(np.float32)                     # rows 2 .. H-3
    e = _exact_sub(t[2:], t[:-2])
    gy = (_fma(e[:, 1:-1], f32(2), e[:, :-2]) + e[:, 2:]).astype(np.float32)
    tr, tt = _thresholds(shift, thr)
    T = np.where(np.arange(1, W - 1) < W - W % 16, tr, tt).astype(np.float32)[None, :]
    r = _fma(-gx, gx, _fma(-gy, gy, np.broadcast_to(T, gx.shape)))
    assert not np.any(r == 0)
    out = np.zeros((H, W), np.uint8)
    out[2:H - 2, 1:W - 1] = np.where(np.signbit(r), 255, 0)
    return out


def _frames(rng, W, H):
    yy, xx = np.indices((H, W))
    return [rng.integers(0, 256, (H, W), dtype=np.uint8),
            ((yy + xx) % 2 * 255).astype(np.uint8),                 # checkerboard: largest |gx|, |gy|
            (xx % 2 * 255).astype(np.uint8),
            ((yy % 3 == 0) * 255).astype(np.uint8),
            (rng.integers(0, 2, (H, W)) * 255).astype(np.uint8)]


@pytest.mark.parametrize("W,H", [(64, 40), (37, 21), (130, 66)])
def test_fp32_chain_matches_oracle(rng, W, H):
    for img in _frames(rng, W, H):
        for shift, thr in [(0, 128), (1, 40), (0, 0), (0, 255), (2, 10), (3, 254), (0, 200), (4, 127)]:
            ref, (sx, sy, ex, ey) = OC.cfg1_chain(img, shift, thr)
            got = fused_c1_fp32(img, shift, thr)
            np.testing.assert_array_equal(got[sy:ey, sx:ex], ref[sy:ey, sx:ex], err_msg=f"{W}x{H} {shift} {thr}")


def test_fp32_chain_every_threshold_and_shift(rng):
    for img in (rng.integers(0, 256, (20, 40), dtype=np.uint8), (rng.integers(0, 2, (20, 40)) * 255).astype(np.uint8)):
        for shift in range(6):
            for thr in range(256):
                ref, (sx, sy, ex, ey) = OC.cfg1_chain(img, shift, thr)
                got = fused_c1_fp32(img, shift, thr)
                assert np.array_equal(got[sy:ey, sx:ex], ref[sy:ey, sx:ex]), (shift, thr)
