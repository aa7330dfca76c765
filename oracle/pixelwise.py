"""Numpy restatement of the AGO element-wise kernels and 3x3 Box / Median / Dilate / Erode
filters -- TEST INFRASTRUCTURE ONLY (imported by tests/ as the checker).

Every function returns the full output plane the reference writes; callers compare the
OpenVX valid region.  The 3x3 filters return rows/columns [1, H-1) x [1, W-1) filled and the
border 0 (the reference's border pixels there depend on bytes outside the row and are
outside the valid region).  File:line references are to amd_openvx/openvx/ago/.
"""
from __future__ import annotations

import numpy as np


def _i32(a):
    return np.asarray(a).astype(np.int32)


def _sat_s16(v):
    return np.clip(v, -32768, 32767).astype(np.int16)


def _wrap_s16(v):
    return v.astype(np.int16)   # two's complement truncation of the exact int32 result


def add(a, b, out_dtype, saturate):
    """HafCpu_Add_* (ago_haf_cpu_arithmetic.cpp:26 U8 wrap, :186 U8 sat, :672 S16 from U8,
    :1050/:1232 S16+U8, :2158/:2346 S16+S16)."""
    s = _i32(a) + _i32(b)
    if out_dtype == np.uint8:
        return (np.minimum(s, 255) if saturate else s & 0xFF).astype(np.uint8)
    return _sat_s16(s) if saturate else _wrap_s16(s)


def sub(a, b, out_dtype, saturate):
    """HafCpu_Sub_* (ago_haf_cpu_arithmetic.cpp:352 U8 wrap, :512 U8 sat, :863 S16 from U8,
    :1418/:1604 S16-U8, :1790/:1972 U8-S16, :2534/:2722 S16-S16)."""
    s = _i32(a) - _i32(b)
    if out_dtype == np.uint8:
        return (np.maximum(s, 0) if saturate else s & 0xFF).astype(np.uint8)
    return _sat_s16(s) if saturate else _wrap_s16(s)


def absdiff(a, b):
    """HafCpu_AbsDiff_U8_U8U8 (ago_haf_cpu_arithmetic.cpp:2910) and
    HafCpu_AbsDiff_S16_S16S16_Sat (:3114): |a - b| exact in 32 bits, S16 clamped to 32767."""
    d = np.abs(_i32(a) - _i32(b))
    return d.astype(np.uint8) if np.asarray(a).dtype == np.uint8 else np.minimum(d, 32767).astype(np.int16)


def convert_depth(a, out_dtype, policy_saturate, shift):
    """HafCpu_ColorDepth_U8_S16_Wrap (ago_haf_cpu_arithmetic.cpp:3488): low byte of v >> shift;
    _Sat (:3546): clamp(v >> shift, 0, 255); HafCpu_ColorDepth_S16_U8 (:3604): v << shift in
    16 bits."""
    v = _i32(a)
    if out_dtype == np.uint8:
        v = v >> shift
        return (np.clip(v, 0, 255) if policy_saturate else v & 0xFF).astype(np.uint8)
    return _wrap_s16(v << shift)


def table_lookup(a, table, offset=0):
    """HafCpu_Lut_U8_U8 / HafCpu_Lut_S16_S16 (ago_haf_cpu_arithmetic.cpp:4916): table[v + offset]
    (offset 0 for U8 tables, count / 2 for S16 ones)."""
    return np.asarray(table)[_i32(a) + int(offset)]


def integral_image(a):
    """HafCpu_IntegralImage_U32_U8 (ago_haf_cpu_arithmetic.cpp:7057): sum over [0, x] x [0, y]."""
    return np.cumsum(np.cumsum(np.asarray(a, np.uint64), axis=0), axis=1).astype(np.uint32)


def histogram(a, bins, offset, rng):
    """OpenVX histogram binning: v in [offset, offset + range) counts into (v - offset) * bins /
    range.  The reference (HafCpu_HistogramFixedBins_DATA_U8, ago_haf_cpu_histogram.cpp:519)
    bins by window = ceil(range / bins) in its fast paths, which agrees when range % bins == 0."""
    v = np.asarray(a, np.int64).ravel()
    v = v[(v >= offset) & (v < offset + rng)]
    return np.bincount((v - offset) * bins // rng, minlength=bins).astype(np.uint32)


def logical(op, a, b=None):
    """HafCpu_And/Or/Xor_U8_U8U8, HafCpu_Not_U8_U8 (ago_haf_cpu_logical.cpp:518, :31)."""
    a = np.asarray(a, np.uint8)
    if op == "not":
        return np.bitwise_not(a)
    b = np.asarray(b, np.uint8)
    return {"and": np.bitwise_and, "or": np.bitwise_or, "xor": np.bitwise_xor}[op](a, b)


def threshold_range(a, lower, upper):
    """HafCpu_Threshold_U8_U8_Range (ago_haf_cpu_arithmetic.cpp:3742): 0 where v > upper or
    v < lower, else 255; both bounds as vx_uint8."""
    a = np.asarray(a, np.uint8)
    lo, hi = int(lower) & 0xFF, int(upper) & 0xFF
    return np.where((a > hi) | (a < lo), 0, 255).astype(np.uint8)


def _windows(img):
    """The nine shifted views of the interior: w[dy+1][dx+1][y-1, x-1] = img[y+dy, x+dx]."""
    H, W = img.shape
    return [[img[1 + dy:H - 1 + dy, 1 + dx:W - 1 + dx] for dx in (-1, 0, 1)] for dy in (-1, 0, 1)]


def _interior(img, vals):
    out = np.zeros_like(np.asarray(img, np.uint8))
    out[1:-1, 1:-1] = vals
    return out


def box3x3(img):
    """HafCpu_Box_U8_U8_3x3 (ago_haf_cpu_filter.cpp:34): the SIMD body's (sum * 7282) >> 16
    (mulhi by ceil(2^16 / 9)) and the scalar parts' (int)((float)sum / 9.0f) are both
    floor(sum / 9) for sums of nine bytes; the body's form is restated here."""
    img = np.asarray(img, np.uint8)
    s = sum(_i32(v) for row in _windows(img) for v in row)
    return _interior(img, ((s * 7282) >> 16).astype(np.uint8))


def gaussian3x3(img):
    """HafCpu_Gaussian_U8_U8_3x3 (ago_haf_cpu_filter.cpp:1518): [1 2 1]^T [1 2 1] sum >> 4."""
    img = np.asarray(img, np.uint8)
    w = _windows(img)
    k = ((1, 2, 1), (2, 4, 2), (1, 2, 1))
    s = sum(k[i][j] * _i32(w[i][j]) for i in range(3) for j in range(3))
    return _interior(img, (s >> 4).astype(np.uint8))


def threshold_binary(a, value):
    """HafCpu_Threshold_U8_U8_Binary (ago_haf_cpu_arithmetic.cpp:3660): 255 where v > value."""
    return np.where(np.asarray(a, np.uint8) > (int(value) & 0xFF), 255, 0).astype(np.uint8)


def motion_mask(prev, cur, thr):
    """AbsDiff(cur, prev) -> Gaussian3x3 -> Threshold(BINARY, thr) -> Dilate3x3 -> Erode3x3 ->
    Median3x3; valid on [4, W-4) x [4, H-4)."""
    return median3x3(erode3x3(dilate3x3(threshold_binary(gaussian3x3(absdiff(cur, prev)), thr))))


def dilate3x3(img):
    """HafCpu_Dilate_U8_U8_3x3 (ago_haf_cpu_filter.cpp:221): maximum of the window."""
    img = np.asarray(img, np.uint8)
    return _interior(img, np.max(np.stack([v for row in _windows(img) for v in row]), axis=0))


def erode3x3(img):
    """HafCpu_Erode_U8_U8_3x3 (ago_haf_cpu_filter.cpp:298): minimum of the window."""
    img = np.asarray(img, np.uint8)
    return _interior(img, np.min(np.stack([v for row in _windows(img) for v in row]), axis=0))


def median3x3(img):
    """HafCpu_Median_U8_U8_3x3 (ago_haf_cpu_filter.cpp:3842): median of the nine pixels."""
    img = np.asarray(img, np.uint8)
    st = np.sort(np.stack([v for row in _windows(img) for v in row]), axis=0)
    return _interior(img, st[4])
