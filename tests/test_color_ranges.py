"""Range facts the fused RGB -> YUV / scale kernel (k_fused_rgb_yuv_scale8,
mivisionx_b200/csrc/geometry.cu) relies on: in the SIMD body of HafCpu_ColorConvert_*_RGB
(color_convert.cpp:2492, :2707) the float Y, U and V of every RGB triple lie in [0, 256), so
trunc_sat16 followed by sat8 is plain truncation, which the kernel takes as one
round-toward-zero add of 2^23.  Checked over all 2^24 triples in float32 with the kernel's
operation order (each product and sum rounded to nearest)."""
import numpy as np

f32 = np.float32


def test_yuv_of_every_rgb_triple_in_0_256():
    v = np.arange(256, dtype=f32)
    r, g = np.meshgrid(v, v, indexing="ij")
    r, g = r.ravel(), g.ravel()
    lo, hi = [np.inf] * 3, [-np.inf] * 3
    for b in range(256):
        bb = f32(b)
        y = (r * f32(0.2126) + g * f32(0.7152)) + bb * f32(0.0722)
        u = ((r * f32(-0.1146) + g * f32(-0.3854)) + bb * f32(0.5)) + f32(128.0)
        w = ((r * f32(0.5) + g * f32(-0.4542)) + bb * f32(-0.0458)) + f32(128.0)
        for k, a in enumerate((y, u, w)):
            assert a.dtype == np.float32
            lo[k] = min(lo[k], float(a.min()))
            hi[k] = max(hi[k], float(a.max()))
    assert min(lo) >= 0.0 and max(hi) < 256.0, (lo, hi)
