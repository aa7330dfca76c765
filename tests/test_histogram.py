"""vxHistogramNode into a vx_distribution.

CPU: the reference AGO library (one execution of a one-node graph) must equal the numpy
binning (oracle/pixelwise.py) for distributions whose range divides into the bins -- the
cases where its window-based fast paths and the OpenVX formula agree -- on images whose width
is a multiple of 16: its SIMD loops read whole 16-pixel groups, so other widths count row
padding into bin 0 or drop the last columns (W = 38: 210 padding zeros counted; W = 33: the
last column missing).  GPU: the engine must equal the formula for every distribution and
width, over repeated executions."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from oracle import pixelwise as P
from mivisionx_b200 import vx as V

DISTS = [(256, 0, 256), (16, 0, 256), (10, 20, 200), (3, 50, 150), (1, 100, 50), (64, 64, 128), (2, 0, 256)]
ODD = [(7, 0, 256), (5, 13, 101), (255, 1, 255)]   # range % bins != 0


def _ref_api():
    lib = O.ref_lib()
    if lib is None:
        pytest.skip("reference library not built")
    return V.OpenVX(lib)


def run_histogram(api, img, bins, offset, rng, reps=1):
    ctx = api.obj(api.vxCreateContext(), "context")
    try:
        h, w = img.shape
        src = api.obj(api.vxCreateImage(ctx, w, h, V.VX_DF_IMAGE_U8), "image")
        api.write_plane(src, img)
        dist = api.obj(api.vxCreateDistribution(ctx, bins, offset, rng), "distribution")
        g = api.obj(api.vxCreateGraph(ctx), "graph")
        api.obj(api.vxHistogramNode(g, src, dist), "node")
        api.ok(api.vxVerifyGraph(g), "verify")
        for _ in range(reps):
            api.ok(api.vxProcessGraph(g), "process")
        out = np.zeros(bins, np.uint32)
        api.ok(api.vxCopyDistribution(dist, out.ctypes.data, V.VX_READ_ONLY, V.VX_MEMORY_TYPE_HOST), "copy")
        return out
    finally:
        api.vxReleaseContext(C.byref(C.c_void_p(ctx)))


def _image(w, h, seed):
    r = np.random.default_rng(seed)
    img = r.integers(0, 256, (h, w), dtype=np.int32).astype(np.uint8)
    img[: h // 3, : w // 3] = 200              # a flat block (one hot bin)
    return img


@pytest.mark.parametrize("W,H", [(64, 48), (48, 21), (1920, 1080)])
@pytest.mark.parametrize("bins,offset,rng", DISTS)
def test_reference_histogram(W, H, bins, offset, rng):
    img = _image(W, H, W + bins)
    np.testing.assert_array_equal(run_histogram(_ref_api(), img, bins, offset, rng), P.histogram(img, bins, offset, rng))


@pytest.mark.gpu
@pytest.mark.parametrize("W,H", [(64, 48), (37, 21), (1920, 1080), (3840, 2160), (1, 1)])
@pytest.mark.parametrize("bins,offset,rng", DISTS + ODD)
def test_engine_histogram(cuda, W, H, bins, offset, rng):
    img = _image(W, H, W + bins)
    got = run_histogram(V.OpenVX(), img, bins, offset, rng, reps=2)
    np.testing.assert_array_equal(got, P.histogram(img, bins, offset, rng))
