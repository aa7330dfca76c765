"""The autotuner's launch-shape table (mivisionx_b200/autotune.py writes it, vxVerifyGraph
reads it): lookup by exact frame size, else the nearest pixel count; and on the GPU, every
shape of the tuning space gives the same graph output as the default one."""
import ctypes as C
import json
import os

import numpy as np
import pytest

from mivisionx_b200 import vx as V
from mivisionx_b200 import workloads as WL


def _lookup(lib, kernel, w, h, n=4):
    out = (C.c_uint32 * n)()
    f = lib.agovx_tune_lookup
    f.argtypes, f.restype = [C.c_char_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p], C.c_int
    got = f(kernel.encode(), w, h, n, C.cast(out, C.c_void_p))
    return list(out) if got else None


@pytest.fixture
def table(tmp_path, monkeypatch):
    from mivisionx_b200 import native
    lib = native.openvx()
    path = tmp_path / "tune.json"
    monkeypatch.setenv("AGO_B200_TUNE_FILE", str(path))

    def write(entries):
        path.write_text(json.dumps({"device": "test", "entries": entries}))
        lib.agovx_tune_reload()
        return lib
    yield write
    monkeypatch.delenv("AGO_B200_TUNE_FILE")
    lib.agovx_tune_reload()


def test_lookup_exact_and_nearest(table):
    lib = table([{"kernel": "k", "width": 1920, "height": 1080, "params": [12, 4, 6, 1]},
                 {"kernel": "k", "width": 640, "height": 480, "params": [6, 2, 12, 1]},
                 {"kernel": "other", "width": 1920, "height": 1080, "params": [1, 2, 3, 4]}])
    assert _lookup(lib, "k", 1920, 1080) == [12, 4, 6, 1]
    assert _lookup(lib, "k", 1280, 720) == [12, 4, 6, 1]      # 0.92 MP: nearer to 2.07 MP than to 0.31 MP in log
    assert _lookup(lib, "k", 320, 240) == [6, 2, 12, 1]
    assert _lookup(lib, "k", 3840, 2160) == [12, 4, 6, 1]
    assert _lookup(lib, "missing", 1920, 1080) is None
    assert _lookup(lib, "k", 1920, 1080, n=3) is None         # parameter count must match


def test_missing_file_gives_defaults(table, tmp_path, monkeypatch):
    from mivisionx_b200 import native
    lib = native.openvx()
    monkeypatch.setenv("AGO_B200_TUNE_FILE", str(tmp_path / "absent.json"))
    lib.agovx_tune_reload()
    assert _lookup(lib, "fused_GaussSobelMagDepthThresh", 1920, 1080) is None


def test_committed_table_is_well_formed():
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "mivisionx_b200", "tune", "b200.json")
    if not os.path.exists(path):
        pytest.skip("no committed table")
    t = json.load(open(path))
    kernels = {e["kernel"] for e in t["entries"]}
    assert {"fused_GaussSobelMagDepthThresh_tma", "fused_GaussSobelMagDepthThresh", "ScaleGaussianHalf_U8_U8_5x5"} <= kernels
    for e in t["entries"]:
        n = 2 if e["kernel"].endswith("_tma") else 4
        assert len(e["params"]) == n and e["width"] > 0 and e["height"] > 0
        if e["kernel"].endswith("_tma"):
            rows, warps = e["params"]
            assert rows in (18, 24, 36, 48) and warps in (1, 2, 4) and (rows, warps) != (48, 4)


CHAIN_SHAPES = [[18, 4, 6, 0], [6, 2, 1, 1], [12, 8, 3, 1], [24, 4, 2, 1], [18, 2, 12, 1]]
HALF_SHAPES = [[32, 8, 1, 0], [32, 2, 16, 1], [64, 4, 4, 1], [128, 8, 1, 1], [128, 2, 4, 1]]


TMA_CHAIN_SHAPES = [[36, 2], [18, 1], [24, 1], [36, 1], [48, 1], [18, 2], [24, 2], [48, 2], [18, 4], [24, 4], [36, 4]]


@pytest.mark.gpu
@pytest.mark.parametrize("params", TMA_CHAIN_SHAPES)
def test_tma_chain_shapes_match_oracle(cuda, table, params):
    """Every tile shape of the TMA-staged chain, taken from the table by the engine."""
    import oracle_chains as OC
    table([{"kernel": "fused_GaussSobelMagDepthThresh_tma", "width": 1920, "height": 1080, "params": params}])
    api = V.OpenVX()
    ctx = api.obj(api.vxCreateContext(), "context")
    try:
        sizes = [(1920, 1080), (640, 480), (333, 97), (1920, 1080), (64, 48), (3840, 2160)]
        frames = [WL.cfg1_image(seed=50 + i, width=w, height=h) for i, (w, h) in enumerate(sizes)]
        g = WL.Cfg1Graph(api, ctx, sizes)
        for _ in range(2):
            g.run(frames)
            for out, img in zip(g.results(), frames):
                ref, (sx, sy, ex, ey) = OC.cfg1_chain(img, 0, 128)
                np.testing.assert_array_equal(out[0][sy:ey, sx:ex], ref[sy:ey, sx:ex])
    finally:
        api.vxReleaseContext(C.byref(C.c_void_p(ctx)))


@pytest.mark.gpu
@pytest.mark.parametrize("params", CHAIN_SHAPES)
def test_chain_shapes_match_oracle(cuda, table, params):
    """The register form's shapes (the no-TMA optimizer flag selects that form)."""
    import oracle_chains as OC
    table([{"kernel": "fused_GaussSobelMagDepthThresh", "width": 1920, "height": 1080, "params": params}])
    api = V.OpenVX()
    ctx = api.obj(api.vxCreateContext(), "context")
    try:
        sizes = [(1920, 1080), (640, 480), (333, 97), (1920, 1080), (64, 48)]
        frames = [WL.cfg1_image(seed=30 + i, width=w, height=h) for i, (w, h) in enumerate(sizes)]
        g = WL.Cfg1Graph(api, ctx, sizes, flags=V.OPT_NO_TMA)
        for _ in range(2):      # the queue words must be back to zero for the second launch
            g.run(frames)
            for out, img in zip(g.results(), frames):
                ref, (sx, sy, ex, ey) = OC.cfg1_chain(img, 0, 128)
                np.testing.assert_array_equal(out[0][sy:ey, sx:ex], ref[sy:ey, sx:ex])
    finally:
        api.vxReleaseContext(C.byref(C.c_void_p(ctx)))


@pytest.mark.gpu
@pytest.mark.parametrize("params", HALF_SHAPES)
def test_pyramid_shapes_match_oracle(cuda, table, params):
    import test_graph_cfg4 as G4
    table([{"kernel": "ScaleGaussianHalf_U8_U8_5x5", "width": 960, "height": 540, "params": params}])
    api = V.OpenVX()
    ctx = api.obj(api.vxCreateContext(), "context")
    try:
        G4.run_and_compare(api, ctx, [(1920, 1080), (640, 480), (320, 240)], 500, executions=2)
    finally:
        api.vxReleaseContext(C.byref(C.c_void_p(ctx)))
