"""Seeded synthetic inputs and OpenVX graph builders for the benchmark configurations.

The graph builders only use the OpenVX API (through ``vx.OpenVX``), so the same function
builds the graph on this package's B200 engine and on the reference AGO CPU library.

Random numbers come from PCG32 (O'Neill's pcg32: 64-bit LCG state, XSH-RR output), generated
in vectorised blocks with LCG jump-ahead so full-size frames are produced in milliseconds.
A uniform byte is the top 8 bits of a PCG32 output.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import vx as V

_MULT = np.uint64(6364136223846793005)


def pcg32(seed: int, n: int, stream: int = 54) -> np.ndarray:
    """n outputs of pcg32 seeded like pcg32_srandom_r(seed, stream)."""
    with np.errstate(over="ignore"):
        inc = np.uint64(((stream << 1) | 1) & 0xFFFFFFFFFFFFFFFF)
        s = np.uint64(0)
        s = s * _MULT + inc
        s = s + np.uint64(seed & 0xFFFFFFFFFFFFFFFF)
        s = s * _MULT + inc
        block = 4096
        # states of the first block, sequentially
        first = np.empty(block, np.uint64)
        x = s
        for i in range(block):
            first[i] = x
            x = x * _MULT + inc
        # affine map of `block` steps: x -> A x + B
        A, B = np.uint64(1), np.uint64(0)
        m, c = _MULT, inc
        k = block
        while k:
            if k & 1:
                A, B = A * m, B * m + c
            m, c = m * m, c * m + c
            k >>= 1
        nb = (n + block - 1) // block
        states = np.empty(nb * block, np.uint64)
        cur = first
        for b in range(nb):
            states[b * block:(b + 1) * block] = cur
            cur = cur * A + B
        old = states[:n]
        xs = (((old >> np.uint64(18)) ^ old) >> np.uint64(27)).astype(np.uint32)
        rot = (old >> np.uint64(59)).astype(np.uint32)
        out = (xs >> rot) | (xs << ((np.uint32(32) - rot) & np.uint32(31)))
    return out.astype(np.uint32)


def uniform_u8(seed: int, shape, stream: int = 54) -> np.ndarray:
    n = int(np.prod(shape))
    return (pcg32(seed, n, stream) >> np.uint32(24)).astype(np.uint8).reshape(shape)


def uniform01(seed: int, n: int, stream: int = 54) -> np.ndarray:
    return pcg32(seed, n, stream).astype(np.float64) / 4294967296.0


def gaussian(seed: int, n: int, stream: int = 54) -> np.ndarray:
    """Standard normal samples (Box-Muller over PCG32 uniforms)."""
    m = (n + 1) // 2
    u = uniform01(seed, 2 * m, stream)
    u1 = np.maximum(u[0::2], 1e-12)
    r = np.sqrt(-2.0 * np.log(u1))
    t = 2.0 * np.pi * u[1::2]
    return np.concatenate([r * np.cos(t), r * np.sin(t)])[:n]


# ---------------------------------------------------------------- inputs
def cfg1_image(seed: int = 1, width: int = 1920, height: int = 1080) -> np.ndarray:
    """One U8 frame, i.i.d. uniform 0..255 from a seeded PCG32."""
    return uniform_u8(seed, (height, width))


def cfg2_scene(seed: int = 2, width: int = 3840, height: int = 2160, rects: int = 200, sigma: float = 8.0) -> np.ndarray:
    """Linear gradient background (0..200 across x) + `rects` seeded axis-aligned rectangles
    (sides 16..400 px, intensity uniform 0..255) + Gaussian noise (sigma 8), clipped."""
    img = np.tile(np.linspace(0.0, 200.0, width, dtype=np.float64), (height, 1))
    r = pcg32(seed, rects * 5, stream=7)
    for i in range(rects):
        w = 16 + int(r[5 * i + 0] % 385)
        h = 16 + int(r[5 * i + 1] % 385)
        x0 = int(r[5 * i + 2] % max(1, width - w))
        y0 = int(r[5 * i + 3] % max(1, height - h))
        img[y0:y0 + h, x0:x0 + w] = float(r[5 * i + 4] >> 24)
    img += sigma * gaussian(seed, width * height, stream=11).reshape(height, width)
    return np.clip(np.rint(img), 0, 255).astype(np.uint8)


CFG4_SIZES = ((640, 480), (1280, 720), (1920, 1080), (3840, 2160))


def cfg4_sizes(n: int = 64, seed: int = 4) -> list[tuple[int, int]]:
    """Per-frame (width, height), each drawn from CFG4_SIZES by a seeded PCG32."""
    r = pcg32(seed, n, stream=19)
    return [CFG4_SIZES[int(v) % len(CFG4_SIZES)] for v in r]


def cfg4_pair(seed: int, width: int, height: int, max_shift: float = 8.0, noise_sigma: float = 2.0):
    """(frame1, frame2, (dx, dy)): frame1 is a config-2 style scene (rectangle count scaled to
    the area); frame2 is frame1 translated by (dx, dy) ~ U(-max_shift, max_shift) with bilinear
    interpolation (edge-clamped) plus N(0, noise_sigma^2) noise, rounded and clipped to U8."""
    rects = max(8, int(round(200 * width * height / (3840 * 2160))))
    f1 = cfg2_scene(seed=seed, width=width, height=height, rects=rects)
    dx, dy = (uniform01(seed, 2, stream=23) * 2.0 - 1.0) * max_shift
    # frame2(x, y) = frame1(x - dx, y - dy)
    xs = np.clip(np.arange(width, dtype=np.float64) - dx, 0, width - 1)
    ys = np.clip(np.arange(height, dtype=np.float64) - dy, 0, height - 1)
    x0 = np.minimum(np.floor(xs).astype(np.int64), width - 2)
    y0 = np.minimum(np.floor(ys).astype(np.int64), height - 2)
    fx, fy = xs - x0, ys - y0
    a = f1.astype(np.float64)
    top = a[y0][:, x0] * (1 - fx) + a[y0][:, x0 + 1] * fx
    bot = a[y0 + 1][:, x0] * (1 - fx) + a[y0 + 1][:, x0 + 1] * fx
    f2 = top * (1 - fy)[:, None] + bot * fy[:, None]
    f2 += noise_sigma * gaussian(seed, width * height, stream=29).reshape(height, width)
    return f1, np.ascontiguousarray(np.clip(np.rint(f2), 0, 255).astype(np.uint8)), (float(dx), float(dy))


KEYPOINT_DTYPE = np.dtype([("x", "<i4"), ("y", "<i4"), ("strength", "<f4"), ("scale", "<f4"),
                           ("orientation", "<f4"), ("tracking_status", "<i4"), ("error", "<f4")])


def cfg4_points(seed: int, width: int, height: int, n: int = 2000) -> np.ndarray:
    """n vx_keypoint_t records at seeded uniform integer positions, tracking_status 1."""
    r = pcg32(seed, 2 * n, stream=31)
    kp = np.zeros(n, KEYPOINT_DTYPE)
    kp["x"] = (r[0::2] % width).astype(np.int32)
    kp["y"] = (r[1::2] % height).astype(np.int32)
    kp["tracking_status"] = 1
    return kp


def pyramid_sizes(width: int, height: int, levels: int, scale: float = 0.5) -> list[tuple[int, int]]:
    """OpenVX pyramid level sizes: level l is ceil(size * scale^l), as AGO computes them."""
    out = [(width, height)]
    for _ in range(1, levels):
        w, h = out[-1]
        out.append((int(np.ceil(np.float32(w) * np.float32(scale))), int(np.ceil(np.float32(h) * np.float32(scale)))))
    return out


def cfg3_frame(seed: int = 3, width: int = 3840, height: int = 2160, waves: int = 8) -> np.ndarray:
    """RGB frame: per channel a sum of `waves` random 2-D sinusoids scaled to 0..255, plus
    uniform noise in [-10, 10], clipped."""
    xs, ys = np.arange(width, dtype=np.float64), np.arange(height, dtype=np.float64)
    out = np.empty((height, width, 3), np.uint8)
    p = uniform01(seed, 3 * waves * 4, stream=13)
    for ch in range(3):
        acc = np.zeros((height, width), np.float32)
        for k in range(waves):
            a, b, c, d = p[(ch * waves + k) * 4:(ch * waves + k) * 4 + 4]
            fx, fy = (a - 0.5) * 0.02, (b - 0.5) * 0.02
            # sin(fx x + fy y + 2 pi c) = sin(fx x) cos(fy y + 2 pi c) + cos(fx x) sin(fy y + 2 pi c)
            u, v = fy * ys + 2 * np.pi * c, fx * xs
            amp = np.float32(0.5 + d)
            acc += np.outer((np.cos(u) * amp).astype(np.float32), np.sin(v).astype(np.float32))
            acc += np.outer((np.sin(u) * amp).astype(np.float32), np.cos(v).astype(np.float32))
        acc = (acc - acc.min()) / max(1e-6, float(acc.max() - acc.min())) * 255.0
        noise = (uniform01(seed + ch + 1, width * height, stream=17).reshape(height, width) * 20.0 - 10.0).astype(np.float32)
        out[..., ch] = np.clip(np.rint(acc + noise), 0, 255).astype(np.uint8)
    return out


def cfg3_affine(seed: int = 3, cx: float = 960.0, cy: float = 540.0) -> np.ndarray:
    """OpenVX 2x3 affine matrix in vx_matrix layout (3 rows x 2 columns, m[j][i]): rotation
    +-15 deg, scale 0.8..1.2, translation +-50 px, about the image centre."""
    u = uniform01(seed, 4, stream=19)
    th = math.radians((u[0] * 2 - 1) * 15.0)
    s = 0.8 + 0.4 * u[1]
    tx, ty = (u[2] * 2 - 1) * 50.0, (u[3] * 2 - 1) * 50.0
    a, b = s * math.cos(th), s * math.sin(th)
    # x' = a x - b y + c0 ; y' = b x + a y + c1 (destination -> source mapping)
    c0 = cx - a * cx + b * cy + tx
    c1 = cy - b * cx - a * cy + ty
    return np.array([[a, b], [-b, a], [c0, c1]], dtype=np.float32)


# ---------------------------------------------------------------- graph builders
def _u8_image(a: V.OpenVX, ctx, w: int, h: int, bufs, i: int):
    """Image i of a graph: from the application buffer bufs[i] when given, else allocated."""
    if bufs is not None:
        return a.image_from_host(ctx, bufs[i])
    return a.obj(a.vxCreateImage(ctx, w, h, V.VX_DF_IMAGE_U8), "image")


class Cfg1Graph:
    """Gaussian3x3 -> Sobel3x3 -> Magnitude -> ConvertDepth(SATURATE, shift) -> Threshold(BINARY)
    for each of `sizes` frames, all in ONE OpenVX graph (independent sub-graphs), border
    UNDEFINED, intermediates virtual."""

    def __init__(self, api: V.OpenVX, ctx, sizes, shift: int = 0, thr: int = 128, flags: int | None = None,
                 host_io: dict | None = None):
        host_io = host_io or {}
        self.api, self.ctx = api, ctx
        a = api
        self.graph = a.obj(a.vxCreateGraph(ctx), "graph")
        if flags is not None:
            a.set_optimizer_flags(self.graph, flags)
        self.inputs, self.outputs = [], []
        self.shift = a.scalar(ctx, V.VX_TYPE_INT32, shift)
        self.thr = a.threshold_binary(ctx, thr)
        g = self.graph
        for i, (w, h) in enumerate(sizes):
            src = _u8_image(a, ctx, w, h, host_io.get("src"), i)
            dst = _u8_image(a, ctx, w, h, host_io.get("dst"), i)
            gau = a.vxCreateVirtualImage(g, w, h, V.VX_DF_IMAGE_U8)
            gx = a.vxCreateVirtualImage(g, w, h, V.VX_DF_IMAGE_S16)
            gy = a.vxCreateVirtualImage(g, w, h, V.VX_DF_IMAGE_S16)
            mag = a.vxCreateVirtualImage(g, w, h, V.VX_DF_IMAGE_S16)
            dep = a.vxCreateVirtualImage(g, w, h, V.VX_DF_IMAGE_U8)
            for n in (a.vxGaussian3x3Node(g, src, gau), a.vxSobel3x3Node(g, gau, gx, gy),
                      a.vxMagnitudeNode(g, gx, gy, mag),
                      a.vxConvertDepthNode(g, mag, dep, V.VX_CONVERT_POLICY_SATURATE, self.shift),
                      a.vxThresholdNode(g, dep, self.thr, dst)):
                a.obj(n, "node")
            self.inputs.append(src)
            self.outputs.append(dst)
        a.ok(a.vxVerifyGraph(g), "vxVerifyGraph")

    def run(self, frames=None):
        a = self.api
        if frames is not None:
            for img, f in zip(self.inputs, frames):
                a.write_plane(img, f)
        a.ok(a.vxProcessGraph(self.graph), "vxProcessGraph")

    def results(self):
        return [(self.api.read_plane(o), self.api.valid_region(o)) for o in self.outputs]


def motion_pair(seed: int = 1, width: int = 3840, height: int = 2160, rects: int = 150, sigma: float = 3.0):
    """Two U8 frames of a scene: a horizontal gradient with `rects` seeded rectangles (sides
    16..256 px, intensity uniform 0..255), each displaced by up to 12 px in the second frame,
    plus independent N(0, sigma^2) noise per frame."""
    r = np.random.default_rng(seed)
    base = np.tile(np.linspace(0.0, 160.0, width), (height, 1))
    f0, f1 = base.copy(), base.copy()
    for _ in range(rects):
        w, h = (int(v) for v in r.integers(16, 257, 2))
        x, y = int(r.integers(0, max(1, width - w))), int(r.integers(0, max(1, height - h)))
        dx, dy = (int(v) for v in r.integers(-12, 13, 2))
        level = float(r.integers(0, 256))
        f0[y:y + h, x:x + w] = level
        x1, y1 = min(max(x + dx, 0), max(0, width - w)), min(max(y + dy, 0), max(0, height - h))
        f1[y1:y1 + h, x1:x1 + w] = level
    out = []
    for f in (f0, f1):
        f = f + sigma * r.standard_normal(f.shape)
        out.append(np.clip(np.rint(f), 0, 255).astype(np.uint8))
    return out[0], out[1]


class MotionGraph:
    """Motion mask of frame pairs: AbsDiff(cur, prev) -> Gaussian3x3 -> Threshold(BINARY, thr) ->
    Dilate3x3 -> Erode3x3 -> Median3x3, for each of `sizes` pairs in one graph, intermediates
    virtual (fused into one pixel-chain kernel by this target)."""

    def __init__(self, api: V.OpenVX, ctx, sizes, thr: int = 24, flags: int | None = None,
                 host_io: dict | None = None):
        host_io = host_io or {}
        self.api, self.ctx = api, ctx
        a = api
        self.graph = a.obj(a.vxCreateGraph(ctx), "graph")
        if flags is not None:
            a.set_optimizer_flags(self.graph, flags)
        self.thr = a.threshold_binary(ctx, thr)
        self.inputs, self.outputs = [], []
        g = self.graph
        for i, (w, h) in enumerate(sizes):
            prev = _u8_image(a, ctx, w, h, host_io.get("prev"), i)
            cur = _u8_image(a, ctx, w, h, host_io.get("cur"), i)
            dst = _u8_image(a, ctx, w, h, host_io.get("dst"), i)
            v = [a.vxCreateVirtualImage(g, w, h, V.VX_DF_IMAGE_U8) for _ in range(5)]
            for n in (a.vxAbsDiffNode(g, cur, prev, v[0]), a.vxGaussian3x3Node(g, v[0], v[1]),
                      a.vxThresholdNode(g, v[1], self.thr, v[2]), a.vxDilate3x3Node(g, v[2], v[3]),
                      a.vxErode3x3Node(g, v[3], v[4]), a.vxMedian3x3Node(g, v[4], dst)):
                a.obj(n, "node")
            self.inputs += [prev, cur]
            self.outputs.append(dst)
        a.ok(a.vxVerifyGraph(g), "vxVerifyGraph")

    def run(self, frames=None):
        """frames: [prev0, cur0, prev1, cur1, ...]"""
        a = self.api
        if frames is not None:
            for img, f in zip(self.inputs, frames):
                a.write_plane(img, f)
        a.ok(a.vxProcessGraph(self.graph), "vxProcessGraph")

    def results(self):
        return [(self.api.read_plane(o), self.api.valid_region(o)) for o in self.outputs]


class Cfg3Graph:
    """Colour and geometry: RGB -> NV12 and RGB -> IYUV, ChannelExtract Y (virtual), ScaleImage
    of Y to half size (bilinear and area), WarpAffine of the bilinear result (nearest and
    bilinear, border CONSTANT 0), for each of `sizes` RGB frames, in one graph."""

    def __init__(self, api: V.OpenVX, ctx, sizes, matrices=None, flags: int | None = None, host_io: dict | None = None):
        """host_io: application buffers per role ("rgb", "nv12", "iyuv", "sb", "sa", "wn", "wb"),
        each a list (one per frame) of per-plane arrays."""
        host_io = host_io or {}
        self.api, self.ctx = api, ctx
        a = api
        self.graph = a.obj(a.vxCreateGraph(ctx), "graph")
        if flags is not None:
            a.set_optimizer_flags(self.graph, flags)
        g = self.graph

        def image(role, i, w, h, fmt):
            if role in host_io:
                return a.image_from_host(ctx, host_io[role][i], fmt, w, h)
            return a.obj(a.vxCreateImage(ctx, w, h, fmt), role)

        self.inputs, self.nv12, self.iyuv, self.scaled, self.warped, self.matrices = [], [], [], [], [], []
        for i, (w, h) in enumerate(sizes):
            m = matrices[i] if matrices is not None else cfg3_affine(seed=17 + i, cx=w / 4, cy=h / 4)
            rgb = image("rgb", i, w, h, V.VX_DF_IMAGE_RGB)
            nv12 = image("nv12", i, w, h, V.VX_DF_IMAGE_NV12)
            iyuv = image("iyuv", i, w, h, V.VX_DF_IMAGE_IYUV)
            y = a.vxCreateVirtualImage(g, w, h, V.VX_DF_IMAGE_U8)
            sb = image("sb", i, w // 2, h // 2, V.VX_DF_IMAGE_U8)
            sa = image("sa", i, w // 2, h // 2, V.VX_DF_IMAGE_U8)
            wn = image("wn", i, w // 2, h // 2, V.VX_DF_IMAGE_U8)
            wb = image("wb", i, w // 2, h // 2, V.VX_DF_IMAGE_U8)
            mat = a.matrix_f32(ctx, m)
            a.obj(a.vxColorConvertNode(g, rgb, nv12), "node")
            a.obj(a.vxColorConvertNode(g, rgb, iyuv), "node")
            a.obj(a.vxChannelExtractNode(g, nv12, V.VX_CHANNEL_Y, y), "node")
            a.obj(a.vxScaleImageNode(g, y, sb, V.VX_INTERPOLATION_BILINEAR), "node")
            a.obj(a.vxScaleImageNode(g, y, sa, V.VX_INTERPOLATION_AREA), "node")
            n1 = a.obj(a.vxWarpAffineNode(g, sb, mat, V.VX_INTERPOLATION_NEAREST_NEIGHBOR, wn), "node")
            n2 = a.obj(a.vxWarpAffineNode(g, sb, mat, V.VX_INTERPOLATION_BILINEAR, wb), "node")
            a.set_border(n1, V.VX_BORDER_CONSTANT, 0)
            a.set_border(n2, V.VX_BORDER_CONSTANT, 0)
            self.inputs.append(rgb); self.nv12.append(nv12); self.iyuv.append(iyuv)
            self.scaled.append((sb, sa)); self.warped.append((wn, wb)); self.matrices.append(m)
        a.ok(a.vxVerifyGraph(g), "vxVerifyGraph")
        self.outputs = [im for i in range(len(sizes)) for im in
                        (self.nv12[i], self.iyuv[i]) + self.scaled[i] + self.warped[i]]

    def run(self, frames=None):
        a = self.api
        if frames is not None:
            for img, f in zip(self.inputs, frames):
                a.write_plane(img, f)
        a.ok(a.vxProcessGraph(self.graph), "vxProcessGraph")

    def results(self):
        """per frame: dict of planes and valid rectangles"""
        a = self.api
        out = []
        for i in range(len(self.inputs)):
            d = {"nv12_y": a.read_plane(self.nv12[i], 0), "nv12_uv": a.read_plane(self.nv12[i], 1),
                 "iyuv_y": a.read_plane(self.iyuv[i], 0), "iyuv_u": a.read_plane(self.iyuv[i], 1),
                 "iyuv_v": a.read_plane(self.iyuv[i], 2)}
            for k, im in (("scale_bilinear", self.scaled[i][0]), ("scale_area", self.scaled[i][1]),
                          ("warp_nearest", self.warped[i][0]), ("warp_bilinear", self.warped[i][1])):
                d[k] = a.read_plane(im)
                d[k + "_rect"] = a.valid_region(im)
            out.append(d)
        return out


class Cfg2Graph:
    """CannyEdgeDetector (3x3 gradient, L1 norm, hysteresis lower/upper) and HarrisCorners
    (gradient 3, block 3, sensitivity k, strength threshold, min distance) on the same U8
    input, for each of `sizes` frames, all in one OpenVX graph."""

    def __init__(self, api: V.OpenVX, ctx, sizes, lower=80, upper=100, k=0.04, strength=1e-3, min_distance=5.0,
                 capacity=32768, flags: int | None = None, host_io: dict | None = None):
        host_io = host_io or {}
        self.api, self.ctx = api, ctx
        a = api
        self.graph = a.obj(a.vxCreateGraph(ctx), "graph")
        if flags is not None:
            a.set_optimizer_flags(self.graph, flags)
        self.hyst = a.threshold_range(ctx, lower, upper)
        self.s_strength = a.scalar(ctx, V.VX_TYPE_FLOAT32, strength)
        self.s_mind = a.scalar(ctx, V.VX_TYPE_FLOAT32, min_distance)
        self.s_k = a.scalar(ctx, V.VX_TYPE_FLOAT32, k)
        self.inputs, self.edges, self.corners, self.num = [], [], [], []
        g = self.graph
        for i, (w, h) in enumerate(sizes):
            src = _u8_image(a, ctx, w, h, host_io.get("src"), i)
            edge = _u8_image(a, ctx, w, h, host_io.get("edge"), i)
            arr = a.obj(a.vxCreateArray(ctx, V.VX_TYPE_KEYPOINT, capacity), "array")
            num = a.scalar(ctx, V.VX_TYPE_SIZE, 0)
            a.obj(a.vxCannyEdgeDetectorNode(g, src, self.hyst, 3, V.VX_NORM_L1, edge), "canny node")
            a.obj(a.vxHarrisCornersNode(g, src, self.s_strength, self.s_mind, self.s_k, 3, 3, arr, num), "harris node")
            self.inputs.append(src); self.edges.append(edge); self.corners.append(arr); self.num.append(num)
        a.ok(a.vxVerifyGraph(g), "vxVerifyGraph")

    def run(self, frames=None):
        a = self.api
        if frames is not None:
            for img, f in zip(self.inputs, frames):
                a.write_plane(img, f)
        a.ok(a.vxProcessGraph(self.graph), "vxProcessGraph")

    def results(self):
        a = self.api
        out = []
        for e, arr, num in zip(self.edges, self.corners, self.num):
            out.append((a.read_plane(e), a.valid_region(e), a.array_items(arr), a.read_scalar(num)))
        return out


class Cfg4Graph:
    """Per frame pair: GaussianPyramid (scale 0.5, `levels` levels, virtual pyramids) of both
    frames and OpticalFlowPyrLK (window, iterations, epsilon, termination) of `points`
    keypoints, all pairs in one OpenVX graph.  The estimates array is the old-points array
    (use_initial_estimate false)."""

    def __init__(self, api: V.OpenVX, ctx, sizes, levels=5, window=9, iterations=20, epsilon=0.01,
                 termination=None, capacity=2000, flags: int | None = None, virtual_pyramids=True,
                 host_io: dict | None = None):
        host_io = host_io or {}
        self.api, self.ctx = api, ctx
        a = api
        self.graph = a.obj(a.vxCreateGraph(ctx), "graph")
        if flags is not None:
            a.set_optimizer_flags(self.graph, flags)
        term = V.VX_TERM_CRITERIA_BOTH if termination is None else termination
        self.s_eps = a.scalar(ctx, V.VX_TYPE_FLOAT32, epsilon)
        self.s_iter = a.scalar(ctx, V.VX_TYPE_UINT32, iterations)
        self.s_est = a.scalar(ctx, V.VX_TYPE_BOOL, 0)
        self.old, self.new, self.pts, self.out, self.pyr = [], [], [], [], []
        g = self.graph
        for i, (w, h) in enumerate(sizes):
            i0 = _u8_image(a, ctx, w, h, host_io.get("old"), i)
            i1 = _u8_image(a, ctx, w, h, host_io.get("new"), i)
            if virtual_pyramids:
                p0 = a.obj(a.vxCreateVirtualPyramid(g, levels, V.VX_SCALE_PYRAMID_HALF, w, h, V.VX_DF_IMAGE_U8), "pyramid")
                p1 = a.obj(a.vxCreateVirtualPyramid(g, levels, V.VX_SCALE_PYRAMID_HALF, w, h, V.VX_DF_IMAGE_U8), "pyramid")
            else:
                p0 = a.obj(a.vxCreatePyramid(ctx, levels, V.VX_SCALE_PYRAMID_HALF, w, h, V.VX_DF_IMAGE_U8), "pyramid")
                p1 = a.obj(a.vxCreatePyramid(ctx, levels, V.VX_SCALE_PYRAMID_HALF, w, h, V.VX_DF_IMAGE_U8), "pyramid")
            pts = a.obj(a.vxCreateArray(ctx, V.VX_TYPE_KEYPOINT, capacity), "array")
            out = a.obj(a.vxCreateArray(ctx, V.VX_TYPE_KEYPOINT, capacity), "array")
            a.obj(a.vxGaussianPyramidNode(g, i0, p0), "pyramid node")
            a.obj(a.vxGaussianPyramidNode(g, i1, p1), "pyramid node")
            a.obj(a.vxOpticalFlowPyrLKNode(g, p0, p1, pts, pts, out, term, self.s_eps, self.s_iter, self.s_est, window),
                  "optical flow node")
            self.old.append(i0); self.new.append(i1); self.pts.append(pts); self.out.append(out)
            self.pyr.append((p0, p1))
        a.ok(a.vxVerifyGraph(g), "vxVerifyGraph")

    @property
    def inputs(self):
        """Input images in (old, new) pair order."""
        return [i for pair in zip(self.old, self.new) for i in pair]

    def set_inputs(self, pairs, points):
        a = self.api
        for i0, i1, arr, (f1, f2), kp in zip(self.old, self.new, self.pts, pairs, points):
            a.write_plane(i0, f1)
            a.write_plane(i1, f2)
            a.array_set(arr, kp)

    def run(self, frames=None):
        """frames: optional flat list of input images in `inputs` order."""
        if frames is not None:
            for img, f in zip(self.inputs, frames):
                self.api.write_plane(img, f)
        self.api.ok(self.api.vxProcessGraph(self.graph), "vxProcessGraph")

    def results(self):
        return [self.api.array_items(o) for o in self.out]


class WarpRemapGraph:
    """WarpPerspective (bilinear, border CONSTANT `border`; nearest, border UNDEFINED) and
    Remap (bilinear, border CONSTANT `border`; nearest, border UNDEFINED) of one U8 image
    into four non-virtual outputs.  `matrix` is the 3x3 vx_matrix data; `table` the
    (dst_h, dst_w, 2) float source coordinates of the remap."""

    def __init__(self, api: V.OpenVX, ctx, size, matrix, table, src_size=None, border=0, flags: int | None = None):
        a = api
        self.api, self.ctx = api, ctx
        W, H = size
        sW, sH = src_size or size
        dH, dW = table.shape[:2]
        self.graph = a.obj(a.vxCreateGraph(ctx), "graph")
        if flags is not None:
            a.set_optimizer_flags(self.graph, flags)
        self.src = a.obj(a.vxCreateImage(ctx, sW, sH, V.VX_DF_IMAGE_U8), "image")
        self.mat = a.matrix_f32(ctx, np.asarray(matrix, np.float32).reshape(3, 3))
        self.remap = a.obj(a.vxCreateRemap(ctx, sW, sH, dW, dH), "remap")
        t = np.ascontiguousarray(table, np.float32)
        rect = V.vx_rectangle_t(0, 0, dW, dH)
        a.ok(a.vxCopyRemapPatch(self.remap, C.byref(rect), dW * 8, t.ctypes.data, V.VX_TYPE_COORDINATES2DF,
                                V.VX_WRITE_ONLY, V.VX_MEMORY_TYPE_HOST), "vxCopyRemapPatch")
        self.outs = {}
        g = self.graph
        for name, bl, const, kind in (("persp_bilinear_constant", True, True, "p"), ("persp_nearest", False, False, "p"),
                                      ("remap_bilinear_constant", True, True, "r"), ("remap_nearest", False, False, "r")):
            ow, oh = (W, H) if kind == "p" else (dW, dH)
            out = a.obj(a.vxCreateImage(ctx, ow, oh, V.VX_DF_IMAGE_U8), "image")
            interp = V.VX_INTERPOLATION_BILINEAR if bl else V.VX_INTERPOLATION_NEAREST_NEIGHBOR
            if kind == "p":
                node = a.obj(a.vxWarpPerspectiveNode(g, self.src, self.mat, interp, out), "warp node")
            else:
                node = a.obj(a.vxRemapNode(g, self.src, self.remap, interp, out), "remap node")
            if const:
                a.set_border(node, V.VX_BORDER_CONSTANT, border)
            self.outs[name] = out
        a.ok(a.vxVerifyGraph(g), "vxVerifyGraph")

    def run(self, frame=None):
        if frame is not None:
            self.api.write_plane(self.src, frame)
        self.api.ok(self.api.vxProcessGraph(self.graph), "vxProcessGraph")

    def results(self):
        return {k: (self.api.read_plane(v), self.api.valid_region(v)) for k, v in self.outs.items()}


# ---------------------------------------------------------------- config 5 (F32 warp + adjoint)
def cfg5_images(n: int = 32, seed: int = 5, size: int = 1024) -> np.ndarray:
    """(n, size, size) float32: uniform [0, 1) from PCG32 smoothed by a Gaussian, sigma 2
    (separable, truncated at 4 sigma, edges reflected)."""
    r = np.arange(-8, 9, dtype=np.float64)
    k = np.exp(-0.5 * (r / 2.0) ** 2)
    k /= k.sum()
    out = np.empty((n, size, size), np.float32)
    for i in range(n):
        u = uniform01(seed + i, size * size, stream=37).reshape(size, size)
        p = np.pad(u, 8, mode="reflect")
        h = sum(k[j] * p[:, j:j + size] for j in range(17))
        out[i] = sum(k[j] * h[j:j + size, :] for j in range(17)).astype(np.float32)
    return out


def affine_theta(angle_deg: float, scale: float, tx: float, ty: float, size: int) -> np.ndarray:
    """Matrix entries (m00, m01, m10, m11, m20, m21) of the map output -> source that rotates
    by `angle_deg` and scales by `scale` about the image centre, then shifts by (tx, ty)."""
    c = (size - 1) / 2.0
    t = np.deg2rad(angle_deg)
    a, b = scale * np.cos(t), -scale * np.sin(t)
    d, e = scale * np.sin(t), scale * np.cos(t)
    return np.array([a, d, b, e, c + tx - a * c - b * c, c + ty - d * c - e * c], np.float64)


def cfg5_params(n: int = 32, seed: int = 5, size: int = 1024):
    """(ground truth, initial estimate) theta per image: rotation U(+-10 deg), scale U(0.9, 1.1),
    shift U(+-20 px); the estimate perturbs them by U(+-2 deg), U(+-0.02), U(+-3 px)."""
    u = uniform01(seed, 8 * n, stream=41).reshape(n, 8) * 2.0 - 1.0
    gt, init = [], []
    for i in range(n):
        ang, sc, tx, ty = 10 * u[i, 0], 1.0 + 0.1 * u[i, 1], 20 * u[i, 2], 20 * u[i, 3]
        gt.append(affine_theta(ang, sc, tx, ty, size))
        init.append(affine_theta(ang + 2 * u[i, 4], sc + 0.02 * u[i, 5], tx + 3 * u[i, 6], ty + 3 * u[i, 7], size))
    return np.array(gt), np.array(init)


def perspective_theta(affine: np.ndarray, px: float, py: float, size: int) -> np.ndarray:
    """The nine entries (m00, m01, m02, m10, m11, m12, m20, m21, m22) of a perspective map
    output -> source: the affine map `affine` (affine_theta order) with a projective row that
    tilts the plane by px, py (z = 1 + (px (x - c) + py (y - c)) / size about the centre c), so
    z stays near 1 over the image."""
    a, d, b, e, c0, f0 = (float(v) for v in affine)
    c = (size - 1) / 2.0
    g, h = px / size, py / size
    i = 1.0 - g * c - h * c
    # xs = (a x + b y + c0) / z keeps the affine map at the centre, where z = 1
    return np.array([a, d, g, b, e, h, c0, f0, i], np.float64)


def cfg5_perspective_params(n: int = 32, seed: int = 6, size: int = 1024):
    """(ground truth, initial estimate) perspective theta per image: the affine draws of
    cfg5_params plus a tilt U(+-0.05) in each direction; the estimate perturbs the tilt by
    U(+-0.01)."""
    gt_a, init_a = cfg5_params(n, seed, size)
    u = uniform01(seed, 4 * n, stream=45).reshape(n, 4) * 2.0 - 1.0
    gt = [perspective_theta(gt_a[i], 0.05 * u[i, 0], 0.05 * u[i, 1], size) for i in range(n)]
    init = [perspective_theta(init_a[i], 0.05 * u[i, 0] + 0.01 * u[i, 2], 0.05 * u[i, 1] + 0.01 * u[i, 3], size)
            for i in range(n)]
    return np.array(gt), np.array(init)


def cfg5_field(seed: int = 5, size: int = 1024, amplitude: float = 4.0) -> np.ndarray:
    """(size, size, 2) float32 displacement field, smooth, within +-amplitude px."""
    yy, xx = np.meshgrid(np.arange(size, dtype=np.float64), np.arange(size, dtype=np.float64), indexing="ij")
    p = uniform01(seed, 12, stream=43)
    fx = np.sin(2 * np.pi * (p[0] * 3 * xx / size + p[1])) * np.cos(2 * np.pi * (p[2] * 3 * yy / size + p[3]))
    fy = np.cos(2 * np.pi * (p[4] * 3 * xx / size + p[5])) * np.sin(2 * np.pi * (p[6] * 3 * yy / size + p[7]))
    return (amplitude * np.stack([fx, fy], -1)).astype(np.float32)
