#!/usr/bin/env python3
"""Benchmark of the OpenVX/AGO vision-graph path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

One JSON line on stdout (rank 0).  A "step" is one vxProcessGraph of a graph that holds
`frames` independent copies of the workload's vision graph (one per frame), so every step
processes a batch whose inputs + outputs exceed the B200 L2 (126 MB): no L2 flush is needed
between steps.  Default workload: Canny (3x3, L1, 80/100) + Harris (3, 3, k 0.04, 1e-3,
min distance 5) on 3840x2160 U8 synthetic scenes.

* value  -- Mpixels/s with the inputs already resident in HBM: the device time of each
            graph launch (CUDA events the engine records on its own stream), summed over
            K steps.  Mpixels counts the pixels of every input image of the graph (one
            per frame; both frames of a pair for the pyramid/LK workload).
* e2e    -- the same metric through the public OpenVX API with host buffers: per step,
            vxCopyImagePatch(WRITE) of every input frame from pinned host memory,
            vxProcessGraph, vxCopyImagePatch(READ) of every output image and
            vxCopyArrayRange of every output array into host memory; CUDA events bracket
            the K steps (every call is synchronous, so this is also wall time).
* roofline -- HBM roofline of one step (all kernels of the captured graph): algorithmic
            bytes (non-virtual graph inputs + outputs, each read or written once) / the
            step's device time, against MEASURED_PEAKS.json's copy bandwidth.
* cpu_baseline -- the reference AGO CPU library (oracle/_ref, built from the reference's own
            sources) running the same graph on one frame on one host core, bounded sample.

With --gpus N under torchrun every rank processes its own batch (weak scaling; frames are
independent, no data collective), times are max over ranks and value is the job total.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


class Workload:
    name = ""
    desc = ""
    width = height = frames = 0

    def make_frames(self, seed0, n):
        raise NotImplementedError

    def build(self, api, ctx, n, flags=None, host_io=None):
        raise NotImplementedError

    def host_io(self, ins, outs):
        """Image roles of build(host_io=...) for application buffers `ins` (input frames in
        make_frames order) and `outs` (output images in out_images order)."""
        raise NotImplementedError

    def alg_bytes(self, g, n):
        raise NotImplementedError


class GaussChain(Workload):
    name = "gauss_sobel_mag_depth_thresh_1080p"
    desc = ("Gaussian3x3->Sobel3x3->Magnitude->ConvertDepth(SATURATE,0)->Threshold(BINARY,128), 1920x1080 U8, "
            "border UNDEFINED, virtual intermediates")
    width, height, frames = 1920, 1080, 64

    def make_frames(self, seed0, n):
        from mivisionx_b200 import workloads as WL
        return [WL.cfg1_image(seed=seed0 + i, width=self.width, height=self.height) for i in range(n)]

    def build(self, api, ctx, n, flags=None, host_io=None):
        from mivisionx_b200 import workloads as WL
        g = WL.Cfg1Graph(api, ctx, [(self.width, self.height)] * n, flags=flags, host_io=host_io)
        g.out_images, g.out_arrays = g.outputs, []
        return g

    def host_io(self, ins, outs):
        return {"src": [p[0] for p in ins], "dst": [p[0] for p in outs]}

    def alg_bytes(self, g, n):
        return 2.0 * self.width * self.height * n   # 1 B in + 1 B out per pixel


class CannyHarris(Workload):
    name = "canny_harris_4k"
    desc = ("CannyEdgeDetector(3x3, L1, hysteresis 80/100) + HarrisCorners(gradient 3, block 3, k 0.04, "
            "strength 1e-3, min distance 5) on one 3840x2160 U8 scene (gradient + 200 rectangles + N(0,8^2) noise)")
    width, height, frames = 3840, 2160, 16

    def make_frames(self, seed0, n):
        from mivisionx_b200 import workloads as WL
        return [WL.cfg2_scene(seed=seed0 + i, width=self.width, height=self.height) for i in range(n)]

    def build(self, api, ctx, n, flags=None, host_io=None):
        from mivisionx_b200 import workloads as WL
        g = WL.Cfg2Graph(api, ctx, [(self.width, self.height)] * n, flags=flags, host_io=host_io)
        g.out_images, g.out_arrays = g.edges, g.corners
        return g

    def host_io(self, ins, outs):
        return {"src": [p[0] for p in ins], "edge": [p[0] for p in outs]}

    def alg_bytes(self, g, n):
        from mivisionx_b200 import vx as V
        corners = sum(len(g.api.array_items(a)) for a in g.corners)
        # 1 B in (shared by both nodes) + 1 B edge map out per pixel, + 28 B per vx_keypoint_t out
        return 2.0 * self.width * self.height * n + corners * C.sizeof(V.vx_keypoint_t)


class PyramidLK(Workload):
    name = "pyramid_lk_uneven_x64"
    desc = ("Per frame pair: GaussianPyramid(5 levels, scale 0.5) of both frames + OpticalFlowPyrLK(9x9 window, "
            "20 iterations, epsilon 0.01, BOTH) of 2000 seeded uniform points; 64 pairs per step with sizes drawn "
            "by seed from {640x480, 1280x720, 1920x1080, 3840x2160}; frame 2 = frame 1 shifted by U(+-8) px "
            "(bilinear) + N(0, 2^2) noise")
    frames = 64
    points = 2000

    def sizes(self, n):
        from mivisionx_b200 import workloads as WL
        return WL.cfg4_sizes(n, seed=4)

    def make_frames(self, seed0, n):
        from mivisionx_b200 import workloads as WL
        out = []
        for i, (w, h) in enumerate(self.sizes(n)):
            f1, f2, _ = WL.cfg4_pair(seed=seed0 + i, width=w, height=h)
            out += [f1, f2]
        return out

    def build(self, api, ctx, n, flags=None, host_io=None, seed0=1):
        from mivisionx_b200 import workloads as WL
        sizes = self.sizes(n)
        g = WL.Cfg4Graph(api, ctx, sizes, capacity=self.points, flags=flags, host_io=host_io)
        pts = [WL.cfg4_points(seed=seed0 + i, width=w, height=h, n=self.points) for i, (w, h) in enumerate(sizes)]
        for arr, kp in zip(g.pts, pts):
            api.array_set(arr, kp)
        g.out_images, g.out_arrays, g.in_arrays = [], g.out, list(zip(g.pts, pts))
        return g

    def host_io(self, ins, outs):
        return {"old": [p[0] for p in ins[0::2]], "new": [p[0] for p in ins[1::2]]}

    def alg_bytes(self, g, n):
        from mivisionx_b200 import vx as V
        px = sum(g.api.query_image(i)[0] * g.api.query_image(i)[1] for i in g.inputs)
        # pyramid: read level 0 once, write levels 1..4 (sum 4^-k); LK: keypoints in + out
        pyr = px * (1.0 + sum(4.0 ** -k for k in range(1, 5)))
        return pyr + 2.0 * self.points * len(g.out) * C.sizeof(V.vx_keypoint_t)


class ColorGeometry(Workload):
    name = "color_geometry_4k"
    desc = ("ColorConvert RGB->NV12 and RGB->IYUV, ChannelExtract Y (virtual), ScaleImage to 1920x1080 "
            "(bilinear and area), WarpAffine of the bilinear result (nearest and bilinear, border CONSTANT 0; "
            "rotation +-15 deg, scale 0.8-1.2, shift +-50 px) on 3840x2160 RGB frames (8 seeded sinusoids per "
            "channel + U(-10, 10) noise)")
    width, height, frames = 3840, 2160, 8
    distinct = 4            # distinct seeded frames, repeated to fill the step

    def make_frames(self, seed0, n):
        from mivisionx_b200 import workloads as WL
        base = [WL.cfg3_frame(seed=seed0 + i, width=self.width, height=self.height) for i in range(min(n, self.distinct))]
        return [base[i % len(base)] for i in range(n)]

    def build(self, api, ctx, n, flags=None, host_io=None):
        from mivisionx_b200 import workloads as WL
        g = WL.Cfg3Graph(api, ctx, [(self.width, self.height)] * n, flags=flags, host_io=host_io)
        g.out_images, g.out_arrays = g.outputs, []
        return g

    def host_io(self, ins, outs):
        # outputs per frame: nv12, iyuv, scaled bilinear, scaled area, warp nearest, warp bilinear
        per = [outs[i:i + 6] for i in range(0, len(outs), 6)]
        return {"rgb": ins, "nv12": [o[0] for o in per], "iyuv": [o[1] for o in per], "sb": [o[2][0] for o in per],
                "sa": [o[3][0] for o in per], "wn": [o[4][0] for o in per], "wb": [o[5][0] for o in per]}

    def alg_bytes(self, g, n):
        # 3 B RGB in + NV12 1.5 + IYUV 1.5 + four quarter-size U8 outputs (Y plane virtual)
        return 7.0 * self.width * self.height * n


class MotionMask(Workload):
    name = "motion_mask_4k"
    desc = ("Motion mask of frame pairs: AbsDiff(cur, prev) -> Gaussian3x3 -> Threshold(BINARY, 24) -> Dilate3x3 -> "
            "Erode3x3 -> Median3x3, border UNDEFINED, virtual intermediates; 3840x2160 U8 pairs (gradient + 150 "
            "seeded rectangles displaced by up to 12 px + N(0, 3^2) noise per frame)")
    width, height, frames = 3840, 2160, 16     # frame pairs per step

    def make_frames(self, seed0, n):
        from mivisionx_b200 import workloads as WL
        out = []
        for i in range(n):
            out += list(WL.motion_pair(seed=seed0 + i, width=self.width, height=self.height))
        return out

    def build(self, api, ctx, n, flags=None, host_io=None):
        from mivisionx_b200 import workloads as WL
        g = WL.MotionGraph(api, ctx, [(self.width, self.height)] * n, flags=flags, host_io=host_io)
        g.out_images, g.out_arrays = g.outputs, []
        return g

    def host_io(self, ins, outs):
        return {"prev": [p[0] for p in ins[0::2]], "cur": [p[0] for p in ins[1::2]], "dst": [p[0] for p in outs]}

    def alg_bytes(self, g, n):
        return 3.0 * self.width * self.height * n   # two U8 frames in + one U8 mask out per pixel


WORKLOADS = {w.name: w for w in (CannyHarris(), GaussChain(), PyramidLK(), ColorGeometry(), MotionMask())}
DEFAULT_WORKLOAD = CannyHarris.name


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled through NVML every 1 ms while the
    timed region runs (the same counters `nvidia-smi --query-gpu=clocks.sm,...` reads)."""

    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown"}

    def __init__(self, cuda_index: int):
        self.cuda_index, self.rows, self.max_mhz, self.err = cuda_index, [], None, None
        self._stop = threading.Event()

    def _handle(self, nv):
        try:
            import torch
            p = torch.cuda.get_device_properties(self.cuda_index)
            bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
            return nv.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.cuda_index)

    def _run(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = self._handle(nv)
            self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            while not self._stop.is_set():
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                try:
                    rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                except AttributeError:
                    rs = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
                self.rows.append((sm, rs))
                self._stop.wait(0.001)
        except Exception as e:   # NVML unavailable: report it instead of inventing numbers
            self.err = repr(e)

    def __enter__(self):
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()
        t0 = time.time()
        while not self.rows and self.err is None and time.time() - t0 < 2.0:
            time.sleep(0.001)
        self.rows.clear()   # keep only samples taken inside the timed region
        return self

    def __exit__(self, *a):
        n = len(self.rows)
        t0 = time.time()
        while len(self.rows) == n and n == 0 and self.err is None and time.time() - t0 < 0.1:
            time.sleep(0.0005)   # a timed region shorter than one period: its closing sample
        self._stop.set()
        self.t.join(timeout=2)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"], "error": self.err}
        reasons = sorted({n for _, r in self.rows for bit, n in self.REASONS.items() if r & bit})
        return {"sm_mhz": statistics.median(s for s, _ in self.rows), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(self.rows), "source": "NVML, 1 ms period, timed region only"}


def _dist():
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def _max_over_ranks(x: float, ws: int) -> float:
    """Max of a per-rank time over the process group (NCCL on the GPU, gloo on the host)."""
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cpu" if dist.get_backend() == "gloo" else "cuda"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def frame_seed(rank: int) -> int:
    """First frame seed of a rank: every rank processes its own frames (weak scaling, no
    data collective), so whole-job throughput is the sum over ranks."""
    return 1000 * rank + 1


def _barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


# ------------------------------------------------------------------------------------------
# reference CPU path (oracle/_ref: the reference AGO library built from its own sources)
# ------------------------------------------------------------------------------------------
def _ref_worker(wl_name, seed, seconds, max_iters, barrier, queue):
    """Spawned process: build the workload on the reference CPU library, wait for all
    workers, then run frames back to back for `seconds` (at most `max_iters`)."""
    sys.path.insert(0, ROOT)
    import oracle
    from mivisionx_b200 import vx as V
    lib = oracle.ref_lib()
    if lib is None:
        barrier.wait()
        queue.put(None)
        return
    api = V.OpenVX(lib)
    wl = WORKLOADS[wl_name]
    ctx = api.vxCreateContext()
    g = wl.build(api, ctx, 1)
    frames = wl.make_frames(seed, 1)
    g.run(frames)                    # warm-up (first process allocates)
    barrier.wait()
    n, t0 = 0, time.perf_counter()
    while n < max_iters and (time.perf_counter() - t0) < seconds:
        g.run()
        n += 1
    queue.put((n, time.perf_counter() - t0, sum(int(f.shape[0] * f.shape[1]) for f in frames)))


def reference_cpu(wl_name: str, procs: int, seconds: float, max_iters: int = 1 << 30):
    """Aggregate Mpixels/s of `procs` independent reference AGO CPU graphs (one process per
    core: AGO CPU graphs run single-threaded and context creation takes a global lock)."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    barrier, queue = ctx.Barrier(procs), ctx.Queue()
    ps = [ctx.Process(target=_ref_worker, args=(wl_name, 100 + i, seconds, max_iters, barrier, queue)) for i in range(procs)]
    for p in ps:
        p.start()
    res = [queue.get() for _ in ps]
    for p in ps:
        p.join()
    if any(r is None for r in res):
        return None
    frames = sum(r[0] for r in res)
    wall = max(r[1] for r in res)
    return sum(r[0] * r[2] for r in res) / wall / 1e6, wall, frames


def run_reference_arm(a, wl_name):
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    import oracle
    if oracle.ref_lib() is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference AGO library (oracle/_ref) not built"}))
        return 0
    wl = WORKLOADS[wl_name]
    cores = os.cpu_count() or 1
    per_step_s = max(0.5, min(3.0, 120.0 / max(1, a.steps + a.warmup)))
    vals, frames = [], 0
    for s in range(a.warmup + a.steps):
        mpx, _, n = reference_cpu(wl_name, cores, per_step_s)
        if s >= a.warmup:
            vals.append(mpx)
            frames += n
    v = statistics.median(vals)
    print(json.dumps({
        "metric": "Mpixels/s per vision graph", "value": round(v, 2), "unit": "Mpixels/s", "n_gpus": ws,
        "steps": a.steps, "warmup": a.warmup, "impl": "reference", "higher_is_better": True,
        "dtype": "u8", "data": "synthetic (seeded PCG32)",
        "config": {"workload": wl_name, "graph": wl.desc, "seconds_per_step": per_step_s},
        "cpu_baseline": {"value": round(v, 2), "unit": "Mpixels/s", "cores": cores, "kind": "reference",
                         "sample": f"{frames} frames over {a.steps} steps of {per_step_s:.2f} s, {cores} independent "
                                   f"AGO CPU graphs (one process per core)"},
        "e2e": {"value": round(v, 2), "unit": "Mpixels/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
    return 0


# ------------------------------------------------------------------------------------------
def device_value(api, wl, B, plain, steps, warmup, ws, rank, local):
    """Device-resident Mpixels/s of `B` frames of workload `wl` in one graph (fused+batched,
    or the plain one-launch-per-node form), in a context of its own that is released after:
    returns (Mpixels/s over all ranks, ms per step, algorithmic bytes per step, kernels per
    step)."""
    import torch

    from mivisionx_b200 import vx as V
    ctx = api.obj(api.vxCreateContext(), "context")
    api.set_device(ctx, local)
    try:
        frames = wl.make_frames(frame_seed(rank), B)
        g = wl.build(api, ctx, B, flags=V.OPT_NO_FUSION if plain else None)
        g.run(frames)
        alg = wl.alg_bytes(g, B)
        kernels = sum(k for _, k in api.plan(g.graph))
        for _ in range(warmup):
            g.run()
        torch.cuda.synchronize()
        _barrier(ws)
        ms = []
        for _ in range(steps):
            g.run()
            ms.append(api.gpu_ms_last(g.graph))
        torch.cuda.synchronize()
        _barrier(ws)
        ms_step = _max_over_ranks(sum(ms), ws) / steps
        px = sum(int(f.shape[0] * f.shape[1]) for f in frames)
        return px * ws / (ms_step / 1e3) / 1e6, ms_step, alg, kernels
    finally:
        api.vxReleaseContext(C.byref(C.c_void_p(ctx)))


# Configurations of the metric besides the headline one, reported in `per_graph` of the
# default line: each at its own batch, fused and plain, with the roofline fraction and a
# short one-core sample of the reference CPU library.
PER_GRAPH = ["gauss_sobel_mag_depth_thresh_1080p", "color_geometry_4k", "pyramid_lk_uneven_x64", "motion_mask_4k"]


def per_graph_lines(a, api, ws, rank, local):
    peak, peak_kind = _peaks()
    out = {}
    steps, warmup = max(3, min(a.steps, 10)), 3
    for name in PER_GRAPH:
        wl = WORKLOADS[name]
        v, ms, alg, kernels = device_value(api, wl, wl.frames, False, steps, warmup, ws, rank, local)
        vp, msp, _, kp = device_value(api, wl, wl.frames, True, steps, warmup, ws, rank, local)
        achieved = alg / (ms / 1e3) / 1e9
        entry = {"value": round(v, 1), "unit": "Mpixels/s", "ms_per_step": round(ms, 4), "frames_per_step_per_gpu": wl.frames,
                 "kernels_per_step": kernels, "plain": {"value": round(vp, 1), "ms_per_step": round(msp, 4),
                                                        "kernels_per_step": kp, "fused_over_plain": round(v / vp, 2)},
                 "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                              "frac": round(achieved / peak, 4), "peak_kind": peak_kind, "alg_bytes_per_step": alg},
                 "cpu_baseline": None, "graph": wl.desc}
        if rank == 0 and ws == 1 and not a.no_cpu_baseline:
            r = reference_cpu(name, 1, a.per_graph_cpu_seconds)
            if r is not None:
                entry["cpu_baseline"] = {"value": round(r[0], 2), "unit": "Mpixels/s", "cores": 1, "kind": "reference",
                                         "sample": f"{r[2]} runs of the one-unit graph through the reference AGO CPU "
                                                   f"library ({r[1]:.1f} s, 1 core)"}
        out[name] = entry
    # configuration 5: the differentiable F32 warp (no OpenVX graph; no plain form)
    v, ms, launches = diffwarp_value(32, steps, warmup, ws)
    achieved = 12.0 * 32 * 1024 * 1024 / (ms / 1e3) / 1e9
    entry = {"value": round(v, 1), "unit": "Mpixels/s", "ms_per_step": round(ms, 4), "frames_per_step_per_gpu": 32,
             "kernels_per_step": launches / steps, "plain": None,
             "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                          "frac": round(achieved / peak, 4), "peak_kind": peak_kind},
             "cpu_baseline": None, "graph": DIFFWARP_DESC}
    if rank == 0 and ws == 1 and not a.no_cpu_baseline:
        cv, dt, n = _diffwarp_cpu(a.per_graph_cpu_seconds)
        entry["cpu_baseline"] = {"value": round(cv, 2), "unit": "Mpixels/s", "cores": 1, "kind": "port",
                                 "sample": f"{n} x warp + loss + adjoint of one 1024x1024 image in FP64 numpy "
                                           f"({dt:.1f} s, 1 core); the reference has no F32 warp"}
    out[DIFFWARP] = entry
    return out


def run_ours(a, wl_name):
    import numpy as np
    import torch

    from mivisionx_b200 import native
    from mivisionx_b200 import vx as V

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    wl = WORKLOADS[wl_name]
    B = a.frames or wl.frames
    api = V.OpenVX()
    lib = native.agocuda()
    ctx = api.obj(api.vxCreateContext(), "context")
    api.set_device(ctx, local)
    frames = wl.make_frames(frame_seed(rank), B)
    g = wl.build(api, ctx, B, flags=((V.OPT_NO_FUSION if a.plain else 0) | a.opt_flags) or None)
    plan = api.plan(g.graph)
    kernels_per_step = sum(k for _, k in plan)
    # page-locked host buffers, one per image plane: (rows, row bytes)
    def planes(img):
        w, h, fmt = api.query_image(img)
        return [(pi, ph, pw, bpp) for pi, (ph, pw, bpp) in enumerate(V.image_plane_layout(fmt, w, h))]
    in_layout = [planes(i) for i in g.inputs]
    out_layout = [planes(i) for i in g.out_images]
    pin_in = [[torch.from_numpy(np.ascontiguousarray(f).reshape(ph, pw * bpp)).pin_memory()
               for (_, ph, pw, bpp) in lay] for f, lay in zip(frames, in_layout)]
    pin_out = [[torch.empty((ph, pw * bpp), dtype=torch.uint8).pin_memory() for (_, ph, pw, bpp) in lay]
               for lay in out_layout]
    in_arrays = [(arr, torch.from_numpy(kp.view('u1')).pin_memory(), kp.dtype.itemsize, len(kp))
                 for arr, kp in getattr(g, "in_arrays", [])]
    g.run([f for f in frames])
    alg_bytes = wl.alg_bytes(g, B)
    shapes = sorted({f.shape for f in frames})
    frame_desc = f"{shapes[0][1]}x{shapes[0][0]}" if len(shapes) == 1 else "uneven: " + ", ".join(
        f"{sum(1 for f in frames if f.shape == sh)} x {sh[1]}x{sh[0]}" for sh in shapes)

    # ---- device-resident throughput
    for _ in range(a.warmup):
        g.run()
    torch.cuda.synchronize()
    _barrier(ws)
    gpu_ms = []
    with ClockSampler(local) as clk:
        for _ in range(a.steps):
            g.run()
            gpu_ms.append(api.gpu_ms_last(g.graph))
        torch.cuda.synchronize()
    _barrier(ws)
    ms_step = _max_over_ranks(sum(gpu_ms), ws) / a.steps
    px_step = sum(int(f.shape[0] * f.shape[1]) for f in frames)   # input pixels of the first node
    value = px_step * ws / (ms_step / 1e3) / 1e6

    # ---- end to end through the OpenVX API with host buffers
    def patches(img, lay):
        w, h, _ = api.query_image(img)
        out = []
        for (pi, ph, pw, bpp) in lay:
            addr = V.vx_imagepatch_addressing_t()
            addr.dim_x, addr.dim_y, addr.stride_x, addr.stride_y = pw, ph, bpp, pw * bpp
            addr.scale_x = addr.scale_y = 1024
            addr.step_x = addr.step_y = 1
            out.append((pi, V.vx_rectangle_t(0, 0, w, h), addr))
        return out
    in_patch = [patches(i, lay) for i, lay in zip(g.inputs, in_layout)]
    out_patch = [patches(i, lay) for i, lay in zip(g.out_images, out_layout)]
    arr_bufs = [np.zeros(1 << 16, V.KEYPOINT_DTYPE) for _ in g.out_arrays]
    d2h_arrays = [0]

    def read_arrays(graph):
        nbytes = 0
        for arr, buf in zip(graph.out_arrays, arr_bufs):
            n = C.c_size_t(0)
            api.ok(api.vxQueryArray(arr, V.VX_ARRAY_NUMITEMS, C.byref(n), C.sizeof(n)), "numitems")
            if n.value:
                api.ok(api.vxCopyArrayRange(arr, 0, n.value, buf.itemsize, buf.ctypes.data, V.VX_READ_ONLY,
                                            V.VX_MEMORY_TYPE_HOST), "read array")
            nbytes += n.value * buf.itemsize
        d2h_arrays[0] = nbytes

    # (a) images created from the application's page-locked buffers: vxProcessGraph uploads
    # the inputs and downloads the outputs inside its CUDA graph, overlapped with the kernels
    gh = wl.build(api, ctx, B, flags=((V.OPT_NO_FUSION if a.plain else 0) | a.opt_flags) or None,
                  host_io=wl.host_io([[p.numpy() for p in ps] for ps in pin_in],
                                     [[p.numpy() for p in ps] for ps in pin_out]))
    in_arrays_h = [(arr, buf, isz, n) for (arr, kp), (_, buf, isz, n) in
                   zip(getattr(gh, "in_arrays", []), in_arrays)]

    def e2e_step():
        for arr, p, isz, n in in_arrays_h:
            api.ok(api.vxCopyArrayRange(arr, 0, n, isz, p.data_ptr(), V.VX_WRITE_ONLY, V.VX_MEMORY_TYPE_HOST),
                   "write array")
        api.ok(api.vxProcessGraph(gh.graph), "process")
        read_arrays(gh)

    # (b) device images written and read with vxCopyImagePatch around vxProcessGraph
    def e2e_copy_step():
        for img, ps, pat in zip(g.inputs, pin_in, in_patch):
            for p, (pi, rect, addr) in zip(ps, pat):
                api.ok(api.vxCopyImagePatch(img, C.byref(rect), pi, C.byref(addr), p.data_ptr(), V.VX_WRITE_ONLY,
                                            V.VX_MEMORY_TYPE_HOST), "write")
        for arr, p, isz, n in in_arrays:
            api.ok(api.vxCopyArrayRange(arr, 0, n, isz, p.data_ptr(), V.VX_WRITE_ONLY, V.VX_MEMORY_TYPE_HOST),
                   "write array")
        api.ok(api.vxProcessGraph(g.graph), "process")
        for img, ps, pat in zip(g.out_images, pin_out, out_patch):
            for p, (pi, rect, addr) in zip(ps, pat):
                api.ok(api.vxCopyImagePatch(img, C.byref(rect), pi, C.byref(addr), p.data_ptr(), V.VX_READ_ONLY,
                                            V.VX_MEMORY_TYPE_HOST), "read")
        read_arrays(g)

    def time_e2e(step):
        for _ in range(a.warmup):
            step()
        torch.cuda.synchronize()
        _barrier(ws)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(a.steps):
            step()
        e1.record()
        torch.cuda.synchronize()
        return _max_over_ranks(e0.elapsed_time(e1) / a.steps, ws)

    e2e_copy_ms = time_e2e(e2e_copy_step)
    e2e_ms = time_e2e(e2e_step)
    e2e = px_step * ws / (e2e_ms / 1e3) / 1e6
    e2e_copy = px_step * ws / (e2e_copy_ms / 1e3) / 1e6

    # the same workload in the plain one-launch-per-node form (the metric's "batched vs plain")
    plain = None
    if not a.plain:
        vp, msp, _, kp = device_value(api, wl, B, True, a.steps, a.warmup, ws, rank, local)
        plain = {"value": round(vp, 1), "unit": "Mpixels/s", "ms_per_step": round(msp, 4), "kernels_per_step": kp,
                 "fused_over_plain": round(value / vp, 2)}
    per_graph = per_graph_lines(a, api, ws, rank, local) if a.per_graph else None

    peak, peak_kind = _peaks()
    achieved = alg_bytes / (ms_step / 1e3) / 1e9
    traffic, traffic_note = None, None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        t = json.load(open(tp)).get(wl_name) or {}
        traffic, traffic_note = t.get("bytes_per_step"), t.get("note")
    if rank == 0:
        cpu = None
        if ws == 1 and not a.no_cpu_baseline:
            r = reference_cpu(wl_name, 1, a.cpu_seconds)
            if r is not None:
                cpu = {"value": round(r[0], 2), "unit": "Mpixels/s", "cores": 1, "kind": "reference",
                       "sample": f"{r[2]} runs of the one-unit graph ({frame_desc.split(',')[0]} class) through "
                                 f"the reference AGO CPU library ({r[1]:.1f} s of CPU work, 1 core)"}
        print(json.dumps({
            "metric": "Mpixels/s per vision graph", "value": round(value, 1), "unit": "Mpixels/s", "n_gpus": ws,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms_step, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded PCG32)",
            "config": {"workload": wl_name, "graph": wl.desc, "frames_per_step_per_gpu": B, "frame": frame_desc,
                       "l2": "inputs+outputs per step exceed the 126 MB L2 (no flush needed)",
                       "plan": [n for n, _ in plan], "plan_form": "plain" if a.plain else "fused+batched", "parallelism": f"replicas x{ws} (frames sharded, no collective)"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic, "traffic_note": traffic_note,
                         "peak_kind": peak_kind,
                         "alg_bytes_per_launch": alg_bytes, "kernel": f"one step: {kernels_per_step} kernels in one CUDA graph"},
            "e2e": {"value": round(e2e, 1), "unit": "Mpixels/s",
                    "h2d_bytes_per_step": sum(p.numel() for ps in pin_in for p in ps) +
                                          sum(isz * n for _, _, isz, n in in_arrays),
                    "d2h_bytes_per_step": sum(p.numel() for ps in pin_out for p in ps) + d2h_arrays[0],
                    "api": "images from page-locked application buffers (vxCreateImageFromHandle HOST) + "
                           "vxProcessGraph (copies inside its CUDA graph) + vxCopyArrayRange for arrays",
                    "ms_per_step": round(e2e_ms, 4),
                    "copy_patch_value": round(e2e_copy, 1),
                    "copy_patch_api": "vxCopyImagePatch in, vxProcessGraph, vxCopyImagePatch out"},
            "gpu_launches": kernels_per_step * a.steps,
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
            "plain": plain,
            "per_graph": per_graph,
        }))
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------------------------------------------
# Differentiable F32 WarpAffine: one step = warp + L2 loss + adjoint for a batch of images
# (the fused kernel of mivisionx_b200.diffwarp).  No OpenVX graph: the reference has no F32
# warp, so its CPU leg is the FP64 port (oracle/diffwarp_f64.py).
# ------------------------------------------------------------------------------------------
DIFFWARP = "diffwarp_affine_32x1024"
DIFFWARP_DESC = ("F32 bilinear WarpAffine (border CONSTANT 0) + L2 loss to the image warped by the ground truth + "
                 "adjoint (d/dsrc, d/dtheta) in one pass; 32 images 1024x1024, uniform [0,1] smoothed by a Gaussian "
                 "(sigma 2); theta = seeded estimate (GT rotation +-10 deg, scale 0.9-1.1, shift +-20 px, perturbed by "
                 "+-2 deg, +-0.02, +-3 px)")


def _diffwarp_inputs(n, size):
    import numpy as np

    from mivisionx_b200 import workloads as WL
    imgs = WL.cfg5_images(n, size=size)
    gt, init = WL.cfg5_params(n, size=size)
    return imgs, gt.astype(np.float32), init.astype(np.float32)


def _diffwarp_cpu(seconds, size=1024):
    """FP64 port on one host core: warp + loss + adjoint of one image, repeated for ~seconds."""
    from oracle import diffwarp_f64 as D
    imgs, gt, init = _diffwarp_inputs(1, size)
    img = imgs[0].astype("float64")
    tgt = D.warp_affine(img, gt[0].astype("float64"))
    n, t0 = 0, time.perf_counter()
    while n == 0 or time.perf_counter() - t0 < seconds:
        out = D.warp_affine(img, init[0].astype("float64"))
        D.warp_affine_adjoint(img, init[0].astype("float64"), 2 * (out - tgt))
        n += 1
    dt = time.perf_counter() - t0
    return n * size * size / dt / 1e6, dt, n


def diffwarp_value(N, steps, warmup, ws, S=1024):
    """Device time of the fused warp + L2 + adjoint step on N images: (Mpixels/s over all
    ranks, ms per step, launches in the timed steps)."""
    import torch

    from mivisionx_b200 import diffwarp, native
    imgs, gt, init = _diffwarp_inputs(N, S)
    d_img = torch.from_numpy(imgs).cuda()
    d_gt, d_th = torch.from_numpy(gt).cuda(), torch.from_numpy(init).cuda()
    d_tgt = diffwarp.warp_affine(d_img, d_gt)
    gsrc = torch.zeros_like(d_img)
    acc = torch.zeros((N, 7), dtype=torch.float64, device="cuda")
    lib = native.agocuda()
    stream = torch.cuda.current_stream()
    for _ in range(warmup):
        diffwarp.warp_affine_l2_step(d_img, d_th, d_tgt, gsrc=gsrc, acc=acc)
    torch.cuda.synchronize()
    _barrier(ws)
    n0 = lib.agocuda_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        diffwarp.warp_affine_l2_step(d_img, d_th, d_tgt, gsrc=gsrc, acc=acc)
    e1.record(stream)
    torch.cuda.synchronize()
    launches = lib.agocuda_launch_count() - n0
    ms = _max_over_ranks(e0.elapsed_time(e1) / steps, ws)
    return N * S * S * ws / (ms / 1e3) / 1e6, ms, launches


def run_diffwarp(a):
    import numpy as np
    import torch

    from mivisionx_b200 import diffwarp, native
    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    N, S = a.frames or 32, 1024
    imgs, gt, init = _diffwarp_inputs(N, S)
    d_img = torch.from_numpy(imgs).cuda()
    d_gt, d_th = torch.from_numpy(gt).cuda(), torch.from_numpy(init).cuda()
    d_tgt = diffwarp.warp_affine(d_img, d_gt)            # target: the image warped by the ground truth
    gsrc = torch.zeros_like(d_img)
    acc = torch.zeros((N, 7), dtype=torch.float64, device="cuda")
    lib = native.agocuda()
    stream = torch.cuda.current_stream()

    def step():
        diffwarp.warp_affine_l2_step(d_img, d_th, d_tgt, gsrc=gsrc, acc=acc)

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    _barrier(ws)
    n0 = lib.agocuda_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(a.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    launches = lib.agocuda_launch_count() - n0
    ms_step = _max_over_ranks(e0.elapsed_time(e1) / a.steps, ws)
    px = N * S * S
    value = px * ws / (ms_step / 1e3) / 1e6

    # end to end: images, targets and theta from pinned host memory, loss + theta gradients back
    h_img = torch.from_numpy(imgs).pin_memory()
    h_tgt = d_tgt.cpu().pin_memory()
    h_th = torch.from_numpy(init).pin_memory()
    h_out = torch.empty((N, 7), dtype=torch.float64).pin_memory()

    def e2e_step():
        d_img.copy_(h_img, non_blocking=True)
        d_tgt.copy_(h_tgt, non_blocking=True)
        d_th.copy_(h_th, non_blocking=True)
        step()
        h_out.copy_(acc, non_blocking=True)
        torch.cuda.current_stream().synchronize()

    for _ in range(a.warmup):
        e2e_step()
    _barrier(ws)
    e0.record(stream)
    for _ in range(a.steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = _max_over_ranks(e0.elapsed_time(e1) / a.steps, ws)
    peak, peak_kind = _peaks()
    alg_bytes = 12.0 * px           # read src + target, write d/dsrc (4 B each per pixel)
    achieved = alg_bytes / (ms_step / 1e3) / 1e9
    if rank == 0:
        cpu = None
        if ws == 1 and not a.no_cpu_baseline:
            v, dt, n = _diffwarp_cpu(a.cpu_seconds)
            cpu = {"value": round(v, 2), "unit": "Mpixels/s", "cores": 1, "kind": "port",
                   "sample": f"{n} x warp + loss + adjoint of one 1024x1024 image in FP64 numpy ({dt:.1f} s, 1 core); "
                             "the reference has no F32 warp"}
        print(json.dumps({
            "metric": "Mpixels/s per vision graph", "value": round(value, 1), "unit": "Mpixels/s", "n_gpus": ws,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms_step, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded PCG32)",
            "config": {"workload": DIFFWARP, "graph": DIFFWARP_DESC, "images_per_step_per_gpu": N, "image": f"{S}x{S}",
                       "l2": "inputs (128 MB src + 128 MB target) exceed the 126 MB L2 (no flush needed)",
                       "parallelism": f"replicas x{ws} (images sharded, no collective)"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": None, "peak_kind": peak_kind,
                         "alg_bytes_per_launch": alg_bytes, "kernel": "k_warp_affine_f32<fused L2>, 1 launch per step"},
            "e2e": {"value": round(px * ws / (e2e_ms / 1e3) / 1e6, 1), "unit": "Mpixels/s",
                    "h2d_bytes_per_step": 2 * 4 * px + N * 6 * 4, "d2h_bytes_per_step": N * 7 * 8},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }))
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_diffwarp_reference(a):
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    per_step = max(0.5, min(3.0, 120.0 / max(1, a.steps + a.warmup)))
    vals = []
    with mp.get_context("spawn").Pool(cores) as pool:
        for s in range(a.warmup + a.steps):
            r = pool.map(_diffwarp_cpu, [per_step] * cores)
            if s >= a.warmup:
                vals.append(sum(v for v, _, _ in r))
    v = statistics.median(vals)
    print(json.dumps({
        "metric": "Mpixels/s per vision graph", "value": round(v, 2), "unit": "Mpixels/s", "n_gpus": ws,
        "steps": a.steps, "warmup": a.warmup, "impl": "reference", "higher_is_better": True, "dtype": "f64",
        "data": "synthetic (seeded PCG32)", "config": {"workload": DIFFWARP, "graph": DIFFWARP_DESC},
        "cpu_baseline": {"value": round(v, 2), "unit": "Mpixels/s", "cores": cores, "kind": "port",
                         "sample": f"{cores} processes x {per_step:.2f} s per step of FP64 warp + loss + adjoint "
                                   "(the reference has no F32 warp)"},
        "e2e": {"value": round(v, 2), "unit": "Mpixels/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
    return 0


def spawn_ranks(n, argv):
    """`--gpus N` without torchrun: start N local ranks of this script, one per GPU, with the
    torchrun environment (127.0.0.1 rendezvous); rank 0 prints the line.  Returns the worst
    exit status."""
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    procs = []
    for r in range(n):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(n), LOCAL_WORLD_SIZE=str(n),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, os.path.abspath(__file__)] + list(argv), env=env))
    rcs = [p.wait() for p in procs]
    return max(rcs, key=abs)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS) + [DIFFWARP])
    ap.add_argument("--frames", type=int, default=0, help="frames per step per GPU (default: the workload's)")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--opt-flags", type=lambda v: int(v, 0), default=0,
                    help="extra VX_GRAPH_ATTRIBUTE_AMD_OPTIMIZER_FLAGS bits for the timed graph (e.g. 0x80000: "
                         "pixel chains stage tiles with cp.async instead of TMA)")
    ap.add_argument("--plain", action="store_true",
                    help="run the one-launch-per-node plan (the unfused, unbatched comparison form)")
    ap.add_argument("--no-per-graph", dest="per_graph", action="store_false",
                    help="leave out the other configurations (per_graph) of the default line")
    ap.add_argument("--per-graph-cpu-seconds", type=float, default=3.0)
    a = ap.parse_args(argv)
    if a.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return spawn_ranks(a.gpus, argv if argv is not None else sys.argv[1:])
    if a.workload != DEFAULT_WORKLOAD or a.plain:
        a.per_graph = False
    if a.workload == DIFFWARP:
        if a.impl == "ours":
            a.warmup = max(a.warmup, 3)
            return run_diffwarp(a)
        return run_diffwarp_reference(a)
    if a.impl == "ours":
        a.warmup = max(a.warmup, 3)
        return run_ours(a, a.workload)
    return run_reference_arm(a, a.workload)


if __name__ == "__main__":
    sys.exit(main())
