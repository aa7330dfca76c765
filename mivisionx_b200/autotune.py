"""Autotuner for the batched stencil kernels: picks, per kernel and frame size, the launch
shape the engine uses and writes the table vxVerifyGraph reads (mivisionx_b200/tune/b200.json,
or the path in AGO_B200_TUNE_FILE).

    python -m mivisionx_b200.autotune [--out PATH] [--quick]

For every (kernel, frame size) it times each candidate shape on a batch of device-resident
frames larger than the B200's L2 (126 MB), with CUDA events on the launching stream (2
warm-up launches, the median of 7), and keeps the fastest.  Every candidate's output must be
byte-identical to the default form's output on the same batch, or the candidate is dropped.

Kernels and their parameters (the `params` of a table entry):
* fused_GaussSobelMagDepthThresh_tma (the configuration-1 chain, TMA-staged: the default
  form): [rows per warp, warps per block].
* fused_GaussSobelMagDepthThresh (the configuration-1 chain, register form, used with the
  no-TMA optimizer flag): [rows per thread, warps per block, resident blocks per SM,
  persistent]; persistent = 0 is the one-block-per-tile grid.
* ScaleGaussianHalf_U8_U8_5x5 (a Gaussian pyramid level): [threads per block, rows per
  thread, resident blocks per SM, persistent].
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(HERE, "tune", "b200.json")
L2_BYTES = 126 << 20

u32, i32, vp = C.c_uint32, C.c_int32, C.c_void_p


def _lib():
    from . import native
    L = native.agocuda()
    sigs = {
        "agocuda_fused_GaussSobelMagDepthThresh": (C.c_int, [vp, vp, u32, u32, u32, i32, i32]),
        "agocuda_fused_GaussSobelMagDepthThresh_tiles": (u32, [u32, u32, u32, u32]),
        "agocuda_fused_GaussSobelMagDepthThresh_persistent": (C.c_int, [vp, vp, u32, vp, vp, u32, u32, u32, i32, i32]),
        "agocuda_fused_ScaleGaussianHalf_batch": (C.c_int, [vp, vp, u32, u32]),
        "agocuda_ScaleGaussianHalf_tiles": (u32, [u32, u32]),
        "agocuda_ScaleGaussianHalf_tiles_shape": (u32, [u32, u32, u32, u32]),
        "agocuda_fused_ScaleGaussianHalf_persistent": (C.c_int, [vp, vp, u32, u32, vp, u32, u32, u32]),
        "agocuda_fused_GaussSobelMagDepthThresh_tensor_maps_size": (C.c_size_t, [u32]),
        "agocuda_fused_GaussSobelMagDepthThresh_tensor_maps_shape": (C.c_int, [vp, u32, u32, u32, vp, C.c_size_t]),
        "agocuda_fused_GaussSobelMagDepthThresh_tma_shape": (C.c_int, [vp, vp, vp, u32, u32, u32, i32, i32, u32, u32, vp]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(L, name)
        fn.restype, fn.argtypes = res, args
    return L


def _time(fn, stream, warmup=2, reps=7):
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1) * 1e3)
    return statistics.median(ts)


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what} returned {rc}")


# ------------------------------------------------------------------ config-1 chain
def tune_chain(L, W, H, quick=False):
    import torch

    from . import native
    n = max(2, int(2 * L2_BYTES // (2 * W * H)) + 1)          # inputs + outputs above twice the L2
    stride = (W + 63) // 64 * 64
    src = torch.randint(0, 256, (n, H, stride), dtype=torch.uint8, device="cuda")
    dst = torch.zeros((n, H, stride), dtype=torch.uint8, device="cuda")
    frames = (native.AgoFrame * n)()
    for i in range(n):
        frames[i] = native.AgoFrame(src[i].data_ptr(), dst[i].data_ptr(), W, H, stride, stride, 0, W - W % 16)
    fbytes = bytes(frames)
    dframes = torch.frombuffer(bytearray(fbytes), dtype=torch.uint8).cuda()
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    # default (grid) form: the reference output and time
    grid = lambda: _check(L.agocuda_fused_GaussSobelMagDepthThresh(sp, dframes.data_ptr(), n, W, H, 0, 128), "chain")
    grid()
    torch.cuda.synchronize()
    want = dst.clone()
    results = [([18, 4, 0, 0], _time(grid, stream))]
    regs_warps = 25                                          # resident warps per SM at 80 registers a thread
    rows_set = (12, 18) if quick else (6, 12, 18, 24)
    for rows in rows_set:
        for warps in (2, 4, 8):
            tiles = L.agocuda_fused_GaussSobelMagDepthThresh_tiles(W, H, rows, warps)
            if not tiles:
                continue
            pre = np.zeros(n + 4, np.uint32)
            pre[1:n + 1] = np.cumsum([tiles] * n)
            dpre = torch.from_numpy(pre.view(np.int32)).cuda()
            queue = dpre.data_ptr() + 4 * ((n + 2) & ~1)
            for bps in sorted({b for b in (1, 2, 3, 4, 6, 8, 12) if b * warps <= regs_warps}):
                def run(rows=rows, warps=warps, bps=bps, dpre=dpre, queue=queue):
                    _check(L.agocuda_fused_GaussSobelMagDepthThresh_persistent(sp, dframes.data_ptr(), n, dpre.data_ptr(),
                                                                               queue, rows, warps, bps, 0, 128), "persistent")
                dst.zero_()
                run()
                torch.cuda.synchronize()
                if not torch.equal(dst, want):
                    continue
                results.append(([rows, warps, bps, 1], _time(run, stream)))
    return results, n


TMA_CHAIN_SHAPES = [(36, 2), (18, 1), (24, 1), (36, 1), (48, 1), (18, 2), (24, 2), (48, 2), (18, 4), (24, 4), (36, 4)]


def tune_chain_tma(L, W, H, quick=False):
    """The TMA-staged chain: every tile shape against the register grid form's output."""
    import torch

    from . import native
    n = max(2, int(2 * L2_BYTES // (2 * W * H)) + 1)
    stride = (W + 255) // 256 * 256
    src = torch.randint(0, 256, (n, H, stride), dtype=torch.uint8, device="cuda")
    dst = torch.zeros((n, H, stride), dtype=torch.uint8, device="cuda")
    frames = (native.AgoFrame * n)()
    for i in range(n):
        frames[i] = native.AgoFrame(src[i].data_ptr(), dst[i].data_ptr(), W, H, stride, stride, 0, W - W % 16)
    dframes = torch.frombuffer(bytearray(bytes(frames)), dtype=torch.uint8).cuda()
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    _check(L.agocuda_fused_GaussSobelMagDepthThresh(sp, dframes.data_ptr(), n, W, H, 0, 128), "chain")
    torch.cuda.synchronize()
    want = dst.clone()
    mb = L.agocuda_fused_GaussSobelMagDepthThresh_tensor_maps_size(n)
    results = []
    for rows, warps in (TMA_CHAIN_SHAPES[:4] if quick else TMA_CHAIN_SHAPES):
        host = np.zeros(mb + 64, np.uint8)
        off = (-host.ctypes.data) % 64
        _check(L.agocuda_fused_GaussSobelMagDepthThresh_tensor_maps_shape(frames, n, rows, warps, host.ctypes.data + off, mb),
               "tensor maps")
        dmaps = torch.from_numpy(host[off:off + mb].copy()).cuda()

        def run(rows=rows, warps=warps, dmaps=dmaps):
            _check(L.agocuda_fused_GaussSobelMagDepthThresh_tma_shape(sp, dframes.data_ptr(), dmaps.data_ptr(), n, W, H, 0,
                                                                      128, rows, warps, status.data_ptr()), "tma")
        dst.zero_()
        run()
        torch.cuda.synchronize()
        if not torch.equal(dst[:, 2:H - 2, 2:W - 2], want[:, 2:H - 2, 2:W - 2]) or int(status.item()):
            continue
        results.append(([rows, warps], _time(run, stream)))
    return results, n


# ------------------------------------------------------------------ pyramid level
def tune_half(L, W, H, quick=False):
    """W x H: the source image of the level (the output is ceil(W/2) x ceil(H/2))."""
    import torch

    from . import native
    dW, dH = (W + 1) // 2, (H + 1) // 2
    n = max(2, int(2 * L2_BYTES // (W * H + dW * dH)) + 1)
    ss, ds = (W + 63) // 64 * 64, (dW + 63) // 64 * 64
    src = torch.randint(0, 256, (n, H, ss), dtype=torch.uint8, device="cuda")
    dst = torch.zeros((n, dH, ds), dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream

    def jobs_for(tiles_per):
        jobs = (native.HalfJob * n)()
        for i in range(n):
            jobs[i] = native.HalfJob(src[i].data_ptr(), dst[i].data_ptr(), W, H, ss, dW, dH, ds, i * tiles_per, 0)
        return torch.frombuffer(bytearray(bytes(jobs)), dtype=torch.uint8).cuda()

    t0 = L.agocuda_ScaleGaussianHalf_tiles(dW, dH)
    dj0 = jobs_for(t0)
    grid = lambda: _check(L.agocuda_fused_ScaleGaussianHalf_batch(sp, dj0.data_ptr(), n, n * t0), "half")
    grid()
    torch.cuda.synchronize()
    want = dst.clone()
    results = [([32, 8, 0, 0], _time(grid, stream))]
    regs_threads = 595                                       # resident threads per SM at 110 registers a thread
    queue = torch.zeros(2, dtype=torch.int32, device="cuda")
    for threads in ((32, 64) if quick else (32, 64, 128)):
        for rows in (2, 4, 8):
            tp = L.agocuda_ScaleGaussianHalf_tiles_shape(dW, dH, threads, rows)
            if not tp:
                continue
            dj = jobs_for(tp)
            for bps in sorted({b for b in (1, 2, 4, 8, 16) if b * threads <= regs_threads}):
                def run(threads=threads, rows=rows, bps=bps, dj=dj, tp=tp):
                    _check(L.agocuda_fused_ScaleGaussianHalf_persistent(sp, dj.data_ptr(), n, n * tp, queue.data_ptr(),
                                                                        threads, rows, bps), "half persistent")
                dst.zero_()
                run()
                torch.cuda.synchronize()
                if not torch.equal(dst, want):
                    continue
                results.append(([threads, rows, bps, 1], _time(run, stream)))
    return results, n


CHAIN_SHAPES = [(640, 480), (1280, 720), (1920, 1080), (3840, 2160)]
HALF_SHAPES = [(3840, 2160), (1920, 1080), (1280, 720), (960, 540), (640, 480), (480, 270), (320, 240), (240, 135)]


def run(out=DEFAULT_OUT, quick=False, log=print, only=None):
    """Tune every kernel (or only the named ones, keeping the other entries of the table at
    `out`) and write the table."""
    import torch
    L = _lib()
    entries = []
    if only and os.path.exists(out):
        entries = [e for e in json.load(open(out))["entries"] if e["kernel"] not in only]
    for kernel, shapes, fn, px_of in (("fused_GaussSobelMagDepthThresh_tma", CHAIN_SHAPES, tune_chain_tma, lambda w, h: w * h),
                                      ("fused_GaussSobelMagDepthThresh", CHAIN_SHAPES, tune_chain, lambda w, h: w * h),
                                      ("ScaleGaussianHalf_U8_U8_5x5", HALF_SHAPES, tune_half,
                                       lambda w, h: ((w + 1) // 2) * ((h + 1) // 2))):
        if only and kernel not in only:
            continue
        for (W, H) in shapes:
            res, n = fn(L, W, H, quick)
            default_us = res[0][1]                            # the first candidate is the default shape
            res.sort(key=lambda r: r[1])
            best, us = res[0]
            grid_us = next((t for p, t in res if len(p) == 4 and p[3] == 0), default_us)
            key_w, key_h = (W, H) if kernel.startswith("fused") else ((W + 1) // 2, (H + 1) // 2)
            entries.append({"kernel": kernel, "width": key_w, "height": key_h, "params": best,
                            "us_per_launch": round(us, 2), "frames": n,
                            "gpx_per_s": round(px_of(W, H) * n / us / 1e3, 1),
                            "default_us_per_launch": round(default_us, 2), "candidates": len(res)})
            if len(best) == 4:
                entries[-1]["grid_us_per_launch"] = round(grid_us, 2)
            log(f"{kernel} {key_w}x{key_h}: {best} {us:.1f} us (default {default_us:.1f} us, {len(res)} candidates)")
    table = {"device": torch.cuda.get_device_name(0), "sm_count": torch.cuda.get_device_properties(0).multi_processor_count,
             "generated_by": "python -m mivisionx_b200.autotune", "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()),
             "entries": entries}
    os.makedirs(os.path.dirname(out), exist_ok=True)
    with open(out, "w") as f:
        json.dump(table, f, indent=1)
    return table


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.environ.get("AGO_B200_TUNE_FILE") or DEFAULT_OUT)
    ap.add_argument("--quick", action="store_true", help="a smaller search (for tests)")
    ap.add_argument("--only", action="append", help="tune this kernel only (repeatable); the table's other entries stay")
    a = ap.parse_args(argv)
    run(a.out, a.quick, only=a.only)


if __name__ == "__main__":
    main()
