"""Build recipe for the native libraries of mivisionx_b200 (in-tree, sm_100a only).

    python -m mivisionx_b200.build           # incremental
    python -m mivisionx_b200.build --clean   # from scratch

Produces
  mivisionx_b200/lib/libagocuda.so  -- CUDA kernels behind include/agocuda.h (C ABI)
  mivisionx_b200/lib/libopenvx.so   -- the OpenVX 1.3 / AGO host engine (C++), linked
                                       against libagocuda.so (rpath $ORIGIN)
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
ENGINE = os.path.join(CSRC, "engine")
INCLUDE = os.path.join(ROOT, "include")
LIBDIR = os.path.join(PKG, "lib")
OBJDIR = os.path.join(PKG, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CUDA_HOME = os.path.dirname(os.path.dirname(NVCC))

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: the reference's float kernels are strictly multiply-then-add (SSE, no FMA);
# contraction would change results in the last bit.
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC",
                     "-Xptxas", "-warn-spills", f"-I{INCLUDE}", f"-I{CSRC}"]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall", "-Wno-unused-function", f"-I{INCLUDE}", f"-I{ENGINE}",
             f"-I{CUDA_HOME}/include", "-ffp-contract=off"]


def _sources(d, exts):
    if not os.path.isdir(d):
        return []
    return sorted(os.path.join(d, f) for f in os.listdir(d) if f.endswith(exts))


def _headers():
    hs = []
    for d in (INCLUDE, CSRC, ENGINE):
        hs += _sources(d, (".h", ".cuh", ".hpp"))
    return hs


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout)
    return r.stdout


def _compile(src, verbose=False):
    obj = os.path.join(OBJDIR, os.path.basename(src) + ".o")
    if not _stale(obj, [src] + _headers()):
        return obj, ""
    if src.endswith(".cu"):
        cmd = [NVCC] + NVCC_FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-c", src, "-o", obj]
    else:
        cmd = ["g++"] + CXX_FLAGS + ["-c", src, "-o", obj]
    out = _run(cmd)
    return obj, out


def build(verbose: bool = False, clean: bool = False) -> None:
    if clean:
        shutil.rmtree(OBJDIR, ignore_errors=True)
        shutil.rmtree(LIBDIR, ignore_errors=True)
    os.makedirs(OBJDIR, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    cu = _sources(CSRC, (".cu",))
    eng = _sources(ENGINE, (".cpp",))
    with cf.ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose), cu + eng))
    if verbose:
        for _, out in results:
            if out.strip():
                print(out)
    cu_objs = [o for (o, _), s in zip(results, cu + eng) if s.endswith(".cu")]
    eng_objs = [o for (o, _), s in zip(results, cu + eng) if s.endswith(".cpp")]
    agocuda = os.path.join(LIBDIR, "libagocuda.so")
    if _stale(agocuda, cu_objs):
        # shared cudart: the engine and the kernels must see one runtime (current device,
        # streams) -- a static copy per library would keep its own device selection
        _run([NVCC] + ARCH + ["-shared", "-cudart", "shared", "-o", agocuda] + cu_objs +
             ["-lcuda", "-Xlinker", f"-rpath,{CUDA_HOME}/lib64"])
    if eng_objs:
        openvx = os.path.join(LIBDIR, "libopenvx.so")
        if _stale(openvx, eng_objs + [agocuda]):
            _run(["g++", "-shared", "-o", openvx] + eng_objs +
                 [f"-L{LIBDIR}", "-lagocuda", f"-L{CUDA_HOME}/lib64", "-lcudart", "-ldl", "-lpthread",
                  "-Wl,-rpath,$ORIGIN", f"-Wl,-rpath,{CUDA_HOME}/lib64", "-Wl,--no-undefined"])


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    build(verbose=a.verbose, clean=a.clean)
    print("built:", ", ".join(sorted(os.listdir(LIBDIR))))


if __name__ == "__main__":
    sys.exit(main())
