"""include/agovx.h must be ABI-identical to the Khronos/AMD headers the reference ships:
every enum constant and struct size declared in agovx.h is compiled once against agovx.h
and once against the reference's VX/vx.h + vx_ext_amd.h, and the values must agree.
Also checks that the built libraries export every function the headers declare."""
import os
import re
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HDR = os.path.join(ROOT, "include", "agovx.h")
AGOCUDA_H = os.path.join(ROOT, "include", "agocuda.h")
REF_INC = "/root/reference/amd_openvx/openvx/include"

STRUCTS = ["vx_imagepatch_addressing_t", "vx_perf_t", "vx_keypoint_t", "vx_rectangle_t", "vx_coordinates2df_t",
           "vx_pixel_value_t", "vx_border_t", "AgoTargetAffinityInfo", "AgoGraphPerfInternalInfo",
           "AgoImageFormatDescription"]


def _enum_names():
    src = open(HDR).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = set()
    for body in re.findall(r"enum\s*\w*\s*\{(.*?)\}", src, flags=re.S):
        for m in re.finditer(r"\b((?:VX|AGO)_[A-Z0-9_a-z]+)\s*=", body):
            names.add(m.group(1))
    return sorted(names)


def _run(prog, incs):
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "p.cpp")   # the reference's vx_ext_amd.h needs C++
        exe = os.path.join(d, "p")
        open(c, "w").write(prog)
        subprocess.run(["g++", "-w", "-o", exe, c] + [f"-I{i}" for i in incs], check=True)
        return subprocess.run([exe], check=True, capture_output=True, text=True).stdout


@pytest.mark.skipif(not os.path.isdir(REF_INC), reason="reference headers not present")
def test_enums_and_structs_match_reference():
    names = _enum_names()
    assert len(names) > 150
    body = "".join(f'printf("{n} %ld\\n", (long)({n}));\n' for n in names)
    body += "".join(f'printf("sizeof_{s} %zu\\n", sizeof({s}));\n' for s in STRUCTS)
    ours = _run('#include <stdio.h>\n#include "agovx.h"\nint main(){' + body + "return 0;}", [os.path.dirname(HDR)])
    ref = _run('#include <stdio.h>\n#include <VX/vx.h>\n#include <VX/vx_compatibility.h>\n#include <vx_ext_amd.h>\n'
               'int main(){' + body + "return 0;}", [REF_INC])
    assert ours == ref


def _declared(path, prefix):
    """Functions the header declares (typedefs of function pointers are not symbols)."""
    src = re.sub(r"/\*.*?\*/", "", open(path).read(), flags=re.S)
    src = re.sub(r"typedef[^;]*;", "", src)
    return sorted(set(re.findall(r"\b(" + prefix + r"\w+)\s*\(", src)))


def test_libraries_export_declared_symbols():
    from mivisionx_b200 import native
    if not (os.path.exists(native.AGOCUDA_SO) and os.path.exists(native.OPENVX_SO)):
        pytest.skip("native libraries not built")
    import ctypes
    ago = ctypes.CDLL(native.AGOCUDA_SO)
    for name in _declared(AGOCUDA_H, "agocuda_"):
        assert hasattr(ago, name), name
    ovx = native.openvx()
    for name in _declared(HDR, "vx"):
        assert hasattr(ovx, name), name


def test_ctypes_mirrors_match_agocuda_structs():
    """The ctypes mirrors in mivisionx_b200/native.py have the C layout of include/agocuda.h."""
    import ctypes
    from mivisionx_b200 import native
    checks = {"agocuda_frame": native.AgoFrame, "agocuda_pyramid_level": native.PyramidLevel,
              "agocuda_half_job": native.HalfJob, "agocuda_lk_frame": native.LkFrame}
    body = "".join(f'printf("{n} %zu\\n", sizeof({n}));\n' for n in checks)
    for f in ("count", "scharrWords", "windowDimension", "newCapacity"):
        body += f'printf("lk.{f} %zu\\n", offsetof(agocuda_lk_frame, {f}));\n'
    out = _run('#include <stdio.h>\n#include <stddef.h>\n#include "agocuda.h"\nint main(){' + body + "return 0;}",
               [os.path.dirname(AGOCUDA_H), "/usr/local/cuda/include"])
    got = dict(line.split() for line in out.strip().splitlines())
    for n, cls in checks.items():
        assert int(got[n]) == ctypes.sizeof(cls), n
    for f in ("count", "scharrWords", "windowDimension", "newCapacity"):
        assert int(got["lk." + f]) == getattr(native.LkFrame, f).offset, f


def test_patch_address_matches_reference():
    """vxFormatImagePatchAddress2d on addressing structures as vxMapImagePatch reports a full
    plane and a plane subsampled by 2 (scale VX_SCALE_UNITY / 2, step 2; vx_api.cpp:27-36,
    :2159-2164): the same byte offset as the reference library's, for every (x, y) probed,
    and NULL outside the patch."""
    import ctypes as C
    import oracle as O
    from mivisionx_b200 import native
    from mivisionx_b200 import vx as V
    ref = O.ref_lib()
    if ref is None or not os.path.exists(native.OPENVX_SO):
        pytest.skip("libraries not built")
    fns = []
    for lib in (native.openvx(), ref):
        f = lib.vxFormatImagePatchAddress2d
        f.argtypes, f.restype = [C.c_void_p, C.c_uint32, C.c_uint32, C.POINTER(V.vx_imagepatch_addressing_t)], C.c_void_p
        fns.append(f)
    base = 1 << 20
    for scale, step, bpp in ((1024, 1, 1), (1024, 1, 2), (512, 2, 1), (512, 2, 2)):
        a = V.vx_imagepatch_addressing_t()
        a.dim_x, a.dim_y, a.stride_x, a.stride_y = 1280, 720, bpp, 1344
        a.scale_x = a.scale_y = scale
        a.step_x = a.step_y = step
        for x, y in ((0, 0), (1, 0), (2, 0), (3, 5), (1279, 719), (640, 2), (1280, 0), (0, 720)):
            got, want = fns[0](base, x, y, C.byref(a)), fns[1](base, x, y, C.byref(a))
            assert got == want, (scale, bpp, x, y, got, want)
