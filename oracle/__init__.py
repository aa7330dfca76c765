"""CPU oracles for the AGO vision path -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import
this package, and only as the checker: nothing in ``mivisionx_b200`` uses it.

* ``oracle_lib()``  -- ctypes handle on ``_ref/libagooracle.so``, the plain-C restatement of
  the reference HAF CPU kernels (``agooracle.c``; each function cites the reference line it
  follows).
* ``ref_lib()``     -- ctypes handle on ``_ref/libopenvx_ref.so``, the reference AMD OpenVX
  library itself compiled from its own sources (``Makefile``), or None when it was not built.
  Its HafCpu_* kernels are reachable through ``ref_haf(name)``; its OpenVX API through the
  same ctypes binding the product uses (``mivisionx_b200.vx``).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
ORACLE_SO = os.path.join(REF_DIR, "libagooracle.so")
REF_SO = os.path.join(REF_DIR, "libopenvx_ref.so")
REF_SYMS = os.path.join(REF_DIR, "ref_symbols.txt")
RUNVX_REF = os.path.join(REF_DIR, "runvx_ref")      # reference runvx on the reference library
RUNVX_B200 = os.path.join(REF_DIR, "runvx_b200")    # the same runvx on this project's libopenvx.so
REFERENCE_TREE = "/root/reference/amd_openvx/openvx"

_oracle = None
_ref = None
_ref_syms = None


def build(with_reference: bool | None = None) -> None:
    """Compile the C restatement and, when the reference tree is present, the reference."""
    targets = ["oracle"]
    if with_reference is None:
        with_reference = os.path.isdir(REFERENCE_TREE)
    if with_reference:
        targets += ["ref", "runvx"]
    subprocess.run(["make", "-s", "-C", HERE, f"-j{min(16, os.cpu_count() or 4)}"] + targets, check=True)


def oracle_lib() -> C.CDLL:
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            build(with_reference=False)
        _oracle = C.CDLL(ORACLE_SO, mode=C.RTLD_LOCAL)
    return _oracle


def ref_lib():
    """The reference libopenvx built from source, or None if it is not available."""
    global _ref
    if _ref is None and os.path.exists(REF_SO):
        _ref = C.CDLL(REF_SO, mode=C.RTLD_LOCAL)
    return _ref


def ref_haf(name: str):
    """Return the reference's C++ function `name` (e.g. 'HafCpu_Gaussian_U8_U8_3x3')."""
    global _ref_syms
    lib = ref_lib()
    if lib is None:
        return None
    if _ref_syms is None:
        _ref_syms = {}
        with open(REF_SYMS) as f:
            for line in f:
                s = line.strip()
                i = 2
                while s[i].isdigit():
                    i += 1
                n = int(s[2:i])
                _ref_syms[s[i:i + n]] = s
    return getattr(lib, _ref_syms[name])
