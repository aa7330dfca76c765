"""The reference's own runvx (utilities/runvx), unmodified, linked against this project's
libopenvx.so: it must link with no missing symbol and run the reference's in-scope GDF graph
tests on the GPU, with every output equal to what the same runvx produces on the reference
library (runvx's compare facility, utilities/runvx/vxImage.cpp:599, inside the rectangle the
reference defines).

Both binaries come from oracle/Makefile (`make -C oracle runvx`): oracle/_ref/runvx_ref on
the reference library, oracle/_ref/runvx_b200 on mivisionx_b200/lib/libopenvx.so."""
import os
import subprocess

import pytest

import oracle as O
import runvx_cases as RC


def _need(path):
    if not os.path.exists(path):
        pytest.skip(f"{os.path.basename(path)} not built (make -C oracle runvx)")


def _run(exe, gdf_text, tmp, tag):
    path = os.path.join(tmp, f"{tag}.gdf")
    with open(path, "w") as f:
        f.write(gdf_text)
    r = subprocess.run([exe, "-frames:1", path], capture_output=True, text=True, timeout=300, cwd=tmp)
    return r.returncode, r.stdout + r.stderr


def test_runvx_links_against_this_library():
    """Every symbol the reference runvx needs resolves in this library (ldd -r reports
    undefined symbols of the executable and its libraries)."""
    _need(O.RUNVX_B200)
    out = subprocess.run(["ldd", "-r", O.RUNVX_B200], capture_output=True, text=True).stdout
    assert "mivisionx_b200/lib/libopenvx.so" in out, out
    assert "undefined symbol" not in out, out
    assert "not found" not in out, out


@pytest.mark.parametrize("case", RC.CASES, ids=RC.case_ids())
def test_reference_runvx_runs_case(tmp_path, case):
    """The generated GDF text is valid for the reference's own parser and library."""
    _need(O.RUNVX_REF)
    tmp = str(tmp_path)
    RC.write_inputs(case, tmp)
    rc, out = _run(O.RUNVX_REF, RC.gdf(case, tmp, "write"), tmp, "ref")
    assert rc == 0, out
    for name, w, h, fmt, _ in case.outputs:
        p = os.path.join(tmp, f"ref_{name}.raw")
        assert os.path.getsize(p) == RC.frame_bytes(w, h, fmt), (name, out)
    for name, cap in case.arrays:                  # vx_keypoint_t records, 28 bytes each
        n = os.path.getsize(os.path.join(tmp, f"ref_{name}.bin"))
        assert n % 28 == 0 and 0 < n // 28 <= cap, (name, n, out)


@pytest.mark.gpu
@pytest.mark.parametrize("case", RC.CASES, ids=RC.case_ids())
def test_runvx_on_this_library_matches_reference(cuda, tmp_path, case):
    _need(O.RUNVX_REF)
    _need(O.RUNVX_B200)
    tmp = str(tmp_path)
    RC.write_inputs(case, tmp)
    rc, out = _run(O.RUNVX_REF, RC.gdf(case, tmp, "write"), tmp, "ref")
    assert rc == 0, out
    rc, out = _run(O.RUNVX_B200, RC.gdf(case, tmp, "compare"), tmp, "b200")
    assert rc == 0, out
    assert "MISMATCHED" not in out, out
    assert out.count("COMPARE MATCHED") == len(case.outputs) + len(case.arrays), out
