"""The N>1 plumbing of bench.py on the host: two gloo ranks (world size 2, 127.0.0.1), the
max-over-ranks timing, the barrier, per-rank frame seeds (weak scaling: no data collective)
and the reference arm's rank rule (rank 0 runs, the others exit without work)."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(ws), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=ws, init_method=f"tcp://127.0.0.1:{port}")
    try:
        bench._barrier(ws)
        slowest = bench._max_over_ranks(1.5 + rank, ws)
        frames = bench.WORKLOADS["gauss_sobel_mag_depth_thresh_1080p"].make_frames(bench.frame_seed(rank), 1)
        bench._barrier(ws)
        q.put((rank, slowest, bench._dist(), int(frames[0][:8, :8].sum())))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [2.5, 2.5]                  # max over ranks on both
    assert [r[2] for r in res] == [(2, 0, 0), (2, 1, 1)]      # WORLD_SIZE, RANK, LOCAL_RANK
    assert res[0][3] != res[1][3]                             # each rank its own frames


def test_reference_arm_runs_on_rank0_only(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    called = []
    monkeypatch.setattr(bench, "reference_cpu", lambda *a, **k: called.append(a))
    assert bench.run_reference_arm(None, bench.DEFAULT_WORKLOAD) == 0   # returns before reading its arguments
    assert not called


def test_gpus_flag_spawns_ranks():
    """`bench.py --gpus 2` outside torchrun starts two local ranks itself (torchrun's
    environment, 127.0.0.1 rendezvous); with the reference arm rank 0 alone prints its line
    and both exit 0."""
    import json
    import subprocess
    import oracle
    if oracle.ref_lib() is None:
        pytest.skip("reference library not built")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--impl", "reference",
                        "--steps", "1", "--warmup", "0", "--workload", "gauss_sobel_mag_depth_thresh_1080p"],
                       capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1, r.stdout
    assert lines[0]["impl"] == "reference" and lines[0]["n_gpus"] == 2 and lines[0]["value"] > 0
