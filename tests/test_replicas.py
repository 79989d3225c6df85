"""The multi-GPU form of bench.py is replicas: each rank reconstructs its own
seeded scan, and the ranks only meet to time the job (barriers and the
maximum of their step times).  These host-side pieces run here as two gloo
ranks on the CPU, rendezvous on 127.0.0.1."""
import json
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist

    import bench
    r, w, local = bench.dist_env()
    bench.init_replicas(w, "gloo", timeout_s=60)
    ms = 100.0 + 25.0 * r                       # the ranks' own step times
    job = bench.max_over_ranks(ms, w, torch.device("cpu"))
    params = bench.phantom_params(2024 + r)     # each replica's scan
    dist.barrier()
    dist.destroy_process_group()
    with open(os.path.join(out_dir, f"rank{r}.json"), "w") as f:
        json.dump({"rank": r, "world": w, "local": local, "job_ms": job, "rate": bench.job_rate(job, w),
                   "phantom_sum": float(params.sum())}, f)


def test_two_gloo_replicas_time_the_job_by_the_slowest_rank(tmp_path):
    mp = pytest.importorskip("torch.multiprocessing")
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(2)]
    assert [x["rank"] for x in res] == [0, 1] and all(x["world"] == 2 for x in res)
    assert all(x["job_ms"] == 125.0 for x in res)                   # the slower rank's time, on both
    assert all(x["rate"] == pytest.approx(2 * 1000.0 / 125.0) for x in res)
    assert res[0]["phantom_sum"] != res[1]["phantom_sum"]           # independent scans


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(12.5, 1, None) == 12.5
    assert bench.job_rate(500.0, 1) == 2.0


def test_reference_arm_runs_on_rank_zero_only(capsys, monkeypatch):
    """Under torchrun the other ranks of the reference arm exit without work."""
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class Args:
        gpus, steps, warmup = 2, 1, 3
    assert bench.run_reference(Args()) is None
    assert capsys.readouterr().out == ""
