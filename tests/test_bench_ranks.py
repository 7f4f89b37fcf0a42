"""The multi-GPU (replicas) plumbing of bench.py on CPU: two gloo ranks.

bench.py --gpus N runs one independent factorization stream per rank with no
data-path collective; the only collectives are the timing reductions (max
over ranks) and barriers.  These tests run that host-side logic with the
gloo backend on 127.0.0.1, and check that the reference arm reports from
rank 0 alone.
"""
import datetime
import json
import os
import socket
import subprocess
import sys

import pytest
import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, outdir: str) -> None:
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench as b
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r "took" 10 + r ms for 3 factorizations of n = 256
        ms = b.max_over_ranks(10.0 + rank, dist, torch.device("cpu"))
        value = b.whole_job_rate(world, 3 * b.lu_flops(256), ms)
        dist.barrier()
        with open(os.path.join(outdir, f"rank{rank}.json"), "w") as f:
            json.dump({"ms": ms, "value": value}, f)
    finally:
        dist.destroy_process_group()


def test_replica_time_is_the_slowest_rank_and_value_is_whole_job(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    got = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    for g in got:
        assert g["ms"] == 11.0  # the slower rank's time, on every rank
        assert g["value"] == pytest.approx(world * 3 * bench.lu_flops(256) / 0.011)


@pytest.mark.parametrize("workload", ["lu_tc32_rl_n16384", "batch_10000_n16_512"])
def test_reference_arm_reports_from_rank_zero_only(workload):
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1",
               MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()))
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "3", "--workload", workload],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def test_whole_job_rate_scales_with_replicas():
    assert bench.whole_job_rate(1, 5.0, 1000.0) == pytest.approx(5.0)
    assert bench.whole_job_rate(8, 5.0, 1000.0) == pytest.approx(40.0)
