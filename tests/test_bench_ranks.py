"""The multi-rank host logic of bench.py (--gpus N: N independent replicas,
one process per GPU) on CPU with two gloo ranks: the case is written once by
rank 0 and read by every rank after a barrier, the timed region's length is
the maximum over ranks on every rank, and the whole-job rate counts every
rank's cells."""
import os
import socket
import sys
from datetime import timedelta
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, base: str, q) -> None:
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        sys.path.insert(0, str(ROOT))
        import bench

        case = bench.shared_case((8, 6, 4), 1, rank, world, dist, base=Path(base))
        ms = bench.max_over_ranks(10.0 * (rank + 1), dist, world, "cpu")
        q.put((rank, str(case), (case / ".ready").exists(), ms))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_share_case_and_time(tmp_path):
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, str(tmp_path), q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[0] for o in out] == [0, 1]
    assert out[0][1] == out[1][1] and all(o[2] for o in out)
    # the slower rank's time on both ranks
    assert [o[3] for o in out] == [20.0, 20.0]


def test_whole_job_rate_counts_every_replica():
    sys.path.insert(0, str(ROOT))
    import bench

    one = bench.whole_job_rate(4_718_592, 1, 20, 500.0)
    assert abs(one - 4_718_592 * 20 / 0.5 / 1e6) < 1e-9
    assert abs(bench.whole_job_rate(4_718_592, 8, 20, 500.0) - 8 * one) < 1e-9
