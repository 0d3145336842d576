"""Multi-rank host logic of bench.py on CPU (gloo, world size 2): replicas
report the max over ranks of their timings and the sum of their counts,
and the whole-job throughput is N replicas' cells over the slowest rank's
time.  No GPU is involved."""
import json
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _rank_main(rank, world, port, outdir):
    sys.path.insert(0, str(ROOT))
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        maxes, sums = bench.combine_ranks(world, "cpu", maxes=(10.0 + rank, 5.0 - rank),
                                          sums=(100.0 * (rank + 1),))
        Path(outdir, f"r{rank}.json").write_text(json.dumps({"maxes": maxes, "sums": sums}))
    finally:
        dist.destroy_process_group()


def test_combine_ranks_gloo_world2(tmp_path):
    port = _free_port()
    mp.spawn(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    for r in range(2):
        d = json.loads((tmp_path / f"r{r}.json").read_text())
        assert d["maxes"] == [11.0, 5.0]
        assert d["sums"] == [300.0]


def test_single_rank_and_weak_value():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.combine_ranks(1, "cpu", maxes=(3.0,), sums=(7.0,)) == ([3.0], [7.0])
    # 4 replicas of 1e6 cells at 100 ms for the slowest rank
    assert bench.weak_value(4, 1_000_000, 100.0) == pytest.approx(4e7)
