"""The multi-GPU bookkeeping of bench.py (replicas, slowest rank's time) with
world_size 2 over gloo on CPU: the same calls the NCCL ranks make."""
import json
import os
import socket

import torch.multiprocessing as mp

from gpugraph_b200 import replicas


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out_dir: str) -> None:
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        replicas.barrier()
        slowest = replicas.max_over_ranks(0.5 * (rank + 1))
        rate, secs = replicas.aggregate_rate(1000.0, 0.1 * (rank + 1))
        with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
            json.dump({"world": replicas.world_size(), "slowest": slowest, "rate": rate, "secs": secs}, f)
    finally:
        dist.destroy_process_group()


def test_two_replicas_over_gloo(tmp_path):
    port = _free_port()
    mp.spawn(_rank, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    for r in range(2):
        got = json.loads((tmp_path / f"r{r}.json").read_text())
        assert got["world"] == 2
        assert got["slowest"] == 1.0
        # both ranks processed 1000 units; the job took the slowest rank's 0.2 s
        assert abs(got["secs"] - 0.2) < 1e-12 and abs(got["rate"] - 2 * 1000.0 / 0.2) < 1e-6


def test_single_process_is_a_no_op():
    assert replicas.world_size() == 1
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.aggregate_rate(10.0, 2.0) == (5.0, 2.0)
