"""The multi-GPU bookkeeping of bench.py (replicas over disjoint shards, the
slowest rank's time, the units summed over ranks) with world_size 2 over gloo
on CPU: the same calls the NCCL ranks make."""
import json
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from gpugraph_b200 import replicas


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _ro():
    # a small CSR-like offsets array: 500 vertices, every third one without out-edges
    deg = np.where(np.arange(500) % 3 == 0, 0, 2)
    return np.concatenate([[0], np.cumsum(deg)]).astype(np.int32)


def _rank(rank: int, world: int, port: int, out_dir: str) -> None:
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        replicas.barrier()
        slowest = replicas.max_over_ranks(0.5 * (rank + 1))
        # ranks processed different numbers of units: the job rate sums them
        rate, secs = replicas.aggregate_rate(1000.0 * (rank + 1), 0.1 * (rank + 1))
        srcs = replicas.source_block(_ro(), 64)
        graphs = replicas.shard(list(range(256)))
        with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
            json.dump({"world": replicas.world_size(), "rank": replicas.rank(), "slowest": slowest, "rate": rate,
                       "secs": secs, "srcs": srcs.tolist(), "graphs": graphs}, f)
    finally:
        dist.destroy_process_group()


def test_two_replicas_over_gloo(tmp_path):
    port = _free_port()
    mp.spawn(_rank, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    got = [json.loads((tmp_path / f"r{r}.json").read_text()) for r in range(2)]
    ro = _ro()
    for r, g in enumerate(got):
        assert g["world"] == 2 and g["rank"] == r
        assert g["slowest"] == 1.0
        # 1000 + 2000 units over the slowest rank's 0.2 s
        assert abs(g["secs"] - 0.2) < 1e-12 and abs(g["rate"] - 3000.0 / 0.2) < 1e-6
        assert len(g["srcs"]) == 64 and all(ro[s + 1] > ro[s] for s in g["srcs"])
    # the shards cover the units exactly once
    allsrc = got[0]["srcs"] + got[1]["srcs"]
    assert len(set(allsrc)) == 128
    assert sorted(got[0]["graphs"] + got[1]["graphs"]) == list(range(256))
    assert got[0]["graphs"] == list(range(128))


def test_shard_bounds_cover_every_unit_once():
    for n in (0, 1, 5, 64, 256, 257):
        for world in (1, 2, 3, 4, 8):
            seen = []
            for r in range(world):
                b, e = replicas.shard_bounds(n, r, world)
                seen.extend(range(b, e))
                assert e - b in (n // world, n // world + 1)
            assert seen == list(range(n))


def test_single_process_is_a_no_op():
    assert replicas.world_size() == 1 and replicas.rank() == 0
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.sum_over_ranks(3.5) == 3.5
    assert replicas.aggregate_rate(10.0, 2.0) == (5.0, 2.0)
    ro = _ro()
    assert np.array_equal(replicas.source_block(ro, 64), replicas.seeded_sources(ro, 64))
    assert replicas.shard([1, 2, 3]) == [1, 2, 3]
