"""The multi-rank host logic of bench.py on two CPU ranks (gloo): the max and sum over ranks
that turn per-rank times and counts into the job's figures, and the batched workload's
per-rank shards.  No GPU: ranks are processes on this host, rendezvous on 127.0.0.1."""

import json
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str) -> None:
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        from ppvm_b200 import circuits as C

        times = bench.over_ranks([1.0 + rank, 10.0 - rank], "cpu", "max")
        counts = bench.over_ranks([100 * (rank + 1)], "cpu", "sum")
        seed = bench.batched_shard_seed(rank)
        shard = C.batched_tfim(count=4, seed=seed)
        first = [(w.n_qubits, len(w.ops)) for w in shard]
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"times": times, "counts": counts, "seed": seed, "first": first}, f)
    finally:
        dist.destroy_process_group()


def test_two_ranks_reduce_and_shard(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    for r in res:
        assert r["times"] == [2.0, 10.0]  # the slowest rank's time, per figure
        assert r["counts"] == [300.0]     # units of all ranks
    assert [r["seed"] for r in res] == [1, 2]  # rank 0 holds the single-GPU batch
    assert res[0]["first"] != res[1]["first"]  # the shards are different instances


def test_one_rank_is_the_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.over_ranks([3.5, 7.0], "cpu", "max") == [3.5, 7.0]
    assert bench.batched_shard_seed(0) == 1


if __name__ == "__main__":
    sys.exit(pytest.main([__file__, "-q"]))
