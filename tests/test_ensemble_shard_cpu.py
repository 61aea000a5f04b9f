"""Round-robin sharding of an ensemble over ranks (replicas only), on CPU.

With one process per GPU the members are dealt round-robin and each rank evolves
its share; the ranks exchange no fields.  These tests check the deal (disjoint,
complete, balanced) and the one exchange there is, the gather of every member's
analyser rows, with 2 and 3 `gloo` ranks on the CPU (127.0.0.1 rendezvous).
"""
import os
import socket

import pytest

from gftevolver_b200.ensemble import member_shard


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("n,world", [(64, 1), (64, 2), (10, 3), (5, 8), (0, 2)])
def test_member_shard_is_a_balanced_partition(n, world):
    shards = [member_shard(n, r, world) for r in range(world)]
    flat = sorted(m for s in shards for m in s)
    assert flat == list(range(n))
    sizes = [len(s) for s in shards]
    assert max(sizes) - min(sizes) <= 1
    assert all(m % world == r for r, s in enumerate(shards) for m in s)


def test_member_shard_rejects_bad_ranks():
    with pytest.raises(ValueError):
        member_shard(4, 2, 2)
    with pytest.raises(ValueError):
        member_shard(4, 0, 0)


def _worker(rank, world, port, n, out_dir):
    import datetime

    import torch.distributed as dist

    from gftevolver_b200.ensemble import ShardedEnsemble, gather_member_rows

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = member_shard(n, rank, world)
        # stand-in rows: what member m would have logged (no device needed)
        local = [[{"member": m, "time_iter": t, "energy": float(100 * m + t)} for t in (0, 10)] for m in mine]
        rows = gather_member_rows(local, n, rank, world)
        assert [r[0]["member"] for r in rows] == list(range(n))
        assert all(r[1]["energy"] == 100 * m + 10 for m, r in enumerate(rows))
        # rank and world come from the process group; a rank with no members holds no device state
        if n < world and rank >= n:
            se = ShardedEnsemble([None] * n)
            assert se.members == [] and se.local is None and se.evolve(5) == []
            assert se.gather_rows([])[0][0]["member"] == 0
        else:
            assert gather_member_rows(local, n, rank, world) == rows
        with open(os.path.join(out_dir, f"ok{rank}"), "w") as f:
            f.write("ok")
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n,world", [(7, 2), (2, 3)])
def test_gather_member_rows_gloo(tmp_path, n, world):
    import torch.multiprocessing as mp

    mp.start_processes(_worker, args=(world, _free_port(), n, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    assert all((tmp_path / f"ok{r}").exists() for r in range(world))
