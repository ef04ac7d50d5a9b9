"""Multi-rank ensemble sharding on CPU (gloo, world size 2): the partition, and
the single end-of-run gather, with a stand-in for the per-member GPU work."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from wildfires_b200.sharding import partition, run_sharded


def test_partition_balances_and_covers():
    costs = [5, 1, 9, 3, 3, 7, 2, 8]
    parts = partition(costs, 3)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)
    assert partition(costs, 3) == parts            # every rank derives the same partition
    assert partition(costs, 1) == [list(range(len(costs)))]
    assert partition([], 4) == [[], [], [], []]
    with pytest.raises(ValueError):
        partition(costs, 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, costs, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seen = []

        def run_members(indices):
            seen.extend(indices)
            return [{"member": i, "rank": rank, "mass": 10.0 * i} for i in indices]

        res = run_sharded(len(costs), costs, run_members)
        with open(os.path.join(out_dir, "rank%d" % rank), "w") as f:
            f.write(repr((seen, res)))
    finally:
        dist.destroy_process_group()


def test_two_ranks_gather_every_member_once(tmp_path):
    costs = [4.0, 1.0, 3.0, 2.0, 5.0]
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, costs, str(tmp_path)), nprocs=2, start_method="spawn")
    seen0, res0 = eval(open(tmp_path / "rank0").read())
    seen1, res1 = eval(open(tmp_path / "rank1").read())
    assert res1 is None
    assert sorted(seen0 + seen1) == list(range(len(costs)))
    assert not set(seen0) & set(seen1)
    assert [r["member"] for r in res0] == list(range(len(costs)))
    assert all(r["mass"] == 10.0 * r["member"] for r in res0)
    assert {r["rank"] for r in res0} == {0, 1}
