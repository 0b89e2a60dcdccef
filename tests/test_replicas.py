"""CPU: the replica split and the result gather of gctffind_b200.replicas,
with world size 2 over gloo (one process per rank, 127.0.0.1)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from gctffind_b200 import replicas


def test_partition_balances_and_covers():
    costs = [5, 1, 1, 1, 4, 2, 2]
    shares = replicas.partition(costs, 2)
    assert sorted(i for s in shares for i in s) == list(range(len(costs)))
    loads = [sum(costs[i] for i in s) for s in shares]
    assert max(loads) - min(loads) <= max(costs)
    assert replicas.partition(costs, 2) == shares            # deterministic
    assert replicas.partition([1.0] * 3, 5)[3:] == [[], []]  # idle ranks allowed
    with pytest.raises(ValueError):
        replicas.partition(costs, 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, items, costs, out_dir):
    import datetime
    import json
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    seen = []

    def process(item):
        seen.append(item["id"])
        return {"id": item["id"], "sum": sum(item["data"]), "rank": rank}

    res = replicas.run_replicas(items, costs, process, rank=rank, world=world)
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"res": res, "seen": seen}, f)
    dist.barrier()
    dist.destroy_process_group()


def test_run_replicas_world2_gloo(tmp_path):
    import json
    items = [{"id": i, "data": list(range(i + 3))} for i in range(7)]
    costs = [len(it["data"]) for it in items]
    mp.spawn(_rank_main, args=(2, _free_port(), items, costs, str(tmp_path)), nprocs=2, join=True)
    r0 = json.load(open(tmp_path / "rank0.json"))
    r1 = json.load(open(tmp_path / "rank1.json"))
    assert r0["res"] == r1["res"]                     # every rank has every row
    assert [r["id"] for r in r0["res"]] == list(range(7))
    assert all(r["sum"] == sum(range(r["id"] + 3)) for r in r0["res"])
    assert sorted(r0["seen"] + r1["seen"]) == list(range(7))   # each item processed once
    assert not set(r0["seen"]) & set(r1["seen"])
    shares = replicas.partition(costs, 2)
    assert sorted(r0["seen"]) == shares[0] and sorted(r1["seen"]) == shares[1]
