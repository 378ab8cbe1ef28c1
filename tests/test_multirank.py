"""The multi-GPU form is replicas only: each rank runs its own disjoint
replicas and the job time is the max over ranks.  Two gloo ranks on CPU check
the sharding and the max reduction that `bench.py --gpus N` uses (no GPU)."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import json
    import sys

    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        pkg = bench.load_pkg()
        wl = bench.workload(pkg, 3, 2, 8, rank)
        elapsed = bench.max_over_ranks(1.5 + rank, dist, "cpu")
        rec = {"dseeds": sorted({w[0] for w in wl}), "seeds": [w[2] for w in wl], "temps": [w[1] for w in wl],
               "elapsed": elapsed}
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump(rec, f)
    finally:
        dist.destroy_process_group()


def test_replica_sharding_and_max_time(tmp_path):
    import json

    import torch.multiprocessing as mp

    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    recs = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    # disjoint disorder realisations and run seeds, same temperature grid
    assert not set(recs[0]["dseeds"]) & set(recs[1]["dseeds"])
    assert not set(recs[0]["seeds"]) & set(recs[1]["seeds"])
    assert recs[0]["temps"] == recs[1]["temps"]
    assert recs[0]["dseeds"] == [20260710, 20260711, 20260712] and recs[1]["dseeds"] == [20260713, 20260714, 20260715]
    # the job time is the slowest rank's
    assert recs[0]["elapsed"] == recs[1]["elapsed"] == 2.5
