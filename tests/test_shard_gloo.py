"""The multi-GPU split on CPU: two `gloo` ranks (one process each) run the
bench's sharding and timing reduction (sysmat_b200/shard.py)."""
import os
import socket

import pytest

from sysmat_b200 import shard


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, n_slabs, steps, out_dir):
    import datetime
    import json
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    slabs = [shard.slab_of(i, rank, world, n_slabs) for i in range(steps)]
    # every rank's timings differ; the job's time is the max over ranks
    t = shard.max_over_ranks([10.0 + rank, 100.0 - rank])
    gathered = [None] * world
    dist.all_gather_object(gathered, slabs)
    dist.barrier()
    dist.destroy_process_group()
    with open(os.path.join(out_dir, "rank%d.json" % rank), "w") as f:
        json.dump({"slabs": slabs, "t": t, "all": gathered}, f)


@pytest.mark.parametrize("n_slabs,steps", [(8, 4), (3, 5)])
def test_two_gloo_ranks_split_slabs_and_reduce_time(tmp_path, n_slabs, steps):
    import json
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), n_slabs, steps, str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    res = [json.load(open(tmp_path / ("rank%d.json" % r))) for r in range(world)]
    for r in range(world):
        assert res[r]["t"] == [10.0 + world - 1, 100.0]          # max over ranks, same on every rank
        assert res[r]["all"] == [res[q]["slabs"] for q in range(world)]
    for i in range(steps):
        step_slabs = [res[r]["slabs"][i] for r in range(world)]
        if n_slabs >= world:
            assert len(set(step_slabs)) == world               # no two ranks on one slab in a step
        assert step_slabs == [(i * world + r) % n_slabs for r in range(world)]
    # over ceil(n_slabs / world) steps every slab is computed
    cover = {res[r]["slabs"][i] for r in range(world) for i in range(min(steps, -(-n_slabs // world)))}
    assert cover == set(range(min(n_slabs, world * steps)))


def test_row_ranges_partition_the_rows():
    for n, world in [(2048, 8), (6400, 3), (5, 8), (0, 2)]:
        ranges = [shard.row_range(n, r, world) for r in range(world)]
        assert ranges[0][0] == 0 and ranges[-1][1] == n
        assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
        sizes = [b - a for a, b in ranges]
        assert max(sizes) - min(sizes) <= 1


def test_single_process_reduction_is_identity():
    assert shard.max_over_ranks([1.5, 2.0]) == [1.5, 2.0]
    with pytest.raises(ValueError):
        shard.slab_of(0, 2, 2, 4)
