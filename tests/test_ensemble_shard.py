"""Ensembles across GPUs, host side (CPU, gloo): the runs are bin-packed onto
the ranks by cost (every run exactly once, loads balanced) and the per-run
statistics are gathered in run order with one all-gather; a run reported by
two ranks is an error on every rank.  World size 2 over gloo on 127.0.0.1."""
import os
import socket
import tempfile

import pytest
import torch.multiprocessing as mp

from pyspectral_b200.ensemble import ensemble_specs, gather_stats, run_cost, shard_specs


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_shards_cover_every_run_once_and_balance(world):
    specs = ensemble_specs()
    shards = shard_specs(specs, world)
    assert len(shards) == world
    flat = sorted(i for sh in shards for i in sh)
    assert flat == list(range(len(specs)))
    loads = [sum(run_cost(specs[i]) for i in sh) for sh in shards]
    avg = sum(loads) / world
    # longest-processing-time-first stays within 4/3 of the optimum (>= the mean
    # load and >= the heaviest single run)
    assert max(loads) <= 4.0 / 3.0 * max(avg, max(run_cost(s) for s in specs)) + 1e-9
    if world > 1:
        assert min(loads) > 0


def test_shard_rejects_empty_world():
    with pytest.raises(ValueError):
        shard_specs(ensemble_specs(per_size=1), 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir, duplicate):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        specs = ensemble_specs(per_size=4)
        shards = shard_specs(specs, world)
        mine = list(shards[rank])
        if duplicate and rank == 1:
            mine.append(shards[0][0])  # a run rank 0 also reports
        local = {i: {"N": specs[i]["N"], "seed": specs[i]["seed"], "energy": 0.5 + i, "rank": rank} for i in mine}
        try:
            stats = gather_stats(local)
            res = "ok:" + ",".join(f"{s['seed']}/{s['rank']}" for s in stats)
        except RuntimeError as e:
            res = "error:" + str(e)
        with open(os.path.join(out_dir, f"r{rank}.txt"), "w") as fh:
            fh.write(res)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("duplicate", [False, True])
def test_gather_stats_world2_gloo(duplicate):
    world = 2
    specs = ensemble_specs(per_size=4)
    shards = shard_specs(specs, world)
    owner = {i: r for r, sh in enumerate(shards) for i in sh}
    with tempfile.TemporaryDirectory() as d:
        mp.spawn(_worker, args=(world, _free_port(), d, duplicate), nprocs=world, join=True)
        out = [open(os.path.join(d, f"r{r}.txt")).read() for r in range(world)]
    if duplicate:
        assert all(o.startswith("error:") and "two ranks" in o for o in out)
    else:
        want = "ok:" + ",".join(f"{specs[i]['seed']}/{owner[i]}" for i in range(len(specs)))
        assert out == [want, want]
