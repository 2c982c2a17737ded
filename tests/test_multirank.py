"""Multi-rank host logic on CPU: two gloo ranks split a walker set, produce per-walker
records, gather them on rank 0 and take the time as the maximum over ranks -- the whole
exchange of the multi-GPU path (no collective touches the force data)."""
import os
import socket

import numpy as np
import pytest

from akmc_b200 import shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, n_walkers, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ids = shard.shard_indices(n_walkers, rank, world)
        # stand-in search results of this rank's walkers (deterministic in the walker id)
        res = np.zeros(len(ids), dtype=[("status", np.int32), ("energy", np.float64),
                                        ("force_calls", np.int32)])
        res["status"] = 1 + (ids % 3 == 0)
        res["energy"] = -100.0 + 0.01 * ids
        res["force_calls"] = 100 + ids
        rec = shard.records(ids, res, e_min=-101.0)
        allr = shard.gather_records(rec, n_walkers)
        t = shard.max_over_ranks(1.0 + rank)
        q.put((rank, None if allr is None else allr.tolist(), t))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n_walkers", [7, 512])
def test_two_ranks_gather_every_walker_once(n_walkers):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, n_walkers, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = {}
    for _ in ps:
        r, allr, t = q.get(timeout=120)
        out[r] = (allr, t)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[1][0] is None
    allr = np.array(out[0][0])
    ids = np.arange(n_walkers)
    assert np.array_equal(allr[:, 0], ids)                      # every walker once, in order
    assert np.array_equal(allr[:, 1], 1 + (ids % 3 == 0))
    assert np.allclose(allr[:, 3], 1.0 + 0.01 * ids)            # barrier = E - E_min
    assert out[0][1] == out[1][1] == 2.0                        # max over ranks


def test_shards_cover_the_set():
    for n in (1, 5, 512, 513):
        for world in (1, 2, 3, 8):
            parts = [shard.shard_indices(n, r, world) for r in range(world)]
            allp = np.concatenate(parts)
            assert np.array_equal(allp, np.arange(n))
            sizes = [len(p) for p in parts]
            assert max(sizes) - min(sizes) <= 1
