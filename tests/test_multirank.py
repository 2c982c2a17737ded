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
        total = shard.sum_over_ranks(len(ids))                  # host tensors under gloo
        q.put((rank, None if allr is None else allr.tolist(), (t, total, str(shard._device(None)))))
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
    assert out[0][1][0] == out[1][1][0] == 2.0                  # max over ranks
    assert out[0][1][1] == out[1][1][1] == n_walkers             # sum over ranks
    assert out[0][1][2] == out[1][1][2] == "cpu"


def test_shards_cover_the_set():
    for n in (1, 5, 512, 513):
        for world in (1, 2, 3, 8):
            parts = [shard.shard_indices(n, r, world) for r in range(world)]
            allp = np.concatenate(parts)
            assert np.array_equal(allp, np.arange(n))
            sizes = [len(p) for p in parts]
            assert max(sizes) - min(sizes) <= 1


class _HostKmc:
    """The KMC calls of the loop's selection on the host, for CPU ranks: the FP64 oracle
    restatement of the same reference loops (kmc/KineticMonteCarlo.cpp:147-199, 1151-1160)."""

    @staticmethod
    def uniforms(seed, counter, n):
        import torch
        from oracle import kmc as K
        return torch.tensor(K.uniforms(seed, counter, n))

    @staticmethod
    def select(es, em, usable, prefactor, temperature, u):
        import torch
        from oracle import kmc as K
        es, em, usable, u = (t.cpu().numpy() for t in (es, em, usable, u))
        r = K.rates(es, em, usable, prefactor, temperature)
        ch, tot, dt = K.select(r, u[0], u[1])
        step = {"chosen": ch, "n_usable": int(usable.sum()), "total_rate": tot, "dt": dt,
                "barrier": float(es[ch] - em[ch]) if ch >= 0 else 0.0}
        return step, torch.tensor(r), torch.tensor(np.cumsum(r))


def _loop_rank_main(rank, world, port, q):
    """One rank of the AKMC loop's exchange: its share of 24 walkers' events (a stand-in for
    the searches, deterministic in the walker id), the all-gather, the cross-rank duplicate
    removal, the selection every rank takes, and the chosen basin 2 broadcast by its owner."""
    import datetime

    import torch
    import torch.distributed as dist
    from akmc_b200 import akmc_loop as AL
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        AL.kmc = _HostKmc
        loop = object.__new__(AL.AkmcLoop)            # the exchange needs no GPU state
        loop.dev = torch.device("cpu")
        loop.world, loop.rank = world, rank
        loop.seed, loop.iteration, loop.time = 3, 5, 0.0
        loop.prefactor, loop.temperature, loop.e_tol = 1e13, 600.0, 1e-3
        loop.box = np.array([10.0, 10.0, 10.0])
        loop.active_radius = 0.0                       # crystal replicas: basin 2 from the search
        loop.history = []
        n_walkers, e1 = 24, -100.0
        ids = shard.shard_indices(n_walkers, rank, world)
        # walker k: a hop of atom k % 5 (so walkers 0 and 5 find the same event, on two ranks)
        bar = 0.8 + 0.05 * (ids % 5)
        usable = ids % 7 != 6
        ev = dict(ids=ids, site=(ids % 3).astype(np.int32), status=np.where(usable, 1, 2).astype(np.int32),
                  e_saddle=e1 + bar, e_basin2=e1 - 0.01 * ids, usable=usable, unique_local=usable,
                  fingerprint=[(int(k % 5),) if u else None for k, u in zip(ids, usable)],
                  force_calls=100 + ids, atom_forces=50.0 * (100 + ids), learned=False, n_fallback=0, atoms=50)
        loop._basin2 = {int(k): np.full((4, 3), float(k)) for k, u in zip(ids, usable) if u}
        tab = AL.gather_events(ev, world)
        rec = loop._select_and_move(tab, ev, np.zeros((4, 3)), e1)
        q.put((rank, rec.chosen, rec.n_unique, rec.time, loop.pos.tolist(), tab["ids"].tolist(),
               tab["owner"].tolist()))
    finally:
        dist.destroy_process_group()


def test_akmc_loop_exchange_two_ranks():
    """The multi-rank AKMC step on two gloo ranks: every rank sees every walker's event once,
    in walker order, with its owner; duplicates across ranks are removed; both ranks choose the
    same event from the same uniforms and move to the basin 2 its owner broadcasts."""
    import multiprocessing as mp
    from oracle import kmc as K
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_loop_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = {}
    for _ in ps:
        r, *rest = q.get(timeout=120)
        out[r] = rest
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    (c0, u0, t0, x0, ids0, own0), (c1, u1, t1, x1, ids1, own1) = out[0], out[1]
    assert ids0 == ids1 == list(range(24))
    assert own0 == own1 == [0] * 12 + [1] * 12
    assert c0 == c1 and t0 == t1 and x0 == x1
    assert u0 == u1 == 5                                   # five distinct hops among 24 walkers
    # the oracle on the whole table: the first walker of each hop is the unique one
    ids = np.arange(24)
    usable = ids % 7 != 6
    first = np.zeros(24, bool)
    for h in range(5):
        ks = [k for k in ids if usable[k] and k % 5 == h]
        first[ks[0]] = True
    r = K.rates(-100.0 + (0.8 + 0.05 * (ids % 5)), np.full(24, -100.0), first, 1e13, 600.0)
    ch, _, dt = K.select(r, *K.uniforms(3, 5, 2))
    assert c0 == ch and abs(t0 - dt) <= 1e-15 * dt
    assert np.array_equal(np.array(x0), np.full((4, 3), float(ch)))
