"""Scene sharding for several GPUs, checked on CPU with gloo ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from mechanic_b200 import scenes, sharding


def test_partition_covers_every_scene_once_and_balances():
    rng = np.random.default_rng(0)
    counts = np.floor(np.exp(rng.uniform(np.log(64), np.log(8192), 256))).astype(int)
    for n in (1, 2, 3, 4, 8):
        parts = sharding.partition(counts, n)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(256))
        for p in parts:   # contiguous ranges
            assert p == list(range(p[0], p[-1] + 1)) if p else True
        # each rank is within one largest scene of its even share
        loads = [counts[p].sum() for p in parts]
        assert max(loads) - counts.sum() / n <= counts.max()
        assert sharding.imbalance(counts, parts) < 1.1 if n <= 4 else True


def test_partition_edge_cases():
    assert sharding.partition([], 2) == [[], []]
    assert sharding.partition([5], 3) == [[0], [], []] or sum(len(p) for p in sharding.partition([5], 3)) == 1
    with pytest.raises(ValueError):
        sharding.partition([1, 2], 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        lst = scenes.batched_uneven(24, seed=3, lo=64, hi=512, bearing_fraction=0.0)
        counts = [s.body_count for s in lst]
        mine = sharding.partition(counts, world)[rank]
        import oracle
        from mechanic_b200 import abi
        c = abi.MkConfig()
        c.collisions_enabled = 1
        c.mechanism_self_collisions = 1
        c.solver_iterations = 8
        w = oracle.OracleWorld.batch([lst[i] for i in mine], c) if mine else None
        for tick in range(1, 4):
            if w is not None:
                w.step(tick)
        res = {"rank": rank, "scenes": mine, "bodies": int(sum(counts[i] for i in mine)),
               "pairs": int(w.pair_count) if w is not None else 0}
        allres = sharding.gather_results(res)
        slowest = sharding.max_over_ranks(float(rank + 1))
        if rank == 0:
            q.put((allres, slowest))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_step_their_shards_and_gather():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    allres, slowest = q.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r["rank"] for r in allres] == [0, 1]
    assert sorted(i for r in allres for i in r["scenes"]) == list(range(24))
    assert slowest == 2.0
    # without mechanisms the scenes do not interact: sharded pair counts equal the whole batch's
    lst = scenes.batched_uneven(24, seed=3, lo=64, hi=512, bearing_fraction=0.0)
    import oracle
    from mechanic_b200 import abi
    c = abi.MkConfig()
    c.collisions_enabled = 1
    c.mechanism_self_collisions = 1
    c.solver_iterations = 8
    whole = oracle.OracleWorld.batch(lst, c)
    for tick in range(1, 4):
        whole.step(tick)
    assert whole.pair_count == sum(r["pairs"] for r in allres)
