"""The multi-GPU replica path on the host, as two gloo ranks on the CPU: the
realisation partition, per-realisation seeds and the timing / count
reductions.  Realisation r must come out the same whether one rank or two
generate the ensemble; the fields here come from the oracle (no GPU)."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from scarl_b200 import replicas as R

AXES = (8, 12, 16, 20)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _ensemble_checksums(lo, hi):
    """FP64 oracle fields of realisations lo..hi-1 of a small ensemble,
    reduced to (index, sum, sum of squares) per realisation."""
    import scarl_b200 as S
    from oracle import oracle as O
    Np, cl = S.ensemble_draw(0, lo, hi - lo, AXES, 1.5, 4.0)
    seeds = R.realisation_seeds(lo, hi)
    out = []
    for i in range(hi - lo):
        P = S.pad_size(S.PAD_AUTO, 3, cl[i], (1, 1, 1), Np[i], 0.5, 1e-3)
        f = O.gen_padded(Np[i], P, (1, 1, 1), cl[i], 3, 0.5, 1, seed=int(seeds[i]))
        out.append((lo + i, float(f.sum()), float((f * f).sum())))
    return out


def _worker(rank, world, port, n, q):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world,
                                timeout=datetime.timedelta(seconds=60))
        lo, hi = R.shard(n, world, rank)
        mine = _ensemble_checksums(lo, hi)
        allc = [None] * world
        dist.all_gather_object(allc, mine)
        t = R.max_over_ranks(1.0 + rank, dist)
        cnt = R.sum_over_ranks(hi - lo, dist)
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, allc, t, cnt, (lo, hi)))
    except Exception as e:  # report instead of hanging the parent
        q.put((rank, repr(e), None, None, None))


def test_shard_partitions_every_realisation():
    for n in (0, 1, 7, 256, 1000):
        for world in (1, 2, 3, 8):
            blocks = [R.shard(n, world, k) for k in range(world)]
            assert blocks[0][0] == 0 and blocks[-1][1] == n
            for (a, b), (c, d) in zip(blocks, blocks[1:]):
                assert b == c
            sizes = [b - a for a, b in blocks]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        R.shard(4, 2, 2)


def test_single_rank_reductions_are_identity():
    assert R.max_over_ranks(3.5) == 3.5 and R.sum_over_ranks(7) == 7.0
    assert list(R.realisation_seeds(3, 6)) == [3, 4, 5]
    assert R.replica_seed_base(2) == 2000


def test_two_gloo_ranks_reproduce_the_single_rank_ensemble():
    n, world = 7, 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(k, world, port, n, q)) for k in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort(key=lambda r: r[0])
    for rank, allc, t, cnt, blk in res:
        assert not isinstance(allc, str), allc
        assert t == 2.0                    # the slowest rank's time
        assert cnt == n                    # every realisation counted once
        assert blk == R.shard(n, world, rank)
    gathered = [c for part in res[0][1] for c in part]
    single = _ensemble_checksums(0, n)
    assert [g[0] for g in gathered] == list(range(n))
    np.testing.assert_array_equal(np.array(gathered), np.array(single))
