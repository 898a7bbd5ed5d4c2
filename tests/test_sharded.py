"""Bucket-sharded sketch (qsketch_b200/sharded.py): the host-side routing as gloo ranks on CPU.

Each rank holds the oracle as its shard's sketch and partitions with a numpy stand-in of
qs_shard_partition (a stable partition by owner shard; the CUDA kernel is checked against the
same definition in tests/test_sharded_gpu.py).  Two and three ranks insert their own skewed
batches over several collective calls; every rank's query estimates, and each shard's own
bucket range of the low table, must equal one oracle that took the ranks' batches in rank
order, call after call."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
N_LOW, N_HIGH, SEED = 4093, 1 << 12, 2654435769


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def owner(keys, world):
    b = (keys.astype(np.uint64) * np.uint64(SEED) % np.uint64(1 << 32)) % np.uint64(N_LOW)
    return (b * np.uint64(world) // np.uint64(N_LOW)).astype(np.int64)


def batches(rank, calls):
    rng = np.random.default_rng(100 + rank)
    return [((rng.zipf(1.2, 1 << 14) % 3000).astype(np.uint32) * np.uint32(2654435761)) ^ np.uint32(rank * 7)
            for _ in range(calls)]


def _worker(rank, world, port, q, calls):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    try:
        import datetime

        import torch
        import torch.distributed as dist

        import oracle
        from qsketch_b200.sharded import ShardedSketch

        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))

        class Local:  # this shard's sketch: the oracle over the whole bucket range
            def __init__(self):
                self.o = oracle.Msws(N_LOW, N_HIGH, SEED, oracle.generate_hashmask(1))

            def insert(self, keys):
                self.o.insert(keys.numpy())

            def search(self, keys):
                return torch.from_numpy(self.o.query(keys.numpy()))

        def partition(keys, with_perm):
            k = keys.numpy()
            own = owner(k, world)
            order = np.argsort(own, kind="stable")
            counts = np.bincount(own, minlength=world).tolist()
            perm = torch.from_numpy(order.astype(np.int64)) if with_perm else None
            return torch.from_numpy(k[order].copy()), counts, perm

        def unpartition(values, perm):
            out = np.empty(values.numel(), np.uint32)
            out[perm.numpy()] = values.numpy()
            return torch.from_numpy(out)

        sk = ShardedSketch(N_LOW, N_HIGH, hash_seed=SEED, local=Local(), partition=partition,
                           unpartition=unpartition)
        for b in batches(rank, calls):
            sk.insert(torch.from_numpy(b))
        queries = np.unique(np.concatenate(batches(rank, calls)))
        est = sk.search(torch.from_numpy(queries)).numpy()
        lo, hi = sk.owned_buckets()
        q.put((rank, queries, est, (lo, hi), sk.local.o.low.reshape(-1, 8)[lo:hi].copy()))
        dist.destroy_process_group()
    except Exception as e:  # report instead of hanging the parent
        import traceback
        q.put((rank, "error", traceback.format_exc()))


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_equals_one_sketch_of_the_rank_ordered_stream(world):
    import sys
    sys.path.insert(0, ROOT)
    import oracle

    calls = 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, calls)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    res.sort(key=lambda x: x[0])
    for r in res:
        assert not (isinstance(r[1], str) and r[1] == "error"), r[2]
    ref = oracle.Msws(N_LOW, N_HIGH, SEED, oracle.generate_hashmask(1))
    per_rank = [batches(r, calls) for r in range(world)]
    for c in range(calls):
        for r in range(world):
            ref.insert(per_rank[r][c])
    covered = 0
    for rank, queries, est, (lo, hi), low in res:
        assert np.array_equal(est, ref.query(queries)), f"rank {rank}: estimates differ from one sketch"
        want = ref.low.reshape(-1, 8)[lo:hi]
        assert np.array_equal(low[:, :7], want[:, :7]), f"shard {rank}: low counters differ"
        assert np.array_equal(low[:, 7] > 1024, want[:, 7] > 1024), f"shard {rank}: linked buckets differ"
        covered += hi - lo
    assert covered == N_LOW
    assert (ref.low.reshape(-1, 8)[:, 7] > 1024).sum() > 10  # the stream links buckets in every shard
