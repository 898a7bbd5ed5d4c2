"""Bucket-sharded sketch on the GPU: the routing kernels (qs_shard_partition and
qs_shard_unpartition) against their definition, and G shards emulated in one process — each
shard's sketch takes the keys the partition routes to it — against one sketch.  (The
all-to-all between ranks is covered by the gloo tests in tests/test_sharded.py.)"""
import numpy as np
import pytest
import torch

import qsketch_b200 as qs
from qsketch_b200 import data
from qsketch_b200.sharded import ShardedSketch, gpu_partition, gpu_unpartition

pytestmark = pytest.mark.gpu
SEED = 2654435769


def owner(keys, n_low, G):
    b = (keys.astype(np.uint64) * np.uint64(SEED) % np.uint64(1 << 32)) % np.uint64(n_low)
    return (b * np.uint64(G) // np.uint64(n_low)).astype(np.int64)


@pytest.mark.parametrize("n,G", [(0, 4), (1, 3), (4095, 2), (1 << 20, 8), ((1 << 20) + 17, 5), (1 << 16, 32)])
def test_partition_is_a_stable_partition_by_owner(gpu, n, G):
    n_low = 2097143
    keys = data.uniform_keys(max(n, 1), seed=9)[:n].contiguous()
    out, counts, perm = gpu_partition(keys, SEED, n_low, G, True)
    k = keys.cpu().numpy()
    own = owner(k, n_low, G)
    order = np.argsort(own, kind="stable")
    assert counts == np.bincount(own, minlength=G).tolist()
    assert np.array_equal(out.cpu().numpy(), k[order])
    assert np.array_equal(perm.cpu().numpy(), order.astype(np.int32))
    if n:
        back = gpu_unpartition(out, perm)
        assert torch.equal(back, keys)


def test_emulated_shards_equal_one_sketch(gpu):
    """Four shards in one process: each shard's full-range sketch takes only its routed keys
    (several batches); each shard answers for the keys it owns exactly as one sketch does."""
    G, n_low, n_high = 4, 65521, 1 << 14
    masks = qs.generate_hashmask(1021, 32, 3, 4, 1)
    one = qs.Sketch_GPU_Sub_Warp_Level(n_low, 8, n_high, 32, hash_seed=SEED, mask_table=masks)
    shards = [qs.Sketch_GPU_Sub_Warp_Level(n_low, 8, n_high, 32, hash_seed=SEED, mask_table=masks) for _ in range(G)]
    for c in range(3):
        keys = data.zipf_keys(1 << 20, 1 << 16, 1.1, seed=20 + c, perm_seed=5)
        one.insert(keys)
        parts, counts, _ = gpu_partition(keys, SEED, n_low, G, False)
        off = np.concatenate([[0], np.cumsum(counts)])
        for g in range(G):
            shards[g].insert(parts[off[g]:off[g + 1]])
    q = data.rank_keys(5, 0, 1 << 16)
    want = one.search(q)
    qp, qc, perm = gpu_partition(q, SEED, n_low, G, True)
    qoff = np.concatenate([[0], np.cumsum(qc)])
    est = torch.cat([shards[g].search(qp[qoff[g]:qoff[g + 1]]) for g in range(G)])
    got = gpu_unpartition(est, perm)
    one.sync()
    assert torch.equal(got, want)
    assert one.stats()["linked_buckets"] > 100
    low1, _ = one.tables()
    for g in range(G):
        lo, hi = (g * n_low + G - 1) // G, ((g + 1) * n_low + G - 1) // G
        lg, _ = shards[g].tables()
        a, b = lg.reshape(-1, 8), low1.reshape(-1, 8)
        assert np.array_equal(a[lo:hi, :7], b[lo:hi, :7])
        assert not a[:lo, :7].any() and not a[hi:, :7].any()  # a shard touches only its own range


def test_single_rank_sharded_sketch_is_the_sketch(gpu):
    masks = qs.generate_hashmask(1021, 32, 3, 4, 1)
    ss = ShardedSketch(16381, 1 << 12, hash_seed=SEED, mask_table=masks)
    one = qs.Sketch_GPU_Sub_Warp_Level(16381, 8, 1 << 12, 32, hash_seed=SEED, mask_table=masks)
    keys = data.zipf_keys(1 << 19, 1 << 14, 1.2, seed=2, perm_seed=3)
    ss.insert(keys)
    one.insert(keys)
    q = data.rank_keys(3, 0, 1 << 14)
    assert torch.equal(ss.search(q), one.search(q))
