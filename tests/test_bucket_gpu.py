"""One-level bucket sketches — the reference's warp sketch (Sketch_GPU_Warp,
device_sketch_v1.h, 32 counters per bucket) and sub-warp sketch (Sketch_GPU_Sub_Warp,
device_sketch_v2.h, 8 or 16) kept for the ablation against the two-level MSWS — against the
oracle's sequential restatement, bit for bit: estimates and the whole table, after inserts
and removals on uniform and skewed streams, and through a snapshot."""
import numpy as np
import pytest

import oracle
import qsketch_b200 as qs
from qsketch_b200 import data

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("m,skewed", [(32, False), (32, True), (16, True), (8, False), (8, True)])
def test_bucket_sketch_matches_oracle(gpu, m, skewed):
    n = 65521
    cls = qs.Sketch_GPU_Warp if m == 32 else qs.Sketch_GPU_Sub_Warp
    sk = cls(n, m, mask_rng=3, hash_seed=2654435769)
    inf = sk.info()
    orc = oracle.BucketSketch(n, m, 2654435769, inf["mask_table"])
    if skewed:
        keys = data.zipf_keys(1 << 21, 1 << 16, 1.1, seed=4, perm_seed=5)
        q = data.rank_keys(5, 0, 1 << 16)
    else:
        keys = data.uniform_keys(1 << 21, seed=4)
        q = keys[: 1 << 18]
    sk.insert(keys)
    orc.insert(keys.cpu().numpy())
    sk.remove(keys[: 1 << 19])
    orc.remove(keys[: 1 << 19].cpu().numpy())
    got = sk.search(q).cpu().numpy()
    sk.sync()
    assert np.array_equal(got, orc.query(q.cpu().numpy()))
    low, _ = sk.tables()
    assert np.array_equal(low, orc.table)
    masks = orc.masks
    assert all(bin(int(x)).count("1") == 3 for x in masks[:100]) and int(masks.max()) < (1 << m)


def test_bucket_sketch_snapshot(gpu):
    a = qs.Sketch_GPU_Sub_Warp(16381, 16, mask_rng=2, hash_seed=12345)
    a.insert(data.uniform_keys(1 << 18, seed=9))
    b = qs.from_snapshot(a.snapshot())
    assert isinstance(b, qs.Sketch_GPU_Warp)
    q = data.uniform_keys(1 << 14, seed=9)
    assert np.array_equal(a.search(q).cpu().numpy(), b.search(q).cpu().numpy())
