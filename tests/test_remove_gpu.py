"""REMOVE on the GPU (qs_remove) against the oracle's sequential restatement, bit for bit:
estimates and both tables after interleaved insert and remove calls, on skewed streams whose
buckets link (removals then land in the high level), removals of absent keys and of more
occurrences than were inserted (floors at 0), a saturated bucket, and the count-min."""
import numpy as np
import pytest
import torch

import oracle
import qsketch_b200 as qs
from qsketch_b200 import _lib, data

pytestmark = pytest.mark.gpu
SEED = 2654435769


def pair(n_low, n_high, mask_rng=1):
    masks = qs.generate_hashmask(1021, 32, 3, 4, mask_rng)
    return (qs.Sketch_GPU_Sub_Warp_Level(n_low, 8, n_high, 32, hash_seed=SEED, mask_table=masks),
            oracle.Msws(n_low, n_high, SEED, masks))


def same_tables(sk, orc):
    low, high = sk.tables()
    assert np.array_equal(low, orc.low), "low tables differ"
    assert np.array_equal(high, orc.high), "high pools differ"
    assert sk.stats()["dropped_keys"] == orc.dropped


@pytest.mark.parametrize("n_ranks,s", [(1 << 12, 1.2), (1 << 16, 1.0)])
def test_remove_after_insert_matches_oracle(gpu, n_ranks, s):
    sk, orc = pair(16381, 1 << 14)
    ins = data.zipf_keys(1 << 21, n_ranks, s, seed=31, perm_seed=8)
    rem = data.zipf_keys(1 << 20, 2 * n_ranks, s, seed=32, perm_seed=8)  # half the ranks never inserted
    q = data.rank_keys(8, 0, 2 * n_ranks)
    for call in range(2):
        sk.insert(ins)
        orc.insert(ins.cpu().numpy())
        sk.remove(rem)
        orc.remove(rem.cpu().numpy())
    got = sk.search(q).cpu().numpy()
    sk.sync()
    assert np.array_equal(got, orc.query(q.cpu().numpy()))
    same_tables(sk, orc)
    assert (orc.low.reshape(-1, 8)[:, 7] > 1024).sum() > 50  # removals reached linked buckets


def test_remove_more_than_inserted_and_a_heavy_key(gpu):
    sk, orc = pair(4093, 1024)
    ins = torch.cat([data.uniform_keys(1 << 18, seed=2), torch.full((5000,), 77, dtype=torch.uint32, device="cuda")])
    rem = torch.cat([data.uniform_keys(1 << 17, seed=2), data.uniform_keys(1 << 17, seed=99),
                     torch.full((7000,), 77, dtype=torch.uint32, device="cuda")])
    sk.insert(ins)
    orc.insert(ins.cpu().numpy())
    sk.remove(rem)
    orc.remove(rem.cpu().numpy())
    q = torch.cat([ins[:4096], torch.tensor([77], dtype=torch.uint32, device="cuda")])
    got = sk.search(q).cpu().numpy()
    sk.sync()
    assert np.array_equal(got, orc.query(q.cpu().numpy()))
    same_tables(sk, orc)


def test_remove_in_saturated_buckets_is_dropped(gpu):
    sk, orc = pair(4093, 8)
    keys = data.zipf_keys(1 << 20, 1 << 12, 1.2, seed=1, perm_seed=2)
    sk.insert(keys)
    orc.insert(keys.cpu().numpy())
    sk.remove(keys[: 1 << 18])
    orc.remove(keys[: 1 << 18].cpu().numpy())
    assert sk.status() == _lib.QS_ERR_POOL_FULL
    same_tables(sk, orc)


def test_count_min_remove_matches_oracle(gpu):
    cm = qs.Sketch_GPU_Thread(65521, 3, seed_rng=4)
    cref = oracle.CountMin(65521, cm.info()["seeds"])
    ins = data.zipf_keys(1 << 20, 1 << 14, 1.1, seed=3, perm_seed=5)
    rem = data.zipf_keys(1 << 19, 1 << 15, 1.1, seed=4, perm_seed=5)
    cm.insert(ins)
    cref.insert(ins.cpu().numpy())
    cm.remove(rem)
    cref.remove(rem.cpu().numpy())
    cm.sync()
    low, _ = cm.tables()
    assert np.array_equal(low, cref.table)
