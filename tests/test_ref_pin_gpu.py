"""Pin of the oracle's insert/query core by the reference's own sketch kernels.

oracle/_ref/libqsref.so is built from the reference's sources (oracle/Makefile) and runs its
Sketch_GPU_Sub_Warp_Level (device_sketch_v3.h:526-634) and Sketch_GPU_Thread
(device_sketch_v0.h:105-191) kernels with their seed and mask engines reseeded.  On inputs
where the reference's result does not depend on the thread schedule — for the MSWS, no low
counter passing 128, so no bucket links (device_sketch_v3.h:160-190); for the count-min,
any input, since its counter additions commute — the reference's estimates and tables must
equal the oracle's and this library's bit for bit.  The seed and the mask table the
reference drew are fed to the oracle and to libqsketch, so all three use the same hash.
"""
import numpy as np
import pytest
import torch

import oracle
import qsketch_b200 as qs
from qsketch_b200 import data

pytestmark = pytest.mark.gpu

N_LOW_CFG1 = 262139  # find_greatest_prime(2^18): 8 MB of 32-byte buckets, the uniform configuration


@pytest.fixture(scope="module")
def ref():
    r = oracle.ref_lib()
    if r is None or not hasattr(r, "ref_msws_gpu"):
        pytest.skip("oracle/_ref/libqsref.so (the reference's kernels) was not built")
    return r


def three_way_msws(keys, queries, n_low, n_high, seed_rng, mask_rng):
    got_ref, seed, masks, low_ref = oracle.ref_msws_gpu(seed_rng, mask_rng, n_low, n_high, keys, queries,
                                                        with_low=True)
    orc = oracle.Msws(n_low, n_high, seed, masks)
    orc.insert(keys)
    want = orc.query(queries)
    sk = qs.Sketch_GPU_Sub_Warp_Level(n_low, 8, n_high, 32, hash_seed=seed, mask_table=masks)
    sk.insert(torch.from_numpy(keys).cuda())
    got = sk.search(torch.from_numpy(queries).cuda()).cpu().numpy()
    sk.sync()
    low, _ = sk.tables()
    return got_ref, want, got, low_ref, orc.low.copy(), low, orc


def assert_three_equal(got_ref, want, got, what):
    bad = np.nonzero(got_ref != want)[0]
    assert bad.size == 0, f"{what}: oracle differs from the reference kernel at {bad.size} keys, first {bad[:5]}"
    bad = np.nonzero(got != want)[0]
    assert bad.size == 0, f"{what}: libqsketch differs from the oracle at {bad.size} keys, first {bad[:5]}"


def test_msws_uniform_2_24_pinned_by_reference_kernels(gpu, ref):
    """The uniform configuration at full size: 2^24 keys, n_low = 262139, query every key."""
    keys = data.uniform_keys(1 << 24, seed=1).cpu().numpy()
    got_ref, want, got, low_ref, low_orc, low, _ = three_way_msws(keys, keys, N_LOW_CFG1, 1024, 7, 3)
    assert_three_equal(got_ref, want, got, "uniform 2^24")
    assert np.array_equal(low_ref, low_orc), "low tables: oracle vs reference kernel"
    assert np.array_equal(low, low_orc), "low tables: libqsketch vs oracle"
    assert (low_ref.reshape(-1, 8)[:, 7] == 0).all()  # nothing linked: the input stayed order-independent
    assert want.min() >= 1


def test_msws_repeated_keys_pinned_by_reference_kernels(gpu, ref):
    """2^20 distinct keys, each 16 times in a shuffled stream: counters up to ~112, close to
    the 128 limit the reference links at; query the distinct keys."""
    rng = np.random.default_rng(5)
    distinct = np.unique(rng.integers(0, 2 ** 32, 1 << 21, dtype=np.uint64).astype(np.uint32))[:1 << 20]
    keys = rng.permutation(np.repeat(distinct, 16)).astype(np.uint32)
    got_ref, want, got, low_ref, low_orc, low, _ = three_way_msws(keys, distinct, N_LOW_CFG1, 1024, 7, 3)
    assert_three_equal(got_ref, want, got, "repeated keys")
    assert np.array_equal(low_ref, low_orc) and np.array_equal(low, low_orc)
    assert low_orc.reshape(-1, 8)[:, :7].copy().view(np.uint8).max() > 96
    assert (want >= 16).all()


def test_msws_reference_runner_refuses_undefined_inputs(gpu, ref):
    """The runner refuses, before any launch, a stream that would take a counter past 128
    (the reference would link through an unbounded, schedule-dependent wait) and a key count
    whose warp shares are not whole multiples of 4."""
    keys = np.full(1 << 18, 12345, np.uint32)  # one key 2^18 times
    with pytest.raises(ValueError):
        oracle.ref_msws_gpu(7, 3, 4093, 64, keys, keys[:4])
    with pytest.raises(ValueError):
        oracle.ref_msws_gpu(7, 3, 4093, 64, np.arange(1 << 18, dtype=np.uint32)[:-2], keys[:4])


@pytest.mark.parametrize("skewed", [False, True])
def test_count_min_pinned_by_reference_kernels(gpu, ref, skewed):
    """Count-min at the uniform configuration's bytes (8 MB, m = 3 rows): 2^24 keys, uniform or
    Zipf 1.1 over 2^20 ranks; estimates and all three rows of counters."""
    n = qs.find_greatest_prime((8 << 20) // 4 // 3)
    if skewed:
        keys = data.zipf_keys(1 << 24, 1 << 20, 1.1, seed=3, perm_seed=9).cpu().numpy()
        queries = data.rank_keys(9, 0, 1 << 20).cpu().numpy()
    else:
        keys = data.uniform_keys(1 << 24, seed=2).cpu().numpy()
        queries = keys[: 1 << 22].copy()
    got_ref, seeds, tab_ref = oracle.ref_cm_gpu(11, n, 3, keys, queries, with_table=True)
    cref = oracle.CountMin(n, seeds)
    cref.insert(keys)
    want = cref.query(queries)
    cm = qs.Sketch_GPU_Thread(n, 3, seeds=seeds)
    cm.insert(torch.from_numpy(keys).cuda())
    got = cm.search(torch.from_numpy(queries).cuda()).cpu().numpy()
    cm.sync()
    assert_three_equal(got_ref, want, got, "count-min")
    low, _ = cm.tables()
    assert np.array_equal(tab_ref, low), "count-min counters: libqsketch vs the reference kernel"
