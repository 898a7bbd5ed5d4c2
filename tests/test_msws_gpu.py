"""GPU parity of the MSWS insert/query path against the sequential CPU oracle.

Every comparison is bit-exact: the per-key query vector and both tables word for word — low
counter words, the high id in word 7 (ids are handed out in the array order of the keys that
switch buckets, as the sequential insert does) and the high pool — and the allocator."""
import numpy as np
import pytest
import torch

import oracle
import qsketch_b200 as qs
from qsketch_b200 import _lib, data

pytestmark = pytest.mark.gpu


def make_pair(n_low, n_high, seed=2654435769, mask_rng=1, compat=False, **kw):
    masks = qs.generate_hashmask(1021, 32, 3, 4, mask_rng)
    sk = qs.Sketch_GPU_Sub_Warp_Level(n_low, 8, n_high, 32, hash_seed=seed, mask_table=masks, compat_v3=compat, **kw)
    orc = oracle.Msws(n_low, n_high, seed, masks, compat_v3=compat)
    return sk, orc


def assert_same_tables(sk, orc):
    low, high = sk.tables()
    gl, ol = low.reshape(-1, 8), orc.low.reshape(-1, 8)
    assert (gl[:, 7] & 0x80000000 == 0).all(), "a bucket is still flagged"
    assert np.array_equal(gl[:, :7], ol[:, :7]), "low counter words differ"
    bad = np.nonzero(gl[:, 7] != ol[:, 7])[0]
    assert bad.size == 0, f"word 7 (high id) differs at {bad.size} buckets, first {bad[:4]}: " \
                          f"{gl[bad[:4], 7]} vs {ol[bad[:4], 7]}"
    assert np.array_equal(high, orc.high), "high pools differ"
    st = sk.stats()
    assert st["next_level_id"] == orc.next_id, (st["next_level_id"], orc.next_id)
    assert st["dropped_keys"] == orc.dropped


def run_and_compare(sk, orc, keys_d, queries_d, pieces=None):
    if pieces is None:
        sk.insert(keys_d)
    else:
        off = 0
        for p in pieces:
            sk.insert(keys_d[off:off + p])
            off += p
        assert off == keys_d.numel()
    got = sk.search(queries_d).cpu().numpy()
    sk.sync()
    orc.insert(keys_d.cpu().numpy())
    want = orc.query(queries_d.cpu().numpy())
    mism = np.nonzero(got != want)[0]
    assert mism.size == 0, f"{mism.size} mismatches, first {mism[:5]}: got {got[mism[:5]]} want {want[mism[:5]]}"
    assert_same_tables(sk, orc)
    return got


def test_uniform_small(gpu):
    sk, orc = make_pair(65521, 1 << 12)
    keys = data.uniform_keys(1 << 20, seed=11)
    run_and_compare(sk, orc, keys, keys)


def test_uniform_config1_full_size(gpu):
    # 2^24 uniform keys into n_low = 262139 (src/test.cu:351), queries = all inserted keys
    sk, orc = make_pair(262139, 1 << 16)
    keys = data.uniform_keys(1 << 24, seed=1)
    run_and_compare(sk, orc, keys, keys)
    assert sk.stats()["linked_buckets"] == 0


@pytest.mark.parametrize("agg,route", [(1, 0), (2, 0), (3, 0), (3, 1), (3, 2), (3, 3)])
def test_zipf_heavy_links(gpu, agg, route):
    sk, orc = make_pair(16381, 1 << 15, aggregate=agg, route=route)
    keys = data.zipf_keys(1 << 22, 1 << 18, 1.1, seed=5, perm_seed=77)
    q = data.rank_keys(77, 0, 1 << 18)
    run_and_compare(sk, orc, keys, q)
    st = sk.stats()
    assert st["linked_buckets"] > 100 and st["repaired_buckets"] == st["linked_buckets"]


@pytest.mark.parametrize("lpk", [1, 2, 4, 8])
def test_fused_routing_every_group_width(gpu, lpk):
    # fused routing (the index word read by the counter atomic) with 1, 2, 4 or 8 lanes per
    # key: linked keys take their low increments back; tables equal the oracle's
    sk, orc = make_pair(16381, 1 << 15, aggregate=3, route=2, lanes_per_key=lpk, max_batch=1 << 19)
    keys = data.zipf_keys(1 << 21, 1 << 18, 1.1, seed=15, perm_seed=71)
    run_and_compare(sk, orc, keys, data.rank_keys(71, 0, 1 << 18))
    assert sk.stats()["linked_buckets"] > 100


def test_zipf_many_chunks_and_uneven_calls(gpu):
    sk, orc = make_pair(8191, 1 << 14, max_batch=1 << 16)
    keys = data.zipf_keys(3 * (1 << 18) + 77, 1 << 16, 1.2, seed=9, perm_seed=3)
    n = keys.numel()
    run_and_compare(sk, orc, keys, data.rank_keys(3, 0, 1 << 16), pieces=[1, 3, 5, 1000, 70001, n - 71010])


def test_compat_v3(gpu):
    sk, orc = make_pair(4093, 1 << 13, compat=True)
    keys = data.zipf_keys(1 << 21, 1 << 16, 1.0, seed=21, perm_seed=8)
    run_and_compare(sk, orc, keys, data.rank_keys(8, 0, 1 << 16))


def test_few_links_fused_routing(gpu):
    # a handful of heavy keys inside a uniform stream: after the first chunk links their
    # buckets, tiles run in the fused routing mode, where a linked key takes its low
    # increments back and counts in the high bucket
    sk, orc = make_pair(65521, 1 << 10, max_batch=1 << 18)
    uni = data.uniform_keys(1 << 21, seed=31).cpu().numpy()
    heavy = np.array([7, 11, 13, 1 << 31], np.uint32)
    keys = uni.copy()
    pos = np.arange(0, keys.size, 97)
    keys[pos] = heavy[np.arange(pos.size) % 4]
    q = np.concatenate([heavy, uni[:4096]])
    run_and_compare(sk, orc, torch.from_numpy(keys).cuda(), torch.from_numpy(q).cuda())
    assert sk.stats()["linked_buckets"] >= 4


def test_sketches_with_different_mask_tables_coexist(gpu):
    # a small-table sketch created after a large-table one must not break the first
    big = qs.generate_hashmask(16384, 32, 3, 4, 2)
    a = qs.Sketch_GPU_Sub_Warp_Level(4093, 8, 1024, 32, 1, 16384, hash_seed=12345, mask_table=big)
    b, orc_b = make_pair(4093, 1024)
    keys = data.zipf_keys(1 << 19, 1 << 12, 1.1, seed=3, perm_seed=5)
    a.insert(keys)
    b.insert(keys)
    a.sync()
    b.sync()
    orc_a = oracle.Msws(4093, 1024, 12345, big)
    hk = keys.cpu().numpy()
    orc_a.insert(hk)
    orc_b.insert(hk)
    q = data.rank_keys(5, 0, 1 << 12)
    assert np.array_equal(a.search(q).cpu().numpy(), orc_a.query(q.cpu().numpy()))
    assert np.array_equal(b.search(q).cpu().numpy(), orc_b.query(q.cpu().numpy()))


def test_single_heavy_key(gpu):
    sk, orc = make_pair(1021, 64)
    keys = torch.full((1 << 20,), 123456789, dtype=torch.uint32, device="cuda")
    got = run_and_compare(sk, orc, keys, keys[:1])
    assert got[0] == 1 << 20


def test_all_keys_one_bucket_many_masks(gpu):
    # n_low = 1: every key shares the bucket, so crossings depend on the exact order
    sk, orc = make_pair(1, 4, seed=1)
    keys = torch.arange(5000, dtype=torch.int64).remainder(37).to(torch.uint32).cuda()
    run_and_compare(sk, orc, keys, torch.arange(37, dtype=torch.int64).to(torch.uint32).cuda())


def test_unaligned_and_tiny_inputs(gpu):
    sk, orc = make_pair(4093, 1024)
    base = data.zipf_keys(200003, 5000, 1.3, seed=4, perm_seed=6)
    for lo, hi in [(1, 2), (1, 6), (3, 3), (5, 1030), (2, 150001), (7, 200003)]:
        sk.insert(base[lo:hi])
        orc.insert(base[lo:hi].cpu().numpy())
    sk.insert(base[:0])
    q = data.rank_keys(6, 0, 5000)
    assert np.array_equal(sk.search(q[1:]).cpu().numpy(), orc.query(q[1:].cpu().numpy()))
    assert sk.search(q[:0]).numel() == 0
    assert_same_tables(sk, orc)


@pytest.mark.parametrize("n_high,max_batch,n_ranks", [
    (8, 1 << 22, 1 << 12),     # few crossed buckets per chunk: one block links them
    (40, 1 << 22, 1 << 12),    # more than one block's warps of crossed buckets: grid-wide link order
    (1000, 1 << 16, 1 << 14),  # 2^16-key chunks: the pool runs out after several of them
    (600, 1 << 20, 1 << 16),   # hundreds of crossed buckets per chunk (sorted replay), pool runs out
])
def test_pool_exhaustion_matches_the_oracle(gpu, n_high, max_batch, n_ranks):
    """Which buckets still get a high bucket when the pool runs out is decided by the array
    order of their switching keys, as in the sequential insert: estimates, both tables, the
    allocator and the dropped-key count equal the oracle's."""
    sk, orc = make_pair(16381, n_high, max_batch=max_batch)
    keys = data.zipf_keys(1 << 21, n_ranks, 1.1, seed=12, perm_seed=13)
    q = data.rank_keys(13, 0, n_ranks)
    sk.insert(keys)
    got = sk.search(q).cpu().numpy()
    assert sk.status() == _lib.QS_ERR_POOL_FULL
    orc.insert(keys.cpu().numpy())
    assert orc.pool_full
    assert np.array_equal(got, orc.query(q.cpu().numpy()))
    assert_same_tables(sk, orc)


def test_pool_exhaustion_is_reported(gpu):
    sk, orc = make_pair(4093, 8)
    keys = data.zipf_keys(1 << 20, 1 << 12, 1.2, seed=1, perm_seed=2)
    sk.insert(keys)
    assert sk.status() == _lib.QS_ERR_POOL_FULL
    with pytest.raises(qs.QsError):
        sk.sync()
    st = sk.stats()
    assert st["linked_buckets"] == 7 and st["dropped_keys"] > 0
    orc.insert(keys.cpu().numpy())
    assert orc.pool_full and orc.next_id == 1024 + 8
    assert_same_tables(sk, orc)
    sk.reset_status()
    assert sk.status() == _lib.QS_OK


def test_clear_resets(gpu):
    sk, orc = make_pair(4093, 1 << 10)
    keys = data.zipf_keys(1 << 20, 1 << 12, 1.2, seed=1, perm_seed=2)
    sk.insert(keys)
    sk.clear()
    assert sk.stats()["next_level_id"] == 1025
    low, high = sk.tables()
    assert not low.any() and not high.any()
    run_and_compare(sk, orc, keys, data.rank_keys(2, 0, 1 << 12))


def test_host_buffers_match_device_path(gpu):
    sk, orc = make_pair(16381, 1 << 14, max_batch=1 << 18)
    keys = data.zipf_keys(1 << 21, 1 << 16, 1.1, seed=3, perm_seed=4)
    hk = keys.cpu().numpy()
    q = data.rank_keys(4, 0, 1 << 16).cpu().numpy()
    sk.insert_host(hk)
    got = sk.search_host(q)
    orc.insert(hk)
    assert np.array_equal(got, orc.query(q))
    pinned = torch.from_numpy(q).pin_memory()
    out = torch.empty_like(pinned).pin_memory()
    sk.search_host(pinned, out)
    assert np.array_equal(out.numpy(), got)


@pytest.mark.parametrize("agg,route", [(2, 0), (3, 1), (3, 2), (1, 2)])
def test_uniform_aggregation_and_routing_modes(gpu, agg, route):
    sk, orc = make_pair(65521, 1 << 12, aggregate=agg, route=route, mask_rng=5)
    keys = data.uniform_keys((1 << 21) + 5, seed=12)
    run_and_compare(sk, orc, keys[3:], keys[3:])


def test_zipf_config2_full_size(gpu):
    # 2^27 keys, Zipf s=1.1 over 2^24 ranks, 64 MB low table, 16 MB high pool
    sk, orc = make_pair(2097143, 1 << 17)
    keys = data.zipf_keys(1 << 27, 1 << 24, 1.1, seed=2024, perm_seed=99)
    q = data.rank_keys(99, 0, 1 << 24)
    sk.insert(keys)
    got = sk.search(q).cpu().numpy()
    sk.sync()
    orc.insert(keys.cpu().numpy(), threads=8)
    want = orc.query(q.cpu().numpy())
    assert np.array_equal(got, want)


def run_mixed(sk, orc, keys, batch, frac=0.9, threads=1):
    """Per batch: insert the first `frac` of it, then query the rest (configuration 3)."""
    ni = int(batch * frac)
    hk = keys.cpu().numpy()
    for b in range(keys.numel() // batch):
        sk.insert(keys[b * batch:b * batch + ni])
        got = sk.search(keys[b * batch + ni:(b + 1) * batch]).cpu().numpy()
        orc.insert(hk[b * batch:b * batch + ni], threads=threads)
        want = orc.query(hk[b * batch + ni:(b + 1) * batch])
        assert np.array_equal(got, want), f"batch {b}: {(got != want).sum()} estimates differ"


def test_mixed_interleaved_small(gpu):
    sk, orc = make_pair(65521, 1 << 13)
    run_mixed(sk, orc, data.zipf_keys(1 << 22, 1 << 22, 0.8, seed=41, perm_seed=42), 1 << 18)
    sk.sync()
    assert_same_tables(sk, orc)


def test_calls_that_reuse_each_others_buffers(gpu):
    # Back-to-back calls on one stream, where each kernel may be scheduled while the previous
    # one drains: a query's output is the next insert's keys, and a key buffer is overwritten
    # by a torch kernel between an insert and the next insert and query.
    sk, orc = make_pair(65521, 1 << 13)
    keys = data.zipf_keys(1 << 20, 1 << 16, 1.1, seed=51, perm_seed=52)
    out = torch.empty_like(keys)
    sk.insert(keys)
    orc.insert(keys.cpu().numpy())
    sk.search(keys, counts=out)
    sk.insert(out)  # the estimates, read as keys
    orc.insert(orc.query(keys.cpu().numpy()))
    buf = keys.clone()
    sk.insert(buf)
    buf.copy_(data.zipf_keys(1 << 20, 1 << 16, 1.1, seed=53, perm_seed=54))
    sk.insert(buf)
    got = sk.search(buf).cpu().numpy()
    sk.sync()
    orc.insert(keys.cpu().numpy())
    hb = buf.cpu().numpy()
    orc.insert(hb)
    want = orc.query(hb)
    assert np.array_equal(got, want), f"{(got != want).sum()} estimates differ"
    assert_same_tables(sk, orc)


def test_mixed_config3_full_size(gpu):
    # 2^28 operations in 2^20 batches (90 % inserts then 10 % queries), Zipf 0.8 over 2^26,
    # 256 MB low table (n_low = 8388593), 64 MB high pool
    sk, orc = make_pair(8388593, 1 << 19)
    run_mixed(sk, orc, data.zipf_keys(1 << 28, 1 << 26, 0.8, seed=1000, perm_seed=99), 1 << 20, threads=8)
    sk.sync()


@pytest.mark.parametrize("lpk", [1, 2, 4, 16, 32])
@pytest.mark.parametrize("agg", [1, 3])
def test_lanes_per_key_variants_bit_exact(gpu, lpk, agg):
    # Every pass-1 width gives the oracle's tables and estimates on a stream that links
    # thousands of buckets and repairs many chunks.
    sk, orc = make_pair(65521, 1 << 14, lanes_per_key=lpk, aggregate=agg, max_batch=1 << 18)
    keys = data.zipf_keys(1 << 21, 1 << 16, 1.1, seed=41, perm_seed=5)
    q = data.rank_keys(5, 0, 1 << 16)
    run_and_compare(sk, orc, keys, q)


@pytest.mark.parametrize("tile", [256, 512, 1024])
def test_keys_per_tile_bit_exact(gpu, tile):
    # smaller CTA tiles (and an unaligned start, so the ragged keys take CTA 0's path)
    sk, orc = make_pair(65521, 1 << 14, keys_per_tile=tile, max_batch=1 << 18)
    keys = data.zipf_keys((1 << 20) + 7, 1 << 16, 1.1, seed=45, perm_seed=7)
    run_and_compare(sk, orc, keys[3:], data.rank_keys(7, 0, 1 << 16))


@pytest.mark.parametrize("ctas", [1, 2])
def test_ctas_per_sm_bit_exact(gpu, ctas):
    sk, orc = make_pair(65521, 1 << 14, lanes_per_key=4, ctas_per_sm=ctas, max_batch=1 << 18)
    keys = data.zipf_keys(1 << 20, 1 << 16, 1.0, seed=43, perm_seed=6)
    run_and_compare(sk, orc, keys, keys[:1 << 16])


def test_autotune_picks_a_timed_setting_and_create_uses_it(gpu):
    from qsketch_b200 import autotune
    autotune.reset()
    keys = data.zipf_keys(1 << 22, 1 << 20, 1.1, seed=47, perm_seed=8)
    best, allc = autotune.autotune(524287, 1 << 15, keys, reps=2)
    print("autotune best:", best, "of", len(allc))
    assert len(allc) >= 10
    # the pick is within 1 % of the fastest setting timed: a setting replaces the incumbent only
    # when 1 % faster, and incumbents only get faster, so every rejected one was >= 0.99 x the pick
    assert best["insert_ms"] <= min(c["insert_ms"] for c in allc) / 0.99 * (1 + 1e-6)
    assert best in allc
    assert autotune.lookup(524287) == best
    assert autotune.lookup(300000) == best  # same size class (2^18 <= n < 2^19)
    # a sketch of that class with knobs left at 0 uses the tuned setting: same results
    tuned = qs.Sketch_GPU_Sub_Warp_Level(524287, 8, 1 << 15, 32, hash_seed=2654435769)
    plain = qs.Sketch_GPU_Sub_Warp_Level(524287, 8, 1 << 15, 32, hash_seed=2654435769, lanes_per_key=8,
                                         aggregate=3, route=1)
    tuned.insert(keys)
    plain.insert(keys)
    q = keys[:1 << 18]
    assert torch.equal(tuned.search(q), plain.search(q))
    autotune.reset()
    assert autotune.lookup(524287) is None


def test_autotune_keeps_a_fixed_chunk_size(gpu):
    # A caller that inserts in calls of one size passes it: only that chunk size is timed.
    from qsketch_b200 import autotune
    autotune.reset()
    keys = data.zipf_keys(1 << 21, 1 << 18, 1.1, seed=53, perm_seed=3)
    best, allc = autotune.autotune(65521, 1 << 13, keys, reps=1, max_batch=3 << 17)
    assert {c["max_batch"] for c in allc} == {3 << 17}
    with pytest.raises(qs.QsError):
        autotune.autotune(65521, 1 << 13, keys, reps=1, max_batch=1000)
    autotune.reset()


@pytest.mark.parametrize("ramp", [True, False])
def test_chunk_ramp_on_and_off_bit_exact(gpu, ramp):
    # After a clear the chunks grow from 2^18 keys (or not); both give the oracle's tables.
    sk, orc = make_pair(131071, 1 << 14, max_batch=1 << 21, chunk_ramp=ramp)
    keys = data.zipf_keys(3 << 20, 1 << 18, 1.2, seed=51, perm_seed=9)
    run_and_compare(sk, orc, keys, data.rank_keys(9, 0, 1 << 16), pieces=[1000, (1 << 20) - 1000, 2 << 20])
    sk.clear()
    orc2 = make_pair(131071, 1 << 14)[1]
    run_and_compare(sk, orc2, keys[:1 << 20], data.rank_keys(9, 0, 1 << 16))


def test_roofline_probes_report_rates(gpu):
    # The bench's denominators: random-sector atomics, loads, a streaming read and the replay's
    # grid barrier all return positive rates; invalid kinds are refused.
    for kind in (0, 1, 2, 3, 4, 5, 7):
        assert data.probe(kind, 64 << 20, 1 << 22) > 0
    assert data.probe(6, 64, 1000) > 1e4  # barriers per second
    with pytest.raises(qs.QsError):
        data.probe(9, 64 << 20)


def test_replay_with_more_records_than_resident_tiles(gpu):
    # One 2^23-key chunk over 2^17 distinct keys into 65521 buckets: about 128 keys per bucket,
    # so most buckets cross and nearly every key becomes a replay record (K > 296 x 4096): the
    # radix passes take the multi-tile-per-block path; the tables must still equal the oracle's.
    sk, orc = make_pair(65521, 1 << 16, max_batch=1 << 23, chunk_ramp=False)
    distinct = data.uniform_keys(1 << 17, seed=71)
    idx = torch.randint(0, 1 << 17, (1 << 23,), generator=torch.Generator().manual_seed(5)).cuda()
    keys = distinct.view(torch.int32)[idx].view(torch.uint32).contiguous()
    run_and_compare(sk, orc, keys, distinct)
    assert sk.stats()["repaired_keys"] > 296 * 4096


def test_replay_with_two_to_four_radix_tiles_per_block(gpu):
    # 2^22 distinct keys into 2039 buckets in one chunk: every bucket crosses, so nearly all
    # 4M keys become replay records (more than one and at most four 4096-record tiles per
    # block of the 296-block grid): the radix keeps per-tile offsets and ranks, reloads the
    # records for the scatter; the tables must equal the oracle's
    sk, orc = make_pair(2039, 1 << 12, max_batch=1 << 22, chunk_ramp=False)
    keys = data.uniform_keys(1 << 22, seed=73)
    run_and_compare(sk, orc, keys, keys[:1 << 16])
    rk = sk.stats()["repaired_keys"]
    assert 296 * 4096 < rk <= 4 * 296 * 4096, rk
