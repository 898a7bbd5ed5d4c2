"""CPU tests of the oracle: pinned against the reference's own code (golden fixtures made by
tests/golden/make_golden.py from oracle/_ref) and hand-worked known-answer cases of the
device_sketch_v3.h semantics."""
import json
import os

import numpy as np
import pytest

import oracle

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
with open(os.path.join(G, "golden.json")) as f:
    GOLD = json.load(f)


@pytest.mark.parametrize("case", GOLD["masks"], ids=lambda c: c["file"])
def test_hashmask_matches_reference(case):
    want = np.fromfile(os.path.join(G, case["file"]), np.uint8)
    got = oracle.generate_hashmask(case["rng_seed"], case["n"], case["m_bits"], case["ones"], case["padding"])
    assert np.array_equal(got, want)
    # every mask has exactly `ones` bits, all below m - padding (lib/hashmask.cu:61-77)
    mb = (case["m_bits"] + 7) // 8
    for i in range(case["n"]):
        v = int.from_bytes(bytes(want[i * mb:(i + 1) * mb]), "little")
        assert bin(v).count("1") == case["ones"]
        assert v >> (case["m_bits"] - case["padding"]) == 0


@pytest.mark.parametrize("case", GOLD["seeds"], ids=lambda c: str(c["rng_seed"]))
def test_seed_draw_matches_reference(case):
    got = oracle.draw_seeds(case["rng_seed"], len(case["values"]))
    assert [int(x) for x in got] == case["values"]
    assert all(1 <= v <= 0xFFFFFFFF for v in case["values"])


def test_primes_match_reference():
    for x, p in GOLD["primes"].items():
        assert oracle.find_greatest_prime(int(x)) == p, x


def test_exact_counts_match_reference_unordered_map():
    e = GOLD["exact"]
    keys = np.fromfile(os.path.join(G, e["keys"]), np.uint32)
    queries = np.fromfile(os.path.join(G, e["queries"]), np.uint32)
    want = np.fromfile(os.path.join(G, e["counts"]), np.uint32)
    assert np.array_equal(oracle.exact_counts(keys, queries), want)


def test_reference_lib_when_present():
    r = oracle.ref_lib()
    if r is None:
        pytest.skip("oracle/_ref not built")
    for seed in (3, 77, 4242):
        a = np.zeros(1021 * 4, np.uint8)
        r.ref_generate_hashmask(seed, 1021, 32, 3, 4, a.ctypes.data)
        assert np.array_equal(a, oracle.generate_hashmask(seed))


# ---- hand-worked known answers (n_low = 1, seed = 1 so key k uses mask k % H) -------------

MASKS = np.array([0b111, 0b11100, (1 << 8) | (1 << 16) | (1 << 24), (1 << 5) | (1 << 26) | (1 << 27)],
                 np.uint32).view(np.uint8)


def one_bucket(compat=False, n_high=4):
    return oracle.Msws(1, n_high, 1, MASKS, compat_v3=compat)


@pytest.mark.parametrize("c", [1, 2, 128, 129, 130, 131, 500])
def test_kat_single_key_is_exact(c):
    # counters 0,1,2 climb to 129 (128 is not > 128, device_sketch_v3.h:160); the 130th key
    # sees 129 > 128, links id 1025 and counts in the high bucket from then on.
    s = one_bucket()
    s.insert(np.zeros(c, np.uint32))
    assert s.query([0])[0] == c
    lo = min(c, 129)
    assert s.low[0] == lo | (lo << 8) | (lo << 16)
    if c >= 130:
        assert s.low[7] == 1025 and s.next_id == 1026
        assert list(s.high[32:35]) == [c - 129] * 3
    else:
        assert s.low[7] == 0 and s.next_id == 1025


def test_kat_compat_v3_linking_key_lands_on_bit_mod_8():
    # key 2 selects counters 8, 16, 24.  Its 130th insert links the bucket; device_sketch_v3.h
    # :187 adds that key's increments at high[stid] = high[bit % 8] = high[0] (three times).
    paper, compat = one_bucket(), one_bucket(compat=True)
    for s in (paper, compat):
        s.insert(np.full(131, 2, np.uint32))
    assert paper.query([2])[0] == 131
    assert compat.query([2])[0] == 130
    assert compat.high[32 + 0] == 3 and list(compat.high[32 + 8:32 + 25:8]) == [1, 1, 1]
    assert list(paper.high[32 + 8:32 + 25:8]) == [2, 2, 2] and paper.high[32] == 0


def test_kat_order_changes_tables_not_these_answers():
    a, b = one_bucket(), one_bucket()
    a.insert(np.r_[np.zeros(129, np.uint32), [1]])      # key 1 sees counter 2 at 129 -> links
    b.insert(np.r_[[1], np.zeros(129, np.uint32)])      # key 0's 129th sees counter 2 at 129 -> links
    for s in (a, b):
        assert list(s.query([0, 1])) == [129, 1]
    assert a.low[0] == 129 | 129 << 8 | 129 << 16 and a.low[1] == 0
    assert b.low[0] == 128 | 128 << 8 | 129 << 16 | 1 << 24 and b.low[1] == 1
    assert list(a.high[32:37]) == [0, 0, 1, 1, 1]
    assert list(b.high[32:37]) == [1, 1, 1, 0, 0]


def test_kat_pool_exhaustion_saturates():
    # n_high = 2 holds one link (index 1); a second bucket that needs one saturates.
    s = oracle.Msws(2, 2, 1, MASKS)
    k0 = np.zeros(131, np.uint32)               # bucket 0 (key 0 -> hv 0 -> bucket 0)
    k1 = np.full(140, 3, np.uint32)             # key 3 -> bucket 1, mask 3
    s.insert(np.r_[k0, k1])
    assert s.query([0])[0] == 131
    assert s.low[8 + 7] == oracle.SATURATED and s.pool_full
    assert s.dropped == 140 - 129 and s.query([3])[0] == 129


def test_mt_insert_equals_sequential():
    rng = np.random.default_rng(3)
    keys = (rng.zipf(1.2, 300000) % 50000).astype(np.uint32) * np.uint32(2654435761)
    masks = oracle.generate_hashmask(11)
    a = oracle.Msws(4093, 4096, 2654435769, masks)
    b = oracle.Msws(4093, 4096, 2654435769, masks)
    a.insert(keys)
    b.insert(keys, threads=4)
    q = np.unique(keys)
    assert np.array_equal(a.query(q), b.query(q))
    assert np.array_equal(a.low.reshape(-1, 8)[:, :7], b.low.reshape(-1, 8)[:, :7])
    assert ((a.low[7::8] > 1024) == (b.low[7::8] > 1024)).all()


def test_msws_estimates_never_under_count():
    rng = np.random.default_rng(4)
    keys = (rng.zipf(1.1, 200000) % 30000).astype(np.uint32) * np.uint32(40503)
    s = oracle.Msws(1021, 2048, 2654435769, oracle.generate_hashmask(5))
    s.insert(keys)
    q = np.unique(keys)
    est, exact = s.query(q), oracle.exact_counts(keys, q)
    assert (est >= exact).all()
    rel, ratio = oracle.error_metrics(est, exact)
    assert rel >= 0 and ratio >= 1.0


def test_count_min_kat():
    cm = oracle.CountMin(7, [1, 3])
    cm.insert([0, 7, 1, 1])    # row0: cols 0,0,1,1 ; row1: cols 0,0(21%7),3,3
    assert list(cm.table[:7]) == [2, 2, 0, 0, 0, 0, 0]
    assert list(cm.table[7:]) == [2, 0, 0, 2, 0, 0, 0]
    assert list(cm.query([0, 1, 2])) == [2, 2, 0]


# ---- REMOVE (deletion as the insertion with a subtraction, doc/main.tex:232) -------------

def test_kat_remove_low_level_floors_at_zero():
    s = one_bucket()
    s.insert(np.zeros(5, np.uint32))
    s.remove(np.zeros(2, np.uint32))
    assert s.query([0])[0] == 3 and s.low[0] == 3 | 3 << 8 | 3 << 16
    s.remove(np.zeros(10, np.uint32))  # more removals than insertions: counters stop at 0
    assert s.query([0])[0] == 0 and s.low[0] == 0


def test_kat_remove_linked_bucket_takes_from_the_high_level():
    s = one_bucket()
    s.insert(np.zeros(200, np.uint32))  # links at the 130th key: low 129, high 71
    s.remove(np.zeros(20, np.uint32))
    assert s.low[0] == 129 | 129 << 8 | 129 << 16 and list(s.high[32:35]) == [51] * 3
    assert s.query([0])[0] == 180
    s.remove(np.zeros(100, np.uint32))  # the high counters floor at 0, the low ones stay
    assert list(s.high[32:35]) == [0] * 3 and s.query([0])[0] == 129 and s.low[7] == 1025


def test_kat_remove_in_a_saturated_bucket_is_dropped():
    s = oracle.Msws(2, 2, 1, MASKS)
    s.insert(np.r_[np.zeros(131, np.uint32), np.full(140, 3, np.uint32)])
    d = s.dropped
    low = s.low.copy()
    s.remove(np.full(7, 3, np.uint32))
    assert s.dropped == d + 7 and np.array_equal(s.low, low)


def test_remove_within_a_call_is_order_independent():
    rng = np.random.default_rng(5)
    masks = oracle.generate_hashmask(3)
    keys = (rng.zipf(1.3, 200000) % 20000).astype(np.uint32) * np.uint32(2654435761)
    rem = (rng.zipf(1.3, 150000) % 30000).astype(np.uint32) * np.uint32(2654435761)
    a, b = (oracle.Msws(1021, 1024, 2654435769, masks) for _ in range(2))
    for s, r in ((a, rem), (b, rng.permutation(rem))):
        s.insert(keys)
        s.remove(r)
    assert np.array_equal(a.low, b.low) and np.array_equal(a.high, b.high)
    assert (a.low.reshape(-1, 8)[:, 7] > 1024).any()


def test_count_min_remove_floors_at_zero():
    seeds, n = [3, 5, 7], 101
    cm = oracle.CountMin(n, seeds)
    cm.insert(np.array([1, 1, 2], np.uint32))
    cm.remove(np.array([1, 9, 9], np.uint32))
    want = np.zeros(3 * n, np.int64)
    for k, d in ((1, 1), (1, 1), (2, 1), (1, -1), (9, -1), (9, -1)):  # device_sketch_v0.h:48-52
        for j, sd in enumerate(seeds):
            c = j * n + (k * sd % (1 << 32)) % n
            want[c] = max(0, want[c] + d)
    assert np.array_equal(cm.table, want.astype(np.uint32)) and cm.query([1])[0] == 1


def test_bucket_sketch_kat():
    # one bucket of 8 counters, one mask {1, 4, 6}: three inserts of key 5, one removal
    mt = np.array([(1 << 1) | (1 << 4) | (1 << 6)], np.uint8)
    s = oracle.BucketSketch(1, 8, 1, mt)
    s.insert(np.full(3, 5, np.uint32))
    s.remove(np.array([5, 9], np.uint32))  # key 9 has the same bucket and mask
    assert list(s.table) == [0, 1, 0, 0, 1, 0, 1, 0] and s.query([5])[0] == 1
