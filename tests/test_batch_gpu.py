"""Batched uneven streams (qs_batch_*): every stream's query vector must equal, bit for bit,
that of the same stream inserted alone into its own sketch (same n_low, n_high, seed and
masks), whatever the window size, the order of streams or the launch form (eager or CUDA
graph).  A subset is also checked against the sequential CPU oracle."""
import numpy as np
import pytest
import torch

import oracle
import qsketch_b200 as qs
from qsketch_b200 import _lib, data
from qsketch_b200.batch import BatchedSketches

pytestmark = pytest.mark.gpu


def workload(n_streams, seed, max_len, n_ranks=1 << 12, max_bytes=1 << 20):
    # Small rank spaces and strong skew make many buckets cross 128 inside a window, so the
    # ordered replay runs for many streams at once.  A pool as large as the low table never
    # runs out (a bucket links at most once).
    w = data.uneven_streams(n_streams, seed, min_len=1 << 10, max_len=max_len, n_ranks=n_ranks,
                            s_range=(0.6, 1.4), min_bytes=32 << 10, max_bytes=max_bytes)
    w["n_high"] = w["n_low"] + 2
    return w


def alone(w, s, seed, queries=None, **kw):
    """Stream s inserted alone into a sketch of its own: estimates (of its keys, or of
    `queries`), status and tables."""
    lo, hi = int(w["offsets"][s]), int(w["offsets"][s + 1])
    mb = min(1 << 22, max(32, (hi - lo + 31) // 32 * 32))  # results do not depend on the chunk size
    sk = qs.Sketch_GPU_Sub_Warp_Level(int(w["n_low"][s]), 8, int(w["n_high"][s]), 32, hash_seed=int(seed),
                                      mask_rng=1, max_batch=mb, **kw)
    sk.insert(w["keys"][lo:hi])
    out = sk.search(w["keys"][lo:hi] if queries is None else queries)
    st = sk.status()
    tables = sk.tables()
    sk.close()
    return out, st, tables


def check_streams(b, w, got, streams=None, tables=True):
    """Every stream's estimates, pool status and low and high tables (all streams, or those in
    the set `tables`) equal those of the stream inserted alone — pool exhaustion included."""
    seeds = b.seeds()
    off = w["offsets"].cpu().numpy()
    sst = b.stream_status()
    for s in (range(b.n_streams) if streams is None else streams):
        want, st, (low, high) = alone(w, s, seeds[s])
        assert (st == _lib.QS_ERR_POOL_FULL) == bool(sst[s] & 1), f"stream {s}: pool status differs"
        g = got[off[s]:off[s + 1]]
        assert torch.equal(g, want), f"stream {s}: {(g != want).sum().item()} of {g.numel()} estimates differ"
        if tables is True or (tables and s in tables):
            bl, bh = b.stream_tables(s)
            assert np.array_equal(bl, low), f"stream {s}: low table differs"
            assert np.array_equal(bh, high), f"stream {s}: high pool differs"


@pytest.mark.parametrize("max_batch,lpk,first", [(1 << 16, 8, 0), (1 << 22, 8, 0), (1 << 18, 4, 0), (1 << 18, 16, 0),
                                                (1 << 14, 4, 1 << 10), (1 << 15, 4, 1 << 16), (1 << 22, 4, None)])
def test_batch_equals_each_stream_alone(gpu, max_batch, lpk, first):
    # first: the per-stream chunk ramp's first slice (0 = default, None = flat windows); small
    # windows split rounds and single streams across windows
    w = workload(64, seed=3, max_len=1 << 17)
    b = BatchedSketches(w["n_low"], w["n_high"], seed_rng=7, max_batch=max_batch, lanes_per_key=lpk,
                        first_chunk=first or 0, chunk_ramp=first is not None)
    b.insert(w["keys"], w["offsets"])
    got = b.search(w["keys"], w["offsets"])
    b.sync()
    info = b.info()
    assert info["streams_pool_full"] == 0
    check_streams(b, w, got)


def test_batch_against_oracle(gpu):
    w = workload(12, seed=5, max_len=1 << 15)
    b = BatchedSketches(w["n_low"], w["n_high"], seed_rng=9, max_batch=1 << 14)
    b.insert(w["keys"], w["offsets"])
    got = b.search(w["keys"], w["offsets"]).cpu().numpy()
    b.sync()
    masks = qs.generate_hashmask(1021, 32, 3, 4, 1)
    seeds = b.seeds()
    keys = w["keys"].cpu().numpy()
    off = w["offsets"].cpu().numpy()
    for s in range(12):
        orc = oracle.Msws(int(w["n_low"][s]), int(w["n_high"][s]), int(seeds[s]), masks)
        ks = keys[off[s]:off[s + 1]]
        orc.insert(ks)
        assert np.array_equal(got[off[s]:off[s + 1]], orc.query(ks)), f"stream {s} differs from the oracle"


def test_batch_order_of_streams_does_not_matter(gpu):
    # The same sketches fed in reverse stream order (and in two calls) give the same counts.
    w = workload(24, seed=8, max_len=1 << 16)
    b1 = BatchedSketches(w["n_low"], w["n_high"], seed_rng=4, max_batch=1 << 15)
    b1.insert(w["keys"], w["offsets"])
    ref = b1.search(w["keys"], w["offsets"])
    b1.sync()
    S = 24
    off = w["offsets"].cpu().numpy()
    order = list(range(S))[::-1]
    seeds = b1.seeds()[order]
    nl, nh = w["n_low"][order], w["n_high"][order]
    parts = [w["keys"][off[s]:off[s + 1]] for s in order]
    rkeys = torch.cat(parts)
    roff = torch.tensor(np.concatenate([[0], np.cumsum([p.numel() for p in parts])]), dtype=torch.int64,
                        device="cuda")
    b2 = BatchedSketches(nl, nh, hash_seeds=seeds, max_batch=1 << 15)
    half = [p[: p.numel() // 2] for p in parts]
    rest = [p[p.numel() // 2:] for p in parts]
    for piece in (half, rest):
        k = torch.cat(piece)
        o = torch.tensor(np.concatenate([[0], np.cumsum([p.numel() for p in piece])]), dtype=torch.int64,
                         device="cuda")
        b2.insert(k, o)
    got = b2.search(rkeys, roff)
    b2.sync()
    for j, s in enumerate(order):
        assert torch.equal(got[roff[j]:roff[j + 1]], ref[off[s]:off[s + 1]]), f"stream {s}"


def test_batch_graph_replay(gpu):
    # Record once, refill the same buffers with another batch, replay: equal to eager runs.
    w1 = workload(32, seed=11, max_len=1 << 15)
    w2 = workload(32, seed=12, max_len=1 << 15)
    n1, n2 = w1["keys"].numel(), w2["keys"].numel()
    cap = max(n1, n2)
    keys = torch.zeros(cap, dtype=torch.uint32, device="cuda")
    offs = torch.zeros(33, dtype=torch.int64, device="cuda")
    counts = torch.zeros(cap, dtype=torch.uint32, device="cuda")
    g = BatchedSketches(w1["n_low"], w1["n_high"], seed_rng=2, max_batch=1 << 20)
    e = BatchedSketches(w1["n_low"], w1["n_high"], seed_rng=2, max_batch=1 << 20)
    for w in (w1, w2):
        n = w["keys"].numel()
        keys[:n].copy_(w["keys"])
        offs.copy_(w["offsets"])
        g.insert_graph(keys, offs, max_total=cap)
        g.search_graph(keys, offs, counts, max_total=cap)
        e.insert(w["keys"], w["offsets"])
        want = e.search(w["keys"], w["offsets"])
        g.sync()
        e.sync()
        assert torch.equal(counts[:n], want)
    info = g.info()
    print("graph info:", info)
    assert info["graph_capture"] == 1 and info["graph_launches"] == 4


def test_batch_empty_streams_and_clear(gpu):
    w = workload(16, seed=21, max_len=1 << 14)
    lengths = w["lengths"].copy()
    off = w["offsets"].cpu().numpy()
    keep = np.ones(16, bool)
    keep[[0, 5, 6, 15]] = False  # empty first, middle run and last stream
    parts = [w["keys"][off[s]:off[s + 1]] for s in range(16) if keep[s]]
    lengths[~keep] = 0
    offs = torch.tensor(np.concatenate([[0], np.cumsum(lengths)]), dtype=torch.int64, device="cuda")
    keys = torch.cat(parts)
    b = BatchedSketches(w["n_low"], w["n_high"], seed_rng=3, max_batch=1 << 13)
    b.insert(keys, offs)
    got = b.search(keys, offs)
    b.sync()
    seeds = b.seeds()
    o = offs.cpu().numpy()
    for s in np.nonzero(keep)[0]:
        sk = qs.Sketch_GPU_Sub_Warp_Level(int(w["n_low"][s]), 8, int(w["n_high"][s]), 32, hash_seed=int(seeds[s]))
        sk.insert(w["keys"][off[s]:off[s + 1]])
        assert torch.equal(got[o[s]:o[s + 1]], sk.search(w["keys"][off[s]:off[s + 1]])), f"stream {s}"
    b.clear()
    b.insert(keys, offs)
    again = b.search(keys, offs)
    b.sync()
    assert torch.equal(again, got), "clear + reinsert differs"


def test_batch_bad_offsets_latch_invalid_arg(gpu):
    b = BatchedSketches([1021, 1021], [64, 64], seed_rng=1)
    keys = data.uniform_keys(1000, seed=1)
    offs = torch.tensor([0, 700, 500], dtype=torch.int64, device="cuda")
    b.insert(keys, offs, total=500)
    with pytest.raises(qs.QsError) as ei:
        b.sync()
    assert ei.value.status == _lib.QS_ERR_INVALID_ARG


def test_batch_pool_exhaustion_is_per_stream(gpu):
    # Stream 1: 40 distinct keys 300 times each into a sketch with a 4-bucket pool (3 links):
    # only it reports its pool full; the other streams stay bit-exact.
    w = workload(4, seed=31, max_len=1 << 15)
    off = w["offsets"].cpu().numpy()
    heavy = data.uniform_keys(40, seed=77).repeat(300)
    parts = [w["keys"][off[0]:off[1]], heavy, w["keys"][off[2]:off[3]], w["keys"][off[3]:off[4]]]
    keys = torch.cat(parts)
    offs = torch.tensor(np.concatenate([[0], np.cumsum([p.numel() for p in parts])]), dtype=torch.int64,
                        device="cuda")
    nh = w["n_high"].copy()
    nh[1] = 4
    b = BatchedSketches(w["n_low"], nh, seed_rng=5, max_batch=1 << 14)
    b.insert(keys, offs)
    got = b.search(keys, offs)
    assert b.status() == _lib.QS_ERR_POOL_FULL
    st = b.stream_status()
    assert st[1] & 1 and not (st[[0, 2, 3]] & 1).any(), st
    assert b.info()["streams_pool_full"] == 1
    w2 = {"keys": keys, "offsets": offs, "n_low": w["n_low"], "n_high": nh}
    check_streams(b, w2, got)  # the exhausted stream too: its links follow its own array order


def test_batch_uneven_streams_full_size(gpu):
    """The batched configuration at full size: 512 streams, lengths log-uniform in [2^10, 2^22]
    (~2.6e8 keys), per-stream Zipf s ~ U[0.6, 1.4] over 2^20 ranks, sketches log-uniform in
    [32 KB, 16 MB] with pools of bytes/4, so dozens of small sketches run out of high buckets.
    Every stream's estimates and pool status equal the stream inserted alone; tables are
    compared for every 8th stream and for every stream whose pool ran out."""
    w = data.uneven_streams(512, seed=1)
    b = BatchedSketches(w["n_low"], w["n_high"], seed_rng=7, lanes_per_key=4)
    b.insert(w["keys"], w["offsets"])
    got = b.search(w["keys"], w["offsets"])
    assert b.status() == _lib.QS_ERR_POOL_FULL
    full = np.nonzero(b.stream_status() & 1)[0]
    assert full.size > 10, "the workload is meant to exhaust some pools"
    check_streams(b, w, got, tables=set(range(0, 512, 8)) | set(full.tolist()))


def test_batch_per_size_class_lanes_per_key(gpu):
    # every size class with its own lanes per key (one pass-1 launch per run of classes): each
    # stream still equals the stream alone, tables included
    w = workload(48, seed=13, max_len=1 << 16)
    classes = sorted({int(np.floor(np.log2(float(n)))) for n in w["n_low"]})
    lpk = {c: [1, 2, 4, 8, 16, 32][i % 6] for i, c in enumerate(classes)}
    b = BatchedSketches(w["n_low"], w["n_high"], seed_rng=7, max_batch=1 << 18, class_lanes_per_key=lpk)
    b.insert(w["keys"], w["offsets"])
    got = b.search(w["keys"], w["offsets"])
    b.sync()
    check_streams(b, w, got)


def test_batch_autotune_picks_per_class_and_keeps_results(gpu):
    w = workload(32, seed=17, max_len=1 << 16)
    b = BatchedSketches(w["n_low"], w["n_high"], seed_rng=3, max_batch=1 << 19)
    picks = b.autotune(w["keys"], w["offsets"], reps=1)
    classes = {int(np.floor(np.log2(float(n)))) for n in w["n_low"]}
    assert set(picks) == classes and set(picks.values()) <= {1, 2, 4, 8, 16, 32}
    b.insert(w["keys"], w["offsets"])
    got = b.search(w["keys"], w["offsets"])
    b.sync()
    check_streams(b, w, got, tables=False)
