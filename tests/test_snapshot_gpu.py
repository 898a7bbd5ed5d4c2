"""Snapshots (qs_save / qs_load, qs_snapshot_save / qs_snapshot_load): the reference declares
read_file / write_file (include/qsketch.h:70-71) and never defines them.  A sketch restored
from a snapshot answers every query as the saved one and, fed the same further keys,
continues word for word as the saved sketch does (MSWS with linked buckets and an exhausted
pool, count-min); a damaged snapshot is refused before any device work."""
import numpy as np
import pytest

import qsketch_b200 as qs
from qsketch_b200 import _lib, data

pytestmark = pytest.mark.gpu


def test_msws_snapshot_round_trip_continues_identically(gpu, tmp_path):
    masks = qs.generate_hashmask(1021, 32, 3, 4, 7)
    a = qs.Sketch_GPU_Sub_Warp_Level(16381, 8, 300, 32, hash_seed=2654435769, mask_table=masks, compat_v3=True)
    k1 = data.zipf_keys(1 << 20, 1 << 14, 1.1, seed=5, perm_seed=6)
    a.insert(k1)
    assert a.status() == _lib.QS_ERR_POOL_FULL  # an exhausted pool travels too
    path = tmp_path / "msws.qsk"
    a.save(path)
    b = qs.load(path)
    c = qs.from_snapshot(a.snapshot())
    q = data.rank_keys(6, 0, 1 << 14)
    ref = a.search(q).cpu().numpy()
    for s in (b, c):
        assert isinstance(s, qs.Sketch_GPU_Sub_Warp_Level)
        assert np.array_equal(s.search(q).cpu().numpy(), ref)
        sa, sb = a.stats(), s.stats()
        for f in ("status_bits", "next_level_id", "linked_buckets", "dropped_keys"):
            assert sa[f] == sb[f], f
    k2 = data.zipf_keys(1 << 20, 1 << 14, 1.1, seed=7, perm_seed=6)
    for s in (a, b):
        s.insert(k2)
        s.remove(k1[: 1 << 16])
    la, ha = a.tables()
    lb, hb = b.tables()
    assert np.array_equal(la, lb) and np.array_equal(ha, hb)
    assert np.array_equal(a.search(q).cpu().numpy(), b.search(q).cpu().numpy())


def test_count_min_snapshot_round_trip(gpu, tmp_path):
    a = qs.Sketch_GPU_Thread(65521, 4, seed_rng=9)
    a.insert(data.uniform_keys(1 << 20, seed=3))
    b = qs.from_snapshot(a.snapshot())
    assert isinstance(b, qs.Sketch_GPU_Thread)
    q = data.uniform_keys(1 << 16, seed=3)
    assert np.array_equal(a.search(q).cpu().numpy(), b.search(q).cpu().numpy())
    assert np.array_equal(a.info()["seeds"], b.info()["seeds"])


def test_damaged_snapshot_is_refused(gpu):
    a = qs.Sketch_GPU_Sub_Warp_Level(4093, 8, 1024, 32, hash_seed=12345)
    a.insert(data.uniform_keys(1 << 16, seed=1))
    snap = bytearray(a.snapshot())
    for bad in (bytes(snap[:50]), bytes(snap[:-1]), bytes(snap[:200] + bytes([snap[200] ^ 1]) + snap[201:])):
        with pytest.raises(qs.QsError) as ei:
            qs.from_snapshot(bad)
        assert ei.value.status == _lib.QS_ERR_INVALID_ARG
