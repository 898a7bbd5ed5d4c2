"""qs_msws_insert_noalloc — the insert for callers that cannot allocate device memory.

Such callers (an engine that owns all device memory in a fixed arena and may not call
cudaMalloc/cudaFree while serving) keep the tables in their own memory; this entry point
takes them, plus the keys, and uses only a fixed scratch array inside the library.  The tests
call it through the C ABI on the same tables several times in a row and check the tables
against the ones qs_insert builds from the same key batches (bit-exact: low counter words,
linked buckets, high counters).  This file sorts last so that a run stopping at the first
failure has already run every other test; it also passes alone in a fresh process.
"""
import numpy as np
import pytest
import torch

import qsketch_b200 as qs
from qsketch_b200 import _lib, data

pytestmark = pytest.mark.gpu

N_LOW, N_HIGH, SEED = 16381, 1 << 13, 2654435769


def canonical(low, high):
    lw = low.reshape(-1, 8)
    ptr = lw[:, 7]
    linked = ptr > 1024
    hb = high.reshape(-1, 32)[ptr[linked] - 1024] if linked.any() else np.zeros((0, 32), np.uint32)
    return lw[:, :7].copy(), linked, ptr == 2, hb


def run_both(masks, n_masks, n_low, n_high, batches, compat_v3=False):
    """Insert each batch through qs_msws_insert_noalloc (caller-owned tables) and through
    qs_insert, comparing the tables after every call; returns the qs_insert sketch and the
    number of buckets each call replayed in stream order."""
    d_masks = torch.from_numpy(masks.view(np.uint32).copy()).cuda()
    low = torch.zeros(n_low * 8, dtype=torch.uint32, device="cuda")
    high = torch.zeros(n_high * 32, dtype=torch.uint32, device="cuda")
    state = torch.zeros(_lib.QS_MSWS_STATE_BYTES // 4, dtype=torch.uint32, device="cuda")
    ref = qs.Sketch_GPU_Sub_Warp_Level(n_low, 8, n_high, 32, n_hash_mask_table=n_masks, hash_seed=SEED,
                                       mask_table=masks, compat_v3=compat_v3)
    stream = torch.cuda.current_stream().cuda_stream
    flags = _lib.QS_FLAG_COMPAT_V3 if compat_v3 else 0
    replayed, before = [], 0
    for keys in batches:
        st = _lib.lib.qs_msws_insert_noalloc(low.data_ptr(), n_low, high.data_ptr(), n_high, state.data_ptr(),
                                             d_masks.data_ptr(), n_masks, SEED, flags, keys.data_ptr(),
                                             keys.numel(), stream)
        assert st == _lib.QS_OK, _lib.lib.qs_last_error_string()
        ref.insert(keys)
        torch.cuda.synchronize()
        ref.sync()
        got_low, got_high = low.cpu().numpy(), high.cpu().numpy()
        want_low, want_high = ref.tables()
        for g, w in zip(canonical(got_low, got_high), canonical(want_low, want_high)):
            assert np.array_equal(g, w)
        # high ids follow the array order of the switching keys on both paths: word for word
        assert np.array_equal(got_low, want_low) and np.array_equal(got_high, want_high)
        after = ref.stats()["repaired_buckets"]
        replayed.append(after - before)
        before = after
    assert int(state[1].item()) == 0  # no latched device status
    return ref, replayed


@pytest.mark.parametrize("n_masks,compat_v3", [(1021, False), (1021, True), (4093, False)])
def test_noalloc_insert_matches_qs_insert_on_two_calls(gpu, n_masks, compat_v3):
    masks = qs.generate_hashmask(n_masks, 32, 3, 4, 3)
    batches = [data.zipf_keys(200003, 1 << 14, 1.1, seed=7, perm_seed=2),
               data.zipf_keys(_lib.QS_NOALLOC_MAX_KEYS, 1 << 14, 1.2, seed=8, perm_seed=2)]
    ref, _ = run_both(masks, n_masks, N_LOW, N_HIGH, batches, compat_v3)
    assert canonical(*ref.tables())[1].sum() > 10  # the batches did link buckets


def test_noalloc_more_crossed_buckets_than_its_totals_slots(gpu):
    """One mask for every key (counters 0, 5, 9) and ~52 keys per bucket per call: the third
    call takes ~5000 buckets across the 8-bit threshold at once, more than the 4096 slots whose
    counter totals the fixed scratch computes grid-wide, so the rest take the fallback path."""
    mask = np.uint32((1 << 0) | (1 << 5) | (1 << 9))
    masks = np.full(1021, mask, np.uint32).view(np.uint8).copy()
    n_low = 5003
    batches = [data.uniform_keys(_lib.QS_NOALLOC_MAX_KEYS, seed=11 + i) for i in range(3)]
    _, replayed = run_both(masks, 1021, n_low, n_low + 2, batches)
    assert replayed[-1] > 4096


def test_noalloc_rejects_sizes_beyond_its_scratch(gpu):
    big = _lib.QS_NOALLOC_MAX_KEYS + 1
    st = _lib.lib.qs_msws_insert_noalloc(256, N_LOW, 256, N_HIGH, 256, 256, 1021, SEED, 0, 256, big, None)
    assert st == _lib.QS_ERR_CAPACITY
    assert b"exceed the fixed scratch" in _lib.lib.qs_last_error_string()
    st = _lib.lib.qs_msws_insert_noalloc(256, _lib.QS_NOALLOC_MAX_BUCKETS + 1, 256, N_HIGH, 256, 256, 1021, SEED,
                                         0, 256, 16, None)
    assert st == _lib.QS_ERR_CAPACITY
    # a state block that is 4- but not 16-byte aligned is refused before any launch
    st = _lib.lib.qs_msws_insert_noalloc(256, N_LOW, 256, N_HIGH, 260, 256, 1021, SEED, 0, 256, 16, None)
    assert st == _lib.QS_ERR_INVALID_ARG
    assert b"16-byte aligned" in _lib.lib.qs_last_error_string()
