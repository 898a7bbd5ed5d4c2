"""qs_msws_insert_noalloc — the insert for callers that cannot allocate device memory.

Such callers (an engine that owns all device memory in a fixed arena and may not call
cudaMalloc/cudaFree while serving) keep the tables in their own memory; this entry point
takes them, plus the keys, and uses only a fixed scratch array inside the library.  The test
calls it through the C ABI twice in a row on the same tables and checks the tables against
the ones qs_insert builds from the same two key batches (bit-exact: low counter words,
linked buckets, high counters).  This file sorts last so that a run stopping at the first
failure has already run every other test; it also passes alone in a fresh process.
"""
import ctypes

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


def test_noalloc_insert_matches_qs_insert_on_two_calls(gpu):
    masks = qs.generate_hashmask(1021, 32, 3, 4, 3)
    d_masks = torch.from_numpy(masks.view(np.uint32).copy()).cuda()
    low = torch.zeros(N_LOW * 8, dtype=torch.uint32, device="cuda")
    high = torch.zeros(N_HIGH * 32, dtype=torch.uint32, device="cuda")
    state = torch.zeros(_lib.QS_MSWS_STATE_BYTES // 4, dtype=torch.uint32, device="cuda")
    batches = [data.zipf_keys(200003, 1 << 14, 1.1, seed=7, perm_seed=2),
               data.zipf_keys(_lib.QS_NOALLOC_MAX_KEYS, 1 << 14, 1.2, seed=8, perm_seed=2)]
    ref = qs.Sketch_GPU_Sub_Warp_Level(N_LOW, 8, N_HIGH, 32, hash_seed=SEED, mask_table=masks)
    stream = torch.cuda.current_stream().cuda_stream
    for keys in batches:
        st = _lib.lib.qs_msws_insert_noalloc(low.data_ptr(), N_LOW, high.data_ptr(), N_HIGH, state.data_ptr(),
                                             d_masks.data_ptr(), 1021, SEED, 0, keys.data_ptr(), keys.numel(),
                                             stream)
        assert st == _lib.QS_OK, _lib.lib.qs_last_error_string()
        ref.insert(keys)
        torch.cuda.synchronize()
        ref.sync()
        got = canonical(low.cpu().numpy(), high.cpu().numpy())
        want = canonical(*ref.tables())
        for g, w in zip(got, want):
            assert np.array_equal(g, w)
    assert int(state[1].item()) == 0  # no latched device status
    assert canonical(*ref.tables())[1].sum() > 10  # the batches did link buckets


def test_noalloc_rejects_sizes_beyond_its_scratch(gpu):
    big = _lib.QS_NOALLOC_MAX_KEYS + 1
    st = _lib.lib.qs_msws_insert_noalloc(256, N_LOW, 256, N_HIGH, 256, 256, 1021, SEED, 0, 256, big, None)
    assert st == _lib.QS_ERR_CAPACITY
    assert b"exceed the fixed scratch" in _lib.lib.qs_last_error_string()
    st = _lib.lib.qs_msws_insert_noalloc(256, _lib.QS_NOALLOC_MAX_BUCKETS + 1, 256, N_HIGH, 256, 256, 1021, SEED,
                                         0, 256, 16, None)
    assert st == _lib.QS_ERR_CAPACITY
