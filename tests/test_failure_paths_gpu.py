"""Failure paths that a healthy run never reaches, made to happen without faulting the GPU.

* A bounded device wait that runs out: a grid-wide barrier of the ordered replay's form that
  one block never reaches (qs_probe kind 8, waits bounded to a few milliseconds).  The waits
  must give up, latch the timeout and return QS_ERR_TIMEOUT, and the context must stay usable.
* A device allocation that fails inside qs_create (injected on the host by
  qs_test_fail_allocations): QS_ERR_OOM, with everything the create had allocated freed.
"""
import ctypes

import numpy as np
import pytest
import torch

import oracle
import qsketch_b200 as qs
from qsketch_b200 import _lib, data

pytestmark = pytest.mark.gpu


def small_round_trip():
    masks = qs.generate_hashmask(1021, 32, 3, 4, 1)
    sk = qs.Sketch_GPU_Sub_Warp_Level(4093, 8, 1 << 10, 32, hash_seed=2654435769, mask_table=masks)
    keys = data.zipf_keys(1 << 18, 1 << 12, 1.2, seed=3, perm_seed=4)
    sk.insert(keys)
    q = data.rank_keys(4, 0, 1 << 12)
    got = sk.search(q).cpu().numpy()
    sk.sync()
    orc = oracle.Msws(4093, 1 << 10, 2654435769, masks)
    orc.insert(keys.cpu().numpy())
    assert np.array_equal(got, orc.query(q.cpu().numpy()))


def test_bounded_barrier_wait_times_out_and_the_context_survives(gpu):
    r = ctypes.c_double()
    st = _lib.lib.qs_probe(8, 0, 1 << 14, ctypes.byref(r))
    assert st == _lib.QS_ERR_TIMEOUT, _lib.lib.qs_last_error_string()
    assert b"gave up" in _lib.lib.qs_last_error_string()
    # the same barrier with every block arriving completes, and the sketch path still works
    assert _lib.lib.qs_probe(6, 0, 64, ctypes.byref(r)) == _lib.QS_OK and r.value > 0
    small_round_trip()


@pytest.mark.parametrize("after", [0, 3, 9, 14])
def test_injected_allocation_failure_returns_oom_and_frees(gpu, after):
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    _lib.lib.qs_test_fail_allocations(after)
    try:
        with pytest.raises(qs.QsError) as ei:
            qs.Sketch_GPU_Sub_Warp_Level(65521, 8, 1 << 12, 32, hash_seed=2654435769, max_batch=1 << 20)
    finally:
        _lib.lib.qs_test_fail_allocations(-1)
    assert ei.value.status == _lib.QS_ERR_OOM
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert abs(free0 - free1) < (2 << 20), f"{free0 - free1} bytes not returned"
    small_round_trip()
