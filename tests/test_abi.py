"""CPU tests of the C ABI boundary: the library loads, exports every entry point the header
declares, and its host-side table preparation matches the reference (golden fixtures)."""
import ctypes
import json
import os
import re
import subprocess

import numpy as np
import pytest

import qsketch_b200 as qs
from qsketch_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "qsketch_c.h")
G = os.path.join(ROOT, "tests", "golden")
with open(os.path.join(G, "golden.json")) as f:
    GOLD = json.load(f)


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(qs_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_bound_api():
    assert set(declared_symbols()) == set(_lib.SIGNATURES)


def test_library_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (qs_[a-z0-9_]+)$", out, flags=re.M))
    missing = set(declared_symbols()) - exported
    assert not missing, missing
    for name in declared_symbols():
        assert getattr(_lib.lib, name) is not None


def test_abi_version_and_status_strings():
    assert _lib.lib.qs_abi_version() == 2
    for s in range(8):
        assert _lib.lib.qs_status_string(s)


def test_params_default_are_reference_defaults():
    p = _lib.qs_params()
    _lib.lib.qs_params_default(ctypes.byref(p))
    assert (p.kind, p.m_low, p.m_high, p.n_high, p.seed_sz, p.hash_mask_table_sz, p.hash_mask_ones) == \
        (0, 8, 32, 1024, 1, 1021, 3)


@pytest.mark.parametrize("case", GOLD["masks"], ids=lambda c: c["file"])
def test_product_hashmask_matches_reference(case):
    want = np.fromfile(os.path.join(G, case["file"]), np.uint8)
    got = qs.generate_hashmask(case["n"], case["m_bits"], case["ones"], case["padding"], case["rng_seed"])
    assert np.array_equal(got, want)


@pytest.mark.parametrize("case", GOLD["seeds"], ids=lambda c: str(c["rng_seed"]))
def test_product_seed_draw_matches_reference(case):
    assert [int(x) for x in qs.draw_seeds(len(case["values"]), case["rng_seed"])] == case["values"]


def test_product_primes_match_reference():
    for x, p in GOLD["primes"].items():
        assert qs.find_greatest_prime(int(x)) == p


def test_number_of_buckets():
    # device_sketch.h:371-376 with 3 ones: ((keys / factor) * 3) / m, then the prime below
    assert qs.number_of_buckets(1 << 20, 8, 1.0) == qs.find_greatest_prime((1 << 20) * 3 // 8)
    assert qs.number_of_buckets(1 << 27, 8, 0.5) == qs.find_greatest_prime((1 << 28) * 3 // 8)
    assert qs.Sketch_GPU_Thread.number_of_buckets(1 << 24, 3, 1.0) == 16777213


def test_bad_arguments_are_errors_not_crashes():
    assert _lib.lib.qs_generate_hashmask(1, 10, 8, 9, 0, None) == _lib.QS_ERR_INVALID_ARG
    assert _lib.lib.qs_insert(None, None, 10, None) == _lib.QS_ERR_INVALID_ARG
    assert _lib.lib.qs_query(None, None, 10, None, None) == _lib.QS_ERR_INVALID_ARG
    assert _lib.lib.qs_destroy(None) == _lib.QS_OK
    assert _lib.lib.qs_create(None, None) == _lib.QS_ERR_INVALID_ARG


def test_create_without_device_reports_no_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(qs.QsError) as ei:
        qs.Sketch_GPU_Sub_Warp_Level(262139)
    assert ei.value.status in (_lib.QS_ERR_NO_DEVICE, _lib.QS_ERR_CUDA)


def test_batch_bad_arguments_are_errors():
    from qsketch_b200._lib import qs_batch_params
    p = qs_batch_params()
    _lib.lib.qs_batch_params_default(ctypes.byref(p))
    assert p.hash_mask_table_sz == 1021 and p.hash_mask_ones == 3 and p.max_batch == 1 << 22
    h = ctypes.c_void_p()
    assert _lib.lib.qs_batch_create(ctypes.byref(p), ctypes.byref(h)) == _lib.QS_ERR_INVALID_ARG  # 0 streams
    nl = np.array([1021, 0], np.uint64)
    nh = np.array([64, 64], np.uint64)
    p.n_streams, p.n_low, p.n_high = 2, nl.ctypes.data, nh.ctypes.data
    assert _lib.lib.qs_batch_create(ctypes.byref(p), ctypes.byref(h)) == _lib.QS_ERR_INVALID_ARG  # n_low 0
    nl[1] = 509
    nh[1] = 1
    assert _lib.lib.qs_batch_create(ctypes.byref(p), ctypes.byref(h)) == _lib.QS_ERR_INVALID_ARG  # n_high < 2
    assert _lib.lib.qs_batch_insert(None, None, None, 10, None) == _lib.QS_ERR_INVALID_ARG
    assert _lib.lib.qs_batch_query(None, None, None, 10, None, None) == _lib.QS_ERR_INVALID_ARG
    assert _lib.lib.qs_batch_destroy(None) == _lib.QS_OK


def test_autotune_table_empty_and_bad_arguments():
    from qsketch_b200 import autotune
    autotune.reset()
    assert autotune.lookup(1 << 20) is None
    assert _lib.lib.qs_autotune(None, None, 0, 1, None, None, 0, None) == _lib.QS_ERR_INVALID_ARG
    # a fixed chunk size must be a multiple of 32 and at most 2^26; rejected before any device
    # work (the key pointer is never dereferenced)
    p = _lib.qs_params()
    _lib.lib.qs_params_default(ctypes.byref(p))
    p.n_low = 1021
    best = _lib.qs_tune_config()
    for mb in (1000, 1 << 27):
        p.max_batch = mb
        assert _lib.lib.qs_autotune(ctypes.byref(p), ctypes.c_void_p(256), 1024, 1, ctypes.byref(best), None, 0,
                                    None) == _lib.QS_ERR_INVALID_ARG


def test_knob_validation_happens_before_any_device_work():
    # lanes_per_key outside {0, 4, 8, 16, 32} is rejected; without a GPU the device check
    # comes first, so only check that an invalid value never reports success.
    p = _lib.qs_params()
    _lib.lib.qs_params_default(ctypes.byref(p))
    p.n_low, p.lanes_per_key = 1021, 12
    h = ctypes.c_void_p()
    assert _lib.lib.qs_create(ctypes.byref(p), ctypes.byref(h)) != _lib.QS_OK


def test_snapshot_load_refuses_bad_input_without_a_device(tmp_path):
    # header, size and checksum checks run on the host before any device work
    import ctypes
    h = ctypes.c_void_p()
    bogus = tmp_path / "bogus.qsk"
    bogus.write_bytes(b"QSKSNAP\0" + bytes(200))
    assert _lib.lib.qs_load(str(bogus).encode(), -1, ctypes.byref(h)) == _lib.QS_ERR_INVALID_ARG
    assert _lib.lib.qs_load(str(tmp_path / "missing.qsk").encode(), -1, ctypes.byref(h)) == _lib.QS_ERR_INVALID_ARG
    assert _lib.lib.qs_snapshot_load(b"short", 5, -1, ctypes.byref(h)) == _lib.QS_ERR_INVALID_ARG
