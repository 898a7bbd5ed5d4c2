"""Synthetic key streams and exact-count helpers on the device (for tests and the bench).

Streams stand in for the reference's cuRAND keys (include/tool/tool.h:391-418) and its
absent data/gpu_random.dat: uniform u32 keys from a seeded xorshift64* stream, and Zipf(s)
keys over n_ranks ranks (rejection-inversion sampling) mapped to distinct u32 keys by a
seeded bijection.
"""
import ctypes

import torch

from ._lib import check, lib


def _s(stream):
    return torch.cuda.current_stream().cuda_stream if stream is None else stream.cuda_stream


def uniform_keys(n, seed, device="cuda", stream=None):
    keys = torch.empty(n, dtype=torch.uint32, device=device)
    check(lib.qs_gen_keys(0, seed, 0, 0.0, 0, keys.data_ptr(), None, n, _s(stream)), "uniform_keys")
    return keys


def zipf_keys(n, n_ranks, s, seed, perm_seed, with_ranks=False, device="cuda", stream=None):
    keys = torch.empty(n, dtype=torch.uint32, device=device)
    ranks = torch.empty(n, dtype=torch.uint32, device=device) if with_ranks else None
    check(lib.qs_gen_keys(1, seed, n_ranks, float(s), perm_seed, keys.data_ptr(),
                          ranks.data_ptr() if ranks is not None else None, n, _s(stream)), "zipf_keys")
    return (keys, ranks) if with_ranks else keys


def class_keys(n, seed, perm_seed, n_class=1 << 16, s_class=1.0, s_suffix=1.2, device="cuda", stream=None):
    """class << 16 | suffix keys of the learned-split workload."""
    keys = torch.empty(n, dtype=torch.uint32, device=device)
    check(lib.qs_gen_class_keys(seed, n_class, float(s_class), float(s_suffix), perm_seed, keys.data_ptr(), n,
                                _s(stream)), "class_keys")
    return keys


def exact_counts(keys):
    """Distinct keys (ascending) and their exact counts (torch sort/unique on the device)."""
    u, c = torch.unique(keys.to(torch.int64), return_counts=True)
    return u.to(torch.uint32), c.to(torch.uint32)


def rank_keys(perm_seed, first, n, device="cuda", stream=None):
    """The distinct keys of ranks [first, first+n) of a zipf_keys stream."""
    keys = torch.empty(n, dtype=torch.uint32, device=device)
    check(lib.qs_gen_rank_keys(perm_seed, first, keys.data_ptr(), n, _s(stream)), "rank_keys")
    return keys


def rank_histogram(ranks, n_ranks, hist=None, stream=None):
    if hist is None:
        hist = torch.zeros(n_ranks, dtype=torch.uint32, device=ranks.device)
    check(lib.qs_rank_histogram(ranks.data_ptr(), ranks.numel(), hist.data_ptr(), n_ranks, _s(stream)),
          "rank_histogram")
    return hist


def error_metrics(est, exact, stream=None):
    """(mean |est-exact|/exact, mean est/exact) over entries with exact > 0."""
    rel, ratio = ctypes.c_double(), ctypes.c_double()
    check(lib.qs_error_metrics(est.data_ptr(), exact.data_ptr(), est.numel(), ctypes.byref(rel),
                               ctypes.byref(ratio), _s(stream)), "error_metrics")
    return rel.value, ratio.value


def probe(kind, nbytes, ops=1 << 26):
    r = ctypes.c_double()
    check(lib.qs_probe(kind, nbytes, ops, ctypes.byref(r)), "probe")
    return r.value
