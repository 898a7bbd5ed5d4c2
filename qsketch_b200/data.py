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


def uneven_streams(n_streams, seed, min_len=1 << 10, max_len=1 << 22, n_ranks=1 << 20, s_range=(0.6, 1.4),
                   min_bytes=32 << 10, max_bytes=16 << 20, pool_div=4, device="cuda", stream=None, key_seed=None):
    """The batched-streams workload: per stream a length and a sketch size drawn log-uniformly,
    a Zipf exponent drawn uniformly, and a Zipf key stream over n_ranks ranks under the
    stream's own seeded bijection.  Sketch of stream s: n_low = find_greatest_prime(bytes/32),
    high pool bytes/pool_div.  Returns a dict: keys (flat uint32), offsets (int64, n+1),
    lengths, s, n_low, n_high (numpy).  key_seed (default: seed) draws other keys for the same
    shapes (lengths, exponents, sketch sizes)."""
    import numpy as np

    from .sketch import find_greatest_prime
    rng = np.random.default_rng(seed)
    lengths = np.exp(rng.uniform(np.log(min_len), np.log(max_len), n_streams)).astype(np.int64)
    expo = rng.uniform(s_range[0], s_range[1], n_streams)
    nbytes = np.exp(rng.uniform(np.log(min_bytes), np.log(max_bytes), n_streams)).astype(np.int64)
    n_low = np.array([find_greatest_prime(int(b) // 32) for b in nbytes], np.uint64)
    n_high = np.maximum(2, nbytes // pool_div // 128).astype(np.uint64)
    offsets = np.zeros(n_streams + 1, np.int64)
    offsets[1:] = np.cumsum(lengths)
    keys = torch.empty(int(offsets[-1]), dtype=torch.uint32, device=device)
    ks = seed if key_seed is None else key_seed
    for i in range(n_streams):
        check(lib.qs_gen_keys(1, ks * 1000003 + i, n_ranks, float(expo[i]), ks * 7919 + i,
                              keys.data_ptr() + int(offsets[i]) * 4, None, int(lengths[i]), _s(stream)),
              "uneven_streams")
    return {"keys": keys, "offsets": torch.from_numpy(offsets).to(device), "lengths": lengths, "s": expo,
            "n_low": n_low, "n_high": n_high, "bytes": nbytes}
