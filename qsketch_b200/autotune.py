"""The insert autotuner over the C ABI (qs_autotune* in include/qsketch_c.h).

No counterpart in the reference, whose kernels have fixed launch shapes (<<<65536, 32>>>,
device_sketch_v3.h:587).  Pass-1 knobs — lanes per key (1, 2, 4, 8, 16, 32 over the fixed 32 B
bucket), duplicate-key aggregation, level routing, CTAs per SM and the chunk size — never
change results, only speed; qs_autotune times them on a sample and records the fastest for
the sketch's size class floor(log2(n_low)), which later sketches of that class use when
their knobs are left at 0.
"""
import ctypes

from ._lib import QS_KIND_MSWS, check, lib, qs_params, qs_tune_config
from .sketch import _ptr

_FIELDS = [f for f, _ in qs_tune_config._fields_]


def _as_dict(c):
    return {f: getattr(c, f) for f in _FIELDS}


def autotune(n_low, n_high, keys, reps=3, hash_seed=2654435769, mask_rng=1, max_all=64, **params):
    """Time the candidate settings on `keys` (a CUDA uint32 tensor); returns (best, all)."""
    p = qs_params()
    lib.qs_params_default(ctypes.byref(p))
    p.kind = QS_KIND_MSWS
    p.n_low, p.n_high, p.hash_seed, p.mask_rng = n_low, n_high, hash_seed, mask_rng
    for k, v in params.items():
        setattr(p, k, v)
    best = qs_tune_config()
    allc = (qs_tune_config * max_all)()
    n_all = ctypes.c_uint32()
    check(lib.qs_autotune(ctypes.byref(p), _ptr(keys, "keys"), keys.numel(), reps, ctypes.byref(best), allc,
                          max_all, ctypes.byref(n_all)), "autotune")
    return _as_dict(best), [_as_dict(allc[i]) for i in range(min(n_all.value, max_all))]


def lookup(n_low):
    """The recorded setting for n_low's size class, or None."""
    c = qs_tune_config()
    return _as_dict(c) if lib.qs_autotune_lookup(n_low, ctypes.byref(c)) == 0 else None


def reset():
    lib.qs_autotune_reset()
