"""CPU oracle for the QSketch insert/query path — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs use this
package, as the checker.  It wraps oracle/liboracle.so (built from oracle.cpp by
oracle/Makefile) and, when present, oracle/_ref/libqsref.so built from the reference's own
library sources.  Parity status: the oracle's mask generator, seed draw, prime table and
exact counter are pinned bit-for-bit against the reference's code (tests/golden/); the MSWS
and count-min insert/query restatements are pinned against the reference's own sketch
kernels run on a GPU (tests/test_ref_pin_gpu.py, on inputs where the reference's result does
not depend on the thread schedule) and by hand-worked known-answer cases derived from
device_sketch_v3.h for the order-dependent part (the reference ships no golden vectors).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libqsref.so")
START = 1024
SATURATED = 2


def build(ref=True):
    """Compile liboracle.so (and oracle/_ref when the reference checkout is present)."""
    subprocess.run(["make", "-s", "-C", HERE, "all" if ref else os.path.join(HERE, "liboracle.so")], check=True)


def _load():
    if not os.path.exists(LIB_PATH):
        build(ref=False)
    lib = ctypes.CDLL(LIB_PATH)
    P, U32, U64, SZ = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_size_t
    sig = {
        "or_find_greatest_prime": (U64, [U64]),
        "or_generate_hashmask": (ctypes.c_int, [U32, SZ, SZ, SZ, SZ, P]),
        "or_draw_seeds": (None, [U32, SZ, P]),
        "or_msws_insert": (None, [P, P, U64]),
        "or_msws_insert_mt": (None, [P, P, U64, ctypes.c_int]),
        "or_msws_query": (None, [P, P, U64, P]),
        "or_msws_remove": (None, [P, P, U64]),
        "or_cm_remove": (None, [P, U64, U32, P, P, U64]),
        "or_bucket_insert": (None, [P, U64, U32, U32, P, U32, P, U64]),
        "or_bucket_query": (None, [P, U64, U32, U32, P, U32, P, U64, P]),
        "or_bucket_remove": (None, [P, U64, U32, U32, P, U32, P, U64]),
        "or_cm_insert": (None, [P, U64, U32, P, P, U64]),
        "or_cm_insert_mt": (None, [P, U64, U32, P, P, U64, ctypes.c_int]),
        "or_cm_query": (None, [P, U64, U32, P, P, U64, P]),
        "or_exact_counts": (None, [P, U64, P, U64, P]),
        "or_error_metrics": (None, [P, P, U64, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    }
    for k, (r, a) in sig.items():
        f = getattr(lib, k)
        f.restype, f.argtypes = r, a
    return lib


lib = _load()


class _MswsState(ctypes.Structure):
    _fields_ = [("low", ctypes.c_void_p), ("n_low", ctypes.c_uint64), ("high", ctypes.c_void_p),
                ("n_high", ctypes.c_uint64), ("masks", ctypes.c_void_p), ("n_masks", ctypes.c_uint32),
                ("seed", ctypes.c_uint32), ("next_id", ctypes.c_uint32), ("compat_v3", ctypes.c_int32),
                ("pool_full", ctypes.c_uint32), ("pad", ctypes.c_uint32), ("dropped", ctypes.c_uint64)]


def _u32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32))


def find_greatest_prime(x):
    return int(lib.or_find_greatest_prime(int(x)))


def generate_hashmask(rng_seed, n=1021, m=32, ones=3, padding=4):
    out = np.zeros(n * ((m + 7) // 8), np.uint8)
    if lib.or_generate_hashmask(rng_seed, n, m, ones, padding, out.ctypes.data) != 0:
        raise ValueError("bad hashmask sizes")
    return out


def draw_seeds(rng_seed, count):
    out = np.zeros(count, np.uint32)
    lib.or_draw_seeds(rng_seed, count, out.ctypes.data)
    return out


class Msws:
    """Sequential MSWS (device_sketch_v3.h semantics) with injected seed and masks."""

    def __init__(self, n_low, n_high, seed, mask_table, compat_v3=False):
        self.low = np.zeros(n_low * 8, np.uint32)
        self.high = np.zeros(n_high * 32, np.uint32)
        mt = np.ascontiguousarray(np.asarray(mask_table, np.uint8))
        self.masks = mt.view(np.uint32).copy()
        self.s = _MswsState(self.low.ctypes.data, n_low, self.high.ctypes.data, n_high, self.masks.ctypes.data,
                            self.masks.size, seed, START + 1, 1 if compat_v3 else 0, 0, 0, 0)

    def insert(self, keys, threads=1):
        k = _u32(keys)
        if threads > 1:
            lib.or_msws_insert_mt(ctypes.byref(self.s), k.ctypes.data, k.size, threads)
        else:
            lib.or_msws_insert(ctypes.byref(self.s), k.ctypes.data, k.size)

    def query(self, keys):
        k = _u32(keys)
        out = np.zeros(k.size, np.uint32)
        lib.or_msws_query(ctypes.byref(self.s), k.ctypes.data, k.size, out.ctypes.data)
        return out

    def remove(self, keys):
        k = _u32(keys)
        lib.or_msws_remove(ctypes.byref(self.s), k.ctypes.data, k.size)

    @property
    def next_id(self):
        return self.s.next_id

    @property
    def pool_full(self):
        return bool(self.s.pool_full)

    @property
    def dropped(self):
        return self.s.dropped


class CountMin:
    """Plain count-min (device_sketch_v0.h) with injected per-row seeds."""

    def __init__(self, n, seeds):
        self.n = n
        self.seeds = _u32(seeds)
        self.m = self.seeds.size
        self.table = np.zeros(n * self.m, np.uint32)

    def insert(self, keys, threads=1):
        k = _u32(keys)
        if threads > 1:
            lib.or_cm_insert_mt(self.table.ctypes.data, self.n, self.m, self.seeds.ctypes.data, k.ctypes.data,
                                k.size, threads)
        else:
            lib.or_cm_insert(self.table.ctypes.data, self.n, self.m, self.seeds.ctypes.data, k.ctypes.data, k.size)

    def remove(self, keys):
        k = _u32(keys)
        lib.or_cm_remove(self.table.ctypes.data, self.n, self.m, self.seeds.ctypes.data, k.ctypes.data, k.size)

    def query(self, keys):
        k = _u32(keys)
        out = np.zeros(k.size, np.uint32)
        lib.or_cm_query(self.table.ctypes.data, self.n, self.m, self.seeds.ctypes.data, k.ctypes.data, k.size,
                        out.ctypes.data)
        return out


class BucketSketch:
    """One-level bucket sketch (the reference's warp / sub-warp sketches, device_sketch_v1.h /
    device_sketch_v2.h): n buckets of m u32 counters, H masks of m bits (byte table)."""

    def __init__(self, n, m, seed, mask_table):
        self.n, self.m, self.seed = n, m, seed
        mt = np.ascontiguousarray(np.asarray(mask_table, np.uint8)).reshape(-1, m // 8)
        self.masks = np.zeros(mt.shape[0], np.uint32)
        for k in range(m // 8):
            self.masks |= mt[:, k].astype(np.uint32) << np.uint32(8 * k)
        self.table = np.zeros(n * m, np.uint32)

    def _args(self, k):
        return (self.table.ctypes.data, self.n, self.m, self.seed, self.masks.ctypes.data, self.masks.size,
                k.ctypes.data, k.size)

    def insert(self, keys):
        k = _u32(keys)
        lib.or_bucket_insert(*self._args(k))

    def remove(self, keys):
        k = _u32(keys)
        lib.or_bucket_remove(*self._args(k))

    def query(self, keys):
        k = _u32(keys)
        out = np.zeros(k.size, np.uint32)
        lib.or_bucket_query(*self._args(k), out.ctypes.data)
        return out


def exact_counts(keys, queries):
    k, q = _u32(keys), _u32(queries)
    out = np.zeros(q.size, np.uint32)
    lib.or_exact_counts(k.ctypes.data, k.size, q.ctypes.data, q.size, out.ctypes.data)
    return out


def error_metrics(est, exact):
    e, a = _u32(est), _u32(exact)
    r, q = ctypes.c_double(), ctypes.c_double()
    lib.or_error_metrics(e.ctypes.data, a.ctypes.data, e.size, ctypes.byref(r), ctypes.byref(q))
    return r.value, q.value


def ref_lib():
    """The reference's own library code (oracle/_ref), or None when it was not built."""
    if not os.path.exists(REF_PATH):
        return None
    r = ctypes.CDLL(REF_PATH)
    P, SZ = ctypes.c_void_p, ctypes.c_size_t
    r.ref_generate_hashmask.argtypes = [ctypes.c_uint, SZ, SZ, SZ, SZ, P]
    r.ref_draw_seeds.argtypes = [ctypes.c_uint, SZ, P]
    r.ref_find_greatest_prime.argtypes = [ctypes.c_ulonglong]
    r.ref_find_greatest_prime.restype = ctypes.c_ulonglong
    r.ref_exact_counts.argtypes = [P, SZ, P, SZ, P]
    if hasattr(r, "ref_msws_gpu"):
        r.ref_msws_gpu.argtypes = [ctypes.c_uint, ctypes.c_uint, SZ, SZ, P, SZ, P, SZ, P, P, P, P]
        r.ref_cm_gpu.argtypes = [ctypes.c_uint, SZ, SZ, P, SZ, P, SZ, P, P, P]
    return r


def ref_msws_gpu(seed_rng, mask_rng, n_low, n_high, keys, queries, with_low=False):
    """The reference's own Sketch_GPU_Sub_Warp_Level kernels on the current GPU
    (device_sketch_v3.h:526-634), engines reseeded.  Returns (estimates, seed, mask table, low
    table or None); raises ValueError for inputs the reference kernel is not defined on (a
    warp share that is not a multiple of 4 keys, or a low counter that would pass 128)."""
    r = ref_lib()
    if r is None or not hasattr(r, "ref_msws_gpu"):
        raise RuntimeError("oracle/_ref/libqsref.so with the reference's sketch kernels is not built")
    k, q = _u32(keys), _u32(queries)
    out = np.zeros(q.size, np.uint32)
    low = np.zeros(n_low * 8, np.uint32) if with_low else None
    seed = np.zeros(1, np.uint32)
    masks = np.zeros(1021 * 4, np.uint8)
    rc = r.ref_msws_gpu(seed_rng, mask_rng, n_low, n_high, k.ctypes.data, k.size, q.ctypes.data, q.size,
                        out.ctypes.data, low.ctypes.data if with_low else None, seed.ctypes.data, masks.ctypes.data)
    if rc == -1:
        raise ValueError("input outside the reference kernel's defined range")
    if rc != 0:
        raise RuntimeError(f"reference MSWS run failed: CUDA error {rc}")
    return out, int(seed[0]), masks, low


def ref_cm_gpu(seed_rng, n, m, keys, queries, with_table=False):
    """The reference's own Sketch_GPU_Thread kernels on the current GPU (device_sketch_v0.h:105-191),
    seed engine reseeded.  Returns (estimates, seeds, table or None)."""
    r = ref_lib()
    if r is None or not hasattr(r, "ref_cm_gpu"):
        raise RuntimeError("oracle/_ref/libqsref.so with the reference's sketch kernels is not built")
    k, q = _u32(keys), _u32(queries)
    out = np.zeros(q.size, np.uint32)
    tab = np.zeros(n * m, np.uint32) if with_table else None
    seeds = np.zeros(m, np.uint32)
    rc = r.ref_cm_gpu(seed_rng, n, m, k.ctypes.data, k.size, q.ctypes.data, q.size, out.ctypes.data,
                      tab.ctypes.data if with_table else None, seeds.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"reference count-min run failed: status {rc}")
    return out, seeds, tab
