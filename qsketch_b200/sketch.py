"""Host-side mirror of the reference's sketch interface over the C ABI.

Reference interface (bu-hpc/QSketch):
  qsketch::Sketch<Key_T, Count_T>                      include/sketch/sketch.h:5-28
      int insert(Key_T *keys, size_t keys_sz)
      int search(Key_T *keys, size_t keys_sz, Count_T *counts)
      void clear()
  Sketch_GPU_Sub_Warp_Level(n_low, m_low, n_high, m_high, seed_sz, n_hash_mask_table)
                                                       device_sketch_v3.h:544-563
  Sketch_GPU_Thread(n, m, seed_sz)                     device_sketch_v0.h:121-131
  Sketch_GPU::number_of_buckets(keys, m, factor)       device_sketch.h:371-376
  find_greatest_prime(upper_bound)                     lib/qsketch.cu:50-115
  generate_hashmask(...)                               lib/hashmask.cu:32-83

Keys and counts are CUDA tensors (uint32 or int32, contiguous) or raw device pointers
(ints); insert/search return 0 like the reference and raise QsError on failure instead
of ignoring it (include/qsketch.h:104-105).  The reference draws its hash seed and mask
table from /dev/urandom (include/tool/tool.h:192-204); here they come from `seed_rng`
and `mask_rng` (or explicit `hash_seed` / `mask_table`), so runs are reproducible.
"""
import ctypes
import os

import numpy as np

from ._lib import (QS_FLAG_COMPAT_V3, QS_FLAG_NO_CHUNK_RAMP, QS_KIND_BUCKET, QS_KIND_MSWS, QS_KIND_PLAIN_CM, QsError,
                   check, lib,
                   qs_params, qs_profile, qs_stats)

try:  # torch only supplies device memory and the current stream
    import torch
except ImportError:  # pragma: no cover
    torch = None


def _ptr(x, what):
    if isinstance(x, int):
        return x
    if torch is not None and isinstance(x, torch.Tensor):
        if not x.is_cuda:
            raise ValueError(f"{what} must be a CUDA tensor (use insert_host/search_host for host data)")
        if x.dtype not in (torch.uint32, torch.int32):
            raise TypeError(f"{what} must be uint32 or int32, got {x.dtype}")
        if not x.is_contiguous():
            raise ValueError(f"{what} must be contiguous")
        return x.data_ptr()
    raise TypeError(f"{what}: expected a CUDA tensor or a device pointer")


def _numel(x):
    if torch is not None and isinstance(x, torch.Tensor):
        return x.numel()
    return None


def _stream(stream):
    if stream is not None:
        return stream if isinstance(stream, int) else stream.cuda_stream
    if torch is not None and torch.cuda.is_available():
        return torch.cuda.current_stream().cuda_stream
    return 0


def find_greatest_prime(upper_bound):
    """lib/qsketch.cu:50-115."""
    return int(lib.qs_find_greatest_prime(int(upper_bound)))


def number_of_buckets(insert_keys_sz, m, factor=1.0, hash_mask_ones=3):
    """Sketch_GPU::number_of_buckets, device_sketch.h:371-376."""
    return int(lib.qs_number_of_buckets(int(insert_keys_sz), int(m), float(factor), int(hash_mask_ones)))


def generate_hashmask(n=1021, m=32, hash_mask_ones=3, padding=4, rng_seed=1):
    """lib/hashmask.cu:32-83 on a std::minstd_rand0 seeded with rng_seed; uint8[n*ceil(m/8)]."""
    out = np.zeros(n * ((m + 7) // 8), np.uint8)
    check(lib.qs_generate_hashmask(rng_seed, n, m, hash_mask_ones, padding, out.ctypes.data), "generate_hashmask")
    return out


def draw_seeds(count, rng_seed=1):
    """The reference's seed draw (uniform in [1, 2^32-1], include/tool/tool.h:206-220)."""
    out = np.zeros(count, np.uint32)
    check(lib.qs_draw_seeds(rng_seed, count, out.ctypes.data), "draw_seeds")
    return out


class Sketch:
    """qsketch::Sketch<uint, uint> over a qs_sketch handle."""

    _handle = None

    def _create(self, p):
        h = ctypes.c_void_p()
        check(lib.qs_create(ctypes.byref(p), ctypes.byref(h)), type(self).__name__)
        self._handle = h

    @property
    def handle(self):
        if not self._handle:
            raise QsError(1, "sketch is closed")
        return self._handle

    def insert(self, keys, keys_sz=None, stream=None):
        n = _numel(keys) if keys_sz is None else int(keys_sz)
        if n is None:
            raise ValueError("keys_sz is required with a raw pointer")
        check(lib.qs_insert(self.handle, _ptr(keys, "keys"), n, _stream(stream)), "insert")
        return 0

    def remove(self, keys, keys_sz=None, stream=None):
        """Take one occurrence of each key out (qs_remove: counters floored at 0)."""
        n = _numel(keys) if keys_sz is None else int(keys_sz)
        if n is None:
            raise ValueError("keys_sz is required with a raw pointer")
        check(lib.qs_remove(self.handle, _ptr(keys, "keys"), n, _stream(stream)), "remove")
        return 0

    def search(self, keys, keys_sz=None, counts=None, stream=None):
        n = _numel(keys) if keys_sz is None else int(keys_sz)
        if n is None:
            raise ValueError("keys_sz is required with a raw pointer")
        if counts is None:
            counts = torch.empty(n, dtype=torch.uint32, device=keys.device)
        check(lib.qs_query(self.handle, _ptr(keys, "keys"), n, _ptr(counts, "counts"), _stream(stream)), "search")
        return counts

    query = search

    def insert_host(self, keys):
        """Insert a host array (numpy uint32 or pinned CPU tensor); copies are pipelined."""
        a, n = _host(keys)
        check(lib.qs_insert_host(self.handle, a, n), "insert_host")
        return 0

    def search_host(self, keys, counts=None):
        a, n = _host(keys)
        if counts is None:
            counts = np.empty(n, np.uint32)
        c, _ = _host(counts)
        check(lib.qs_query_host(self.handle, a, n, c), "search_host")
        return counts

    def clear(self, stream=None):
        check(lib.qs_clear(self.handle, _stream(stream)), "clear")

    def sync(self, stream=None):
        """Synchronise and raise on a latched device status (pool full, timeout)."""
        check(lib.qs_sync(self.handle, _stream(stream)), "sync")

    def status(self, stream=None):
        return lib.qs_sync(self.handle, _stream(stream))

    def stats(self):
        s = qs_stats()
        check(lib.qs_get_stats(self.handle, ctypes.byref(s)), "stats")
        return {f: getattr(s, f) for f, _ in qs_stats._fields_}

    def set_profiling(self, enable=True):
        check(lib.qs_set_profiling(self.handle, 1 if enable else 0), "set_profiling")

    def profile(self):
        p = qs_profile()
        check(lib.qs_get_profile(self.handle, ctypes.byref(p)), "profile")
        d = {f: getattr(p, f) for f, _ in qs_profile._fields_}
        d["repair_phase_ms"] = list(d["repair_phase_ms"])
        return d

    def reset_status(self):
        check(lib.qs_reset_status(self.handle), "reset_status")

    def info(self):
        nl, nh, m = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint32()
        check(lib.qs_get_info(self.handle, ctypes.byref(nl), ctypes.byref(nh), ctypes.byref(m), None, None), "info")
        seeds = np.zeros(max(1, m.value if isinstance(self, Sketch_GPU_Thread) else 1), np.uint32)
        masks = np.zeros(self._n_masks * 4, np.uint8) if self._n_masks else None
        check(lib.qs_get_info(self.handle, None, None, None, seeds.ctypes.data,
                              masks.ctypes.data if masks is not None else None), "info")
        return {"n_low": nl.value, "n_high": nh.value, "m_low": m.value, "seeds": seeds, "mask_table": masks}

    def tables(self):
        inf = self.info()
        low = np.zeros(inf["n_low"] * inf["m_low"], np.uint32)
        high = np.zeros(inf["n_high"] * 32, np.uint32) if inf["n_high"] else None
        check(lib.qs_get_tables(self.handle, low.ctypes.data, high.ctypes.data if high is not None else None),
              "tables")
        return low, high

    def snapshot(self):
        """The sketch's whole state as bytes (qs_snapshot_save)."""
        n = ctypes.c_uint64()
        check(lib.qs_snapshot_bytes(self.handle, ctypes.byref(n)), "snapshot")
        buf = ctypes.create_string_buffer(n.value)
        check(lib.qs_snapshot_save(self.handle, buf, n.value), "snapshot")
        return buf.raw

    def save(self, path):
        """write_file (include/qsketch.h:70-71): the snapshot as a file (qs_save)."""
        check(lib.qs_save(self.handle, os.fsencode(str(path))), "save")

    def close(self):
        if self._handle:
            lib.qs_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def _adopt(h):
    """A Python object over a qs_sketch handle made by qs_load / qs_snapshot_load."""
    p = qs_params()
    check(lib.qs_get_params(h, ctypes.byref(p)), "params")
    cls = {QS_KIND_PLAIN_CM: Sketch_GPU_Thread, QS_KIND_BUCKET: Sketch_GPU_Warp}.get(p.kind, Sketch_GPU_Sub_Warp_Level)
    obj = object.__new__(cls)
    obj._handle = h
    obj._keep = None
    obj._n_masks = p.hash_mask_table_sz if p.kind == QS_KIND_MSWS else 0
    return obj


def load(path, device=None):
    """read_file (include/qsketch.h:70-71): a sketch from a snapshot file (qs_load)."""
    h = ctypes.c_void_p()
    check(lib.qs_load(os.fsencode(str(path)), -1 if device is None else int(device), ctypes.byref(h)), "load")
    return _adopt(h)


def from_snapshot(data, device=None):
    """A sketch from snapshot bytes (qs_snapshot_load)."""
    h = ctypes.c_void_p()
    check(lib.qs_snapshot_load(data, len(data), -1 if device is None else int(device), ctypes.byref(h)), "load")
    return _adopt(h)


def _host(x):
    if isinstance(x, np.ndarray):
        if x.dtype not in (np.uint32, np.int32) or not x.flags["C_CONTIGUOUS"]:
            raise TypeError("host arrays must be contiguous uint32/int32")
        return x.ctypes.data, x.size
    if torch is not None and isinstance(x, torch.Tensor) and not x.is_cuda:
        return x.data_ptr(), x.numel()
    raise TypeError("expected a numpy array or a CPU tensor")


class Sketch_GPU_Sub_Warp_Level(Sketch):
    """MSWS / "Level" QSketch (device_sketch_v3.h:526-634)."""

    def __init__(self, n_low=0, m_low=8, n_high=1024, m_high=32, seed_sz=1, n_hash_mask_table=1021, *,
                 low_bytes=0, hash_mask_ones=3, hash_seed=0, seed_rng=1, mask_rng=1, mask_table=None,
                 compat_v3=False, max_batch=0, device=None, aggregate=0, lanes_per_key=0, route=0,
                 ctas_per_sm=0, chunk_ramp=True, keys_per_tile=0, first_chunk=0):
        p = qs_params()
        lib.qs_params_default(ctypes.byref(p))
        p.kind = QS_KIND_MSWS
        p.flags = (QS_FLAG_COMPAT_V3 if compat_v3 else 0) | (0 if chunk_ramp else QS_FLAG_NO_CHUNK_RAMP)
        p.n_low, p.low_bytes, p.m_low, p.m_high, p.n_high = n_low, low_bytes, m_low, m_high, n_high
        p.seed_sz, p.hash_mask_table_sz, p.hash_mask_ones = seed_sz, n_hash_mask_table, hash_mask_ones
        p.hash_seed, p.seed_rng, p.mask_rng = hash_seed, seed_rng, mask_rng
        p.max_batch, p.aggregate, p.lanes_per_key, p.route = max_batch, aggregate, lanes_per_key, route
        p.ctas_per_sm, p.keys_per_tile, p.first_chunk = ctas_per_sm, keys_per_tile, first_chunk
        p.device = -1 if device is None else int(device)
        self._keep = None
        if mask_table is not None:
            mt = np.ascontiguousarray(np.asarray(mask_table).view(np.uint8).ravel())
            if mt.size != n_hash_mask_table * 4:
                raise ValueError("mask_table must hold n_hash_mask_table * 4 bytes")
            self._keep = mt
            p.mask_table = mt.ctypes.data
        self._n_masks = n_hash_mask_table
        self._create(p)


class Sketch_GPU_Warp(Sketch):
    """One-level warp sketch (device_sketch_v1.h:237-334): n buckets of m (= 32) u32 counters,
    each key's mask of m bits selecting hash_mask_ones of them.  Kept for the ablation against
    the two-level MSWS."""

    def __init__(self, n=0, m=32, seed_sz=1, n_hash_mask_table=1021, *, low_bytes=0, hash_mask_ones=3, hash_seed=0,
                 seed_rng=1, mask_rng=1, mask_table=None, device=None, aggregate=0):
        p = qs_params()
        lib.qs_params_default(ctypes.byref(p))
        p.kind = QS_KIND_BUCKET
        p.n_low, p.low_bytes, p.m_low, p.seed_sz = n, low_bytes, m, seed_sz
        p.hash_mask_table_sz, p.hash_mask_ones = n_hash_mask_table, hash_mask_ones
        p.hash_seed, p.seed_rng, p.mask_rng, p.aggregate = hash_seed, seed_rng, mask_rng, aggregate
        p.device = -1 if device is None else int(device)
        self._keep = None
        if mask_table is not None:
            mt = np.ascontiguousarray(np.asarray(mask_table).view(np.uint8).ravel())
            if mt.size != n_hash_mask_table * m // 8:
                raise ValueError("mask_table must hold n_hash_mask_table * m / 8 bytes")
            self._keep = mt
            p.mask_table = mt.ctypes.data
        self._n_masks = 0
        self._create(p)

    def info(self):
        d = super().info()
        nl, nh, m = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint32()
        check(lib.qs_get_info(self.handle, ctypes.byref(nl), ctypes.byref(nh), ctypes.byref(m), None, None), "info")
        pp = qs_params()
        check(lib.qs_get_params(self.handle, ctypes.byref(pp)), "params")
        masks = np.zeros(pp.hash_mask_table_sz * m.value // 8, np.uint8)
        check(lib.qs_get_info(self.handle, None, None, None, None, masks.ctypes.data), "info")
        d["mask_table"] = masks
        return d


class Sketch_GPU_Sub_Warp(Sketch_GPU_Warp):
    """One-level sub-warp sketch (device_sketch_v2.h:289-387): buckets of m = 8 or 16 counters."""

    def __init__(self, n=0, m=8, seed_sz=1, n_hash_mask_table=1021, **kw):
        super().__init__(n, m, seed_sz, n_hash_mask_table, **kw)


class Sketch_GPU_Thread(Sketch):
    """Plain count-min, thread per key (device_sketch_v0.h:105-191)."""

    def __init__(self, n=0, m=3, seed_sz=1, *, low_bytes=0, seeds=None, seed_rng=1, device=None, aggregate=0):
        p = qs_params()
        lib.qs_params_default(ctypes.byref(p))
        p.kind = QS_KIND_PLAIN_CM
        p.n_low, p.low_bytes, p.m_low, p.seed_sz, p.seed_rng = n, low_bytes, m, seed_sz, seed_rng
        p.aggregate = aggregate
        p.device = -1 if device is None else int(device)
        self._keep = None
        if seeds is not None:
            s = np.ascontiguousarray(np.asarray(seeds, np.uint32))
            if s.size != m:
                raise ValueError("seeds must hold m values")
            self._keep = s
            p.seeds = s.ctypes.data
        self._n_masks = 0
        self._create(p)

    @staticmethod
    def number_of_buckets(insert_keys_sz, m, factor):
        """device_sketch_v0.h:133-138: find_greatest_prime(keys / factor)."""
        return find_greatest_prime(int(insert_keys_sz / factor))
