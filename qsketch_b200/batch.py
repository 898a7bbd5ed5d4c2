"""Batched uneven streams over the C ABI (qs_batch_* in include/qsketch_c.h).

No counterpart in the reference.  One handle owns many independent MSWS sketches (one per
stream, each with its own size and hash multiplier, one mask table for all) in a single
table arena; a call inserts or queries the keys of every stream at once from one flat key
array plus offsets, in one persistent launch.  Each stream's result equals inserting its
keys alone into `Sketch_GPU_Sub_Warp_Level(n_low[s], 8, n_high[s], 32, hash_seed=seed[s],
mask_rng=...)`.
"""
import ctypes

import numpy as np
import torch

from ._lib import QS_FLAG_COMPAT_V3, QS_FLAG_NO_CHUNK_RAMP, QsError, check, lib, qs_batch_info, qs_batch_params
from .sketch import _ptr, _stream


def _offsets_ptr(offsets):
    if not (isinstance(offsets, torch.Tensor) and offsets.is_cuda and offsets.dtype == torch.int64
            and offsets.is_contiguous()):
        raise TypeError("offsets must be a contiguous CUDA int64 tensor of n_streams + 1 entries")
    return offsets.data_ptr()


class BatchedSketches:
    """n_streams MSWS sketches updated together (qs_batch_create)."""

    def __init__(self, n_low, n_high, *, hash_seeds=None, seed_rng=1, mask_rng=1, hash_mask_table_sz=1021,
                 hash_mask_ones=3, compat_v3=False, aggregate=0, route=0, lanes_per_key=0, ctas_per_sm=0,
                 max_batch=0, first_chunk=0, chunk_ramp=True, device=None, class_lanes_per_key=None):
        nl = np.ascontiguousarray(n_low, dtype=np.uint64)
        nh = np.ascontiguousarray(n_high, dtype=np.uint64)
        if nl.shape != nh.shape or nl.ndim != 1:
            raise ValueError("n_low and n_high must be 1-D and of equal length")
        p = qs_batch_params()
        lib.qs_batch_params_default(ctypes.byref(p))
        p.n_streams = nl.size
        p.n_low = nl.ctypes.data
        p.n_high = nh.ctypes.data
        seeds = None
        if hash_seeds is not None:
            seeds = np.ascontiguousarray(hash_seeds, dtype=np.uint32)
            if seeds.size != nl.size:
                raise ValueError("one hash seed per stream")
            p.hash_seeds = seeds.ctypes.data
        p.seed_rng, p.mask_rng = seed_rng, mask_rng
        p.hash_mask_table_sz, p.hash_mask_ones = hash_mask_table_sz, hash_mask_ones
        p.flags = (QS_FLAG_COMPAT_V3 if compat_v3 else 0) | (0 if chunk_ramp else QS_FLAG_NO_CHUNK_RAMP)
        p.first_chunk = first_chunk
        p.aggregate, p.route = aggregate, route
        p.lanes_per_key, p.ctas_per_sm = lanes_per_key, ctas_per_sm
        if max_batch:
            p.max_batch = max_batch
        if device is None:
            device = torch.cuda.current_device() if torch.cuda.is_available() else -1
        p.device = device
        self._cls = None
        if class_lanes_per_key is not None:  # {size class: lanes per key} or a 64-entry sequence
            arr = np.zeros(64, np.uint32)
            items = class_lanes_per_key.items() if isinstance(class_lanes_per_key, dict) else \
                enumerate(class_lanes_per_key)
            for c, v in items:
                arr[int(c)] = int(v)
            self._cls = arr
            p.class_lanes_per_key = arr.ctypes.data
        h = ctypes.c_void_p()
        check(lib.qs_batch_create(ctypes.byref(p), ctypes.byref(h)), "BatchedSketches")
        self._h = h
        self.n_streams = int(nl.size)
        self.n_low, self.n_high = nl.copy(), nh.copy()

    @property
    def handle(self):
        if not self._h:
            raise QsError(1, "batch is closed")
        return self._h

    @staticmethod
    def _total(offsets, total):
        return int(offsets[-1].item()) if total is None else int(total)

    def insert(self, keys, offsets, total=None, stream=None):
        check(lib.qs_batch_insert(self.handle, _ptr(keys, "keys"), _offsets_ptr(offsets),
                                  self._total(offsets, total), _stream(stream)), "insert")
        return 0

    def search(self, keys, offsets, total=None, counts=None, stream=None):
        if counts is None:
            counts = torch.empty(keys.numel(), dtype=torch.uint32, device=keys.device)
        check(lib.qs_batch_query(self.handle, _ptr(keys, "keys"), _offsets_ptr(offsets),
                                 self._total(offsets, total), _ptr(counts, "counts"), _stream(stream)), "search")
        return counts

    query = search

    def insert_graph(self, keys, offsets, max_total=None, stream=None):
        """Replay (recording on first use) the insert of whatever `keys`/`offsets` hold."""
        mt = keys.numel() if max_total is None else int(max_total)
        check(lib.qs_batch_insert_graph(self.handle, _ptr(keys, "keys"), _offsets_ptr(offsets), mt,
                                        _stream(stream)), "insert_graph")
        return 0

    def search_graph(self, keys, offsets, counts, max_total=None, stream=None):
        mt = keys.numel() if max_total is None else int(max_total)
        check(lib.qs_batch_query_graph(self.handle, _ptr(keys, "keys"), _offsets_ptr(offsets), mt,
                                       _ptr(counts, "counts"), _stream(stream)), "search_graph")
        return counts

    def clear(self, stream=None):
        check(lib.qs_batch_clear(self.handle, _stream(stream)), "clear")

    def autotune(self, keys, offsets, total=None, reps=3):
        """qs_batch_autotune: the fastest lanes per key of each size class (floor(log2 n_low)),
        timed on the first window of this batch; returns {size class: lanes per key}.  Leaves
        the sketches cleared."""
        out = np.zeros(64, np.uint32)
        check(lib.qs_batch_autotune(self.handle, _ptr(keys, "keys"), _offsets_ptr(offsets),
                                    self._total(offsets, total), reps, out.ctypes.data), "batch autotune")
        return {c: int(v) for c, v in enumerate(out) if v}

    def sync(self, stream=None):
        check(lib.qs_batch_sync(self.handle, _stream(stream)), "sync")

    def status(self, stream=None):
        return lib.qs_batch_sync(self.handle, _stream(stream))

    def stream_status(self):
        out = np.zeros(self.n_streams, np.uint32)
        check(lib.qs_batch_stream_status(self.handle, out.ctypes.data), "stream_status")
        return out

    def seeds(self):
        out = np.zeros(self.n_streams, np.uint32)
        check(lib.qs_batch_seeds(self.handle, out.ctypes.data), "seeds")
        return out

    def info(self):
        i = qs_batch_info()
        check(lib.qs_batch_get_info(self.handle, ctypes.byref(i)), "info")
        return {f: getattr(i, f) for f, _ in qs_batch_info._fields_}

    def stream_tables(self, s):
        """Stream s's low table (n_low[s]*8 words) and high pool (n_high[s]*32 words), copied out
        of the arena, with the stream's own high ids in word 7 (as a sketch of its own holds
        them)."""
        arena = lib.qs_batch_arena(self.handle)
        nl, nh = ctypes.c_uint64(), ctypes.c_uint64()
        m = ctypes.c_uint32()
        check(lib.qs_get_info(arena, ctypes.byref(nl), ctypes.byref(nh), ctypes.byref(m), None, None), "info")
        low = np.zeros(nl.value * 8, np.uint32)
        high = np.zeros(nh.value * 32, np.uint32)
        check(lib.qs_get_tables(arena, low.ctypes.data, high.ctypes.data), "tables")
        lb, hb = int(self.n_low[:s].sum()), int(self.n_high[:s].sum())
        sl = low[lb * 8:(lb + int(self.n_low[s])) * 8].copy()
        sh = high[hb * 32:(hb + int(self.n_high[s])) * 32].copy()
        w7 = sl[7::8]
        w7[w7 > 1024] -= np.uint32(hb)
        return sl, sh

    def set_profiling(self, enable=True):
        check(lib.qs_set_profiling(lib.qs_batch_arena(self.handle), 1 if enable else 0), "set_profiling")

    def profile(self):
        """Per-launch CUDA-event times of eager calls since the last read (qs_get_profile)."""
        from ._lib import qs_profile
        p = qs_profile()
        check(lib.qs_get_profile(lib.qs_batch_arena(self.handle), ctypes.byref(p)), "profile")
        d = {f: getattr(p, f) for f, _ in qs_profile._fields_}
        d["repair_phase_ms"] = list(p.repair_phase_ms)
        return d

    def close(self):
        if self._h:
            lib.qs_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
