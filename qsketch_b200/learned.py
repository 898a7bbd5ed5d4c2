"""The learned heavy-hitter split over the C ABI (qs_learned_* in include/qsketch_c.h).

No counterpart in the reference.  An MLP over the key bits, trained on the sketch's own
warm-up estimates, routes predicted-heavy keys to an exact table carved from the same byte
budget; all other keys go to the MSWS sketch.
"""
import ctypes

import numpy as np
import torch

from ._lib import QS_MLP_PARAMS, QsError, check, lib, qs_learned_info, qs_learned_params
from .sketch import _ptr, _stream


def default_params(**kw):
    p = qs_learned_params()
    lib.qs_learned_params_default(ctypes.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise TypeError(f"unknown learned parameter {k}")
        setattr(p, k, v)
    return p


class LearnedSketch:
    """MSWS + exact heavy table + MLP router sharing one byte budget."""

    def __init__(self, **params):
        p = default_params(**params)
        h = ctypes.c_void_p()
        check(lib.qs_learned_create(ctypes.byref(p), ctypes.byref(h)), "LearnedSketch")
        self._h = h

    @property
    def handle(self):
        if not self._h:
            raise QsError(1, "learned sketch is closed")
        return self._h

    def insert(self, keys, stream=None):
        check(lib.qs_learned_insert(self.handle, _ptr(keys, "keys"), keys.numel(), _stream(stream)), "insert")
        return 0

    def search(self, keys, counts=None, stream=None):
        if counts is None:
            counts = torch.empty(keys.numel(), dtype=torch.uint32, device=keys.device)
        check(lib.qs_learned_query(self.handle, _ptr(keys, "keys"), keys.numel(), _ptr(counts, "counts"),
                                   _stream(stream)), "search")
        return counts

    query = search

    def admit_keys(self, keys):
        """Diagnostic admission (qs_learned_admit_keys): these host keys enter the exact table in
        order, up to its max fill, and the warm-up ends without training."""
        k = np.ascontiguousarray(np.asarray(keys, np.uint32))
        check(lib.qs_learned_admit_keys(self.handle, k.ctypes.data, k.size), "admit_keys")

    def info(self):
        i = qs_learned_info()
        check(lib.qs_learned_get_info(self.handle, ctypes.byref(i)), "info")
        d = {f: getattr(i, f) for f, _ in qs_learned_info._fields_}
        d["train_phase_ms"] = list(d["train_phase_ms"])
        return d

    def table(self):
        """The exact table: (keys, counts) of its occupied slots, and the sketch's multiplier."""
        n = self.info()["table_slots"]
        k = np.zeros(n, np.uint32)
        c = np.zeros(n, np.uint32)
        seed = ctypes.c_uint32()
        check(lib.qs_learned_get_table(self.handle, k.ctypes.data, c.ctypes.data, ctypes.byref(seed)), "table")
        used = k != 0xffffffff
        return k[used], c[used], seed.value

    # ---- the classifier alone -----------------------------------------------------------
    def mlp_params(self):
        out = np.zeros(QS_MLP_PARAMS, np.float32)
        check(lib.qs_mlp_get_params(self.handle, out.ctypes.data), "mlp_params")
        return out

    def set_mlp_params(self, params):
        a = np.ascontiguousarray(params, np.float32)
        assert a.size == QS_MLP_PARAMS
        check(lib.qs_mlp_set_params(self.handle, a.ctypes.data), "set_mlp_params")

    def mlp_forward(self, keys):
        out = torch.empty(keys.numel(), dtype=torch.float32, device=keys.device)
        check(lib.qs_mlp_forward(self.handle, _ptr(keys, "keys"), keys.numel(), out.data_ptr(), _stream(None)),
              "mlp_forward")
        return out

    def mlp_grads(self, keys, labels, pos_weight):
        g = np.zeros(QS_MLP_PARAMS, np.float32)
        loss = ctypes.c_double()
        lab = labels.to(torch.uint8).contiguous()
        check(lib.qs_mlp_grads(self.handle, _ptr(keys, "keys"), lab.data_ptr(), keys.numel(), float(pos_weight),
                               g.ctypes.data, ctypes.byref(loss)), "mlp_grads")
        return g, loss.value

    def mlp_train(self, keys, labels, epochs, batch, lr, pos_weight):
        loss = ctypes.c_double()
        lab = labels.to(torch.uint8).contiguous()
        check(lib.qs_mlp_train(self.handle, _ptr(keys, "keys"), lab.data_ptr(), keys.numel(), epochs, batch,
                               float(lr), float(pos_weight), ctypes.byref(loss)), "mlp_train")
        return loss.value

    def close(self):
        if self._h:
            lib.qs_learned_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def plain_equal_bytes(budget_bytes, **kw):
    """The plain MSWS sketch with the whole budget and the same 4:1 low:high split."""
    from .sketch import Sketch_GPU_Sub_Warp_Level, find_greatest_prime
    n_low = find_greatest_prime(budget_bytes * 4 // 5 // 32)
    n_high = (budget_bytes - n_low * 32) // 128
    return Sketch_GPU_Sub_Warp_Level(n_low, 8, n_high, 32, **kw)
