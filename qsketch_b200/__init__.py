"""B200-native (sm_100a) QSketch insert/query path behind a C ABI (include/qsketch_c.h).

The sketch kernels live in libqsketch.so; this package is the Python mirror of the
reference's host interface (qsketch::Sketch, Sketch_GPU_Sub_Warp_Level, Sketch_GPU_Thread).
"""
from ._lib import LIB_PATH, QsError, check, lib  # noqa: F401  (raises ImportError if unbuilt)
from .sketch import (Sketch, Sketch_GPU_Sub_Warp, Sketch_GPU_Sub_Warp_Level, Sketch_GPU_Thread,  # noqa: F401
                     Sketch_GPU_Warp, draw_seeds,
                     find_greatest_prime, from_snapshot, generate_hashmask, load, number_of_buckets)

__all__ = ["Sketch", "Sketch_GPU_Sub_Warp_Level", "Sketch_GPU_Thread", "Sketch_GPU_Warp", "Sketch_GPU_Sub_Warp", "find_greatest_prime",
           "number_of_buckets", "generate_hashmask", "draw_seeds", "load", "from_snapshot", "QsError", "LIB_PATH"]
