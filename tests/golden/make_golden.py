"""Regenerate the golden fixtures in tests/golden/ from the reference's own code.

Runs the reference's library sources (lib/hashmask.cu, lib/qsketch.cu, lib/default.cu and
the header-only Unordered_Map) through oracle/_ref/libqsref.so, built by `make -C oracle`
from the reference checkout.  The fixtures are committed, so the tests need neither the
checkout nor this script:

    make -C oracle && python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
import oracle  # noqa: E402

MASK_CASES = [  # (rng_seed, n, m_bits, ones, padding); the first row is device_sketch_v3.h:559
    (1, 1021, 32, 3, 4),
    (12345, 1021, 32, 3, 4),
    (3735928559, 1021, 32, 3, 4),
    (2024, 1021, 32, 4, 4),
    (99, 509, 32, 1, 4),
    (7, 257, 16, 3, 4),
]
SEED_CASES = [(1, 8), (42, 8), (3735928559, 8), (123456789, 3)]
PRIME_INPUTS = sorted(set([0, 1, 2, 3, 4, 100, 1021, 1022, 262138, 262139, 262140, 2097143, 8388592, 8388593,
                           (1 << 18), (1 << 21), (1 << 23), (1 << 24), (1 << 28), 402653171, 402653172, 1 << 40]
                          + [(1 << k) + d for k in range(4, 30) for d in (-1, 0, 1)]))


def main():
    r = oracle.ref_lib()
    if r is None:
        sys.exit("oracle/_ref/libqsref.so is missing: run `make -C oracle` in a checkout with the reference")
    fixtures = {"masks": [], "seeds": [], "primes": {}, "exact": {}}
    for seed, n, m, ones, pad in MASK_CASES:
        out = np.zeros(n * ((m + 7) // 8), np.uint8)
        r.ref_generate_hashmask(seed, n, m, ones, pad, out.ctypes.data)
        name = f"hashmask_s{seed}_n{n}_m{m}_o{ones}_p{pad}.bin"
        out.tofile(os.path.join(HERE, name))
        fixtures["masks"].append({"rng_seed": seed, "n": n, "m_bits": m, "ones": ones, "padding": pad, "file": name})
    for seed, count in SEED_CASES:
        out = np.zeros(count, np.uint32)
        r.ref_draw_seeds(seed, count, out.ctypes.data)
        fixtures["seeds"].append({"rng_seed": seed, "values": [int(x) for x in out]})
    for x in PRIME_INPUTS:
        fixtures["primes"][str(x)] = int(r.ref_find_greatest_prime(x))
    # Unordered_Map exact counts on a small skewed stream (host_sketch.h:20-39)
    rng = np.random.default_rng(5)
    keys = (rng.zipf(1.3, 20000) % 5000).astype(np.uint32) * np.uint32(2654435761)
    queries = np.unique(keys)[:3000].astype(np.uint32)
    out = np.zeros(queries.size, np.uint32)
    r.ref_exact_counts(keys.ctypes.data, keys.size, queries.ctypes.data, queries.size, out.ctypes.data)
    keys.tofile(os.path.join(HERE, "exact_keys.bin"))
    queries.tofile(os.path.join(HERE, "exact_queries.bin"))
    out.tofile(os.path.join(HERE, "exact_counts.bin"))
    fixtures["exact"] = {"keys": "exact_keys.bin", "queries": "exact_queries.bin", "counts": "exact_counts.bin"}
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(fixtures, f, indent=1)
    print("wrote", len(fixtures["masks"]), "mask tables,", len(fixtures["seeds"]), "seed draws,",
          len(fixtures["primes"]), "primes, exact counts of", queries.size, "keys")


if __name__ == "__main__":
    main()
