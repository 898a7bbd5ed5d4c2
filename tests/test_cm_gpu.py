"""GPU parity of the plain count-min baseline (device_sketch_v0.h) against the oracle."""
import numpy as np
import pytest
import torch

import oracle
import qsketch_b200 as qs
from qsketch_b200 import data

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("rows,agg", [(3, 1), (3, 2), (1, 2), (4, 2)])
def test_cm_matches_oracle(gpu, rows, agg):
    n = 1048573
    sk = qs.Sketch_GPU_Thread(n, rows, seed_rng=17, aggregate=agg)
    seeds = sk.info()["seeds"]
    assert np.array_equal(seeds, oracle.draw_seeds(17, rows))
    keys = data.zipf_keys(1 << 22, 1 << 20, 1.1, seed=8, perm_seed=1)
    sk.insert(keys)
    q = data.rank_keys(1, 0, 1 << 20)
    got = sk.search(q).cpu().numpy()
    cm = oracle.CountMin(n, seeds)
    cm.insert(keys.cpu().numpy())
    assert np.array_equal(got, cm.query(q.cpu().numpy()))
    low, _ = sk.tables()
    assert np.array_equal(low, cm.table)


def test_cm_uniform_and_edges(gpu):
    sk = qs.Sketch_GPU_Thread(65521, 3, seeds=[3, 5, 2654435761])
    cm = oracle.CountMin(65521, [3, 5, 2654435761])
    keys = data.uniform_keys((1 << 20) + 3, seed=2)
    sk.insert(keys[1:])
    sk.insert(keys[:0])
    cm.insert(keys[1:].cpu().numpy())
    assert np.array_equal(sk.search(keys[1:]).cpu().numpy(), cm.query(keys[1:].cpu().numpy()))
