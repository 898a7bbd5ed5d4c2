"""Multi-process (world size 2, gloo on CPU) tests of the multi-GPU host logic: the insert path
runs one independent sketch per rank with its own seeded stream ("replicas"), so the only
collectives are the barrier and the max-over-ranks of the times.  Each rank here inserts its
own stream into the CPU oracle; the test checks that ranks hold different data, agree on
the gathered values, and that the job time and aggregate rate follow the slowest rank."""
import multiprocessing as mp
import os
import socket

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    try:
        import oracle
        from qsketch_b200.replicas import Ranks, aggregate_rate
        r = Ranks(backend="gloo", timeout_s=60)
        seed = r.stream_seed(1000)
        rng = np.random.default_rng(seed)
        keys = (rng.zipf(1.3, 1 << 15) % 4096).astype(np.uint32) * np.uint32(2654435761)
        s = oracle.Msws(1021, 512, 2654435769, oracle.generate_hashmask(1))
        s.insert(keys)
        est = s.query(np.unique(keys))
        checksum = float(est.astype(np.float64).sum() + keys[:64].astype(np.float64).sum())
        gathered = r.gather(checksum)
        local_ms = 1.0 + rank  # rank 1 is the slow one
        job_ms = r.max(local_ms)
        total = r.sum(float(keys.size))
        r.barrier()
        q.put((rank, seed, gathered, job_ms, total, aggregate_rate(keys.size, world, job_ms)))
        r.close()
    except Exception as e:  # report instead of hanging the parent
        q.put((rank, "error", repr(e)))


def test_two_ranks_replicas_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort(key=lambda x: x[0])
    for r in res:
        assert r[1] != "error", r
    (r0, s0, g0, m0, t0, a0), (r1, s1, g1, m1, t1, a1) = res
    assert s0 != s1, "ranks must draw different streams"
    assert g0 == g1 and len(g0) == 2 and g0[0] != g0[1], "each rank's sketch holds its own data"
    assert m0 == m1 == 2.0, "the job time is the slowest rank's"
    assert t0 == t1 == 2.0 * (1 << 15)
    assert a0 == a1 == 2 * (1 << 15) / (2.0 * 1e6)
