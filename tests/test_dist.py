"""Frame sharding across ranks (one process per GPU), exercised with two
gloo ranks on the CPU: the shards cover every candidate once, in frame
order, the throughput bookkeeping takes the slowest rank's time and the
summed work, and gathered rows equal the single-process rows."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import localizer_b200 as L
from localizer_b200 import dist as D


def _cands(n_frames=37, seed=3):
    rng = np.random.default_rng(seed)
    counts = rng.integers(0, 9, size=n_frames)
    c = np.zeros(int(counts.sum()), dtype=L.CANDIDATE_DTYPE)
    c["frame"] = np.repeat(np.arange(n_frames), counts)
    c["x"] = rng.uniform(5, 100, len(c))
    c["y"] = rng.uniform(5, 100, len(c))
    return c, n_frames


def _fake_fit(c):
    # stands in for the GPU fit: a deterministic per-candidate row
    rows = np.stack([c["frame"].astype(float), c["x"] * 2.0, c["y"] + 1.0], axis=1)
    flags = (c["x"] > 50).astype(np.uint8)
    return rows, flags


def test_frame_shard_partitions():
    for n in (0, 1, 7, 100):
        for w in (1, 2, 3, 8):
            spans = [D.frame_shard(n, r, w) for r in range(w)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        D.frame_shard(10, 2, 2)


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        c, nf = _cands()
        idx = D.candidate_shard(c, rank, world, nf)
        rows, flags = _fake_fit(c[idx])
        total, ms, rate = D.job_throughput(len(idx), 10.0 * (rank + 1))
        got = D.gather_rows(rows, flags)
        q.put((rank, idx.tolist(), total, ms, rate, None if got is None else (got[0].tolist(), got[1].tolist())))
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_gloo_ranks_cover_and_gather():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    world = 2
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=120) for _ in range(world)])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    c, nf = _cands()
    idx = sorted(res[0][1] + res[1][1])
    assert idx == list(range(len(c)))                       # each candidate exactly once
    assert max(res[0][1]) < min(res[1][1])                  # rank 0 holds the earlier frames
    assert res[0][2] == res[1][2] == float(len(c))          # summed work
    assert res[0][3] == res[1][3] == 20.0                   # slowest rank's time
    rows, flags = _fake_fit(c)
    g_rows, g_flags = res[0][5]
    np.testing.assert_array_equal(np.array(g_rows), rows)   # gathered in frame order
    np.testing.assert_array_equal(np.array(g_flags), flags)
    assert res[1][5] is None
