"""Shot partition over ranks and the max-over-ranks timing, run as two gloo
ranks on the CPU (the multi-GPU bench shards shots with no data-path
collective).  CPU only."""
import importlib.util
import os
import socket

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RANKS_PY = os.path.join(ROOT, "model-based-seismic-data-redatuming-with-daws_b200", "ranks.py")


def _ranks():
    spec = importlib.util.spec_from_file_location("daw_ranks", RANKS_PY)
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_para_range_blocks_cover_once():
    R = _ranks()
    for n in (1, 2, 7, 50, 51, 256, 1024):
        for p in (1, 2, 3, 4, 8, 16):
            seen = []
            prev_end = 0
            for r in range(p):
                a, b = R.para_range(1, n, p, r)
                assert a == prev_end + 1  # contiguous blocks in rank order
                seen += list(range(a, b + 1))
                prev_end = b
                assert b - a + 1 in (n // p, n // p + 1)
            assert seen == list(range(1, n + 1))


def test_para_range_matches_reference_examples():
    R = _ranks()
    # 50 shots over 8 ranks: the first 2 ranks take 7, the others 6
    assert [R.para_range(1, 50, 8, r) for r in range(8)] == [
        (1, 7), (8, 14), (15, 20), (21, 26), (27, 32), (33, 38), (39, 44), (45, 50)]
    # more ranks than shots: trailing ranks get an empty range
    a, b = R.para_range(1, 3, 4, 3)
    assert b < a
    with pytest.raises(ValueError):
        R.para_range(1, 10, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    R = _ranks()
    r, w, local = R.rank_env()
    dist = R.init_group(w, timeout_s=60)
    try:
        ids = R.rank_shots(50, 2, r, w)
        R.barrier(dist)
        fake_ms = 100.0 + 25.0 * r  # this rank's device time
        tmax = R.max_over_ranks(dist, fake_ms)
        total = R.sum_over_ranks(dist, len(ids))
        import torch
        gathered = [None] * w
        dist.all_gather_object(gathered, ids)
        R.barrier(dist)
        q.put((r, local, ids, tmax, total, gathered))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_partition_and_timing():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    res.sort()
    (r0, l0, ids0, t0, n0, g0), (r1, l1, ids1, t1, n1, g1) = res
    assert (r0, r1) == (0, 1) and (l0, l1) == (0, 1)
    # every rank sees the slowest rank's time, and the job counts all shots
    assert t0 == t1 == 125.0
    assert n0 == n1 == 4
    # disjoint shot sets drawn from each rank's para_range block
    assert set(ids0).isdisjoint(ids1)
    assert all(0 <= i < 25 for i in ids0) and all(25 <= i < 50 for i in ids1)
    assert g0 == g1 == [ids0, ids1]
