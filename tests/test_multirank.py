"""The N > 1 path of bench.py on the CPU: two gloo ranks (one process each, as torchrun
launches them) shard the sweep's frequencies with no data-path collective, take the
maximum of their device times with one all-reduce, and the reference arm runs on rank 0
alone. Nothing here touches a GPU."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    sys.path.insert(0, ROOT)
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    got_ws, got_rank = bench.dist_env()
    dist = bench.init_dist(got_ws)
    freqs = np.arange(512) * 5e6 + 5e6
    shards = [bench.step_freqs(freqs, s, 128, got_rank, got_ws) for s in range(4)]
    t_max = bench.max_over_ranks(dist, 1.0 + got_rank)        # rank 1 is the slow one
    bench.barrier(dist)
    import torch.distributed as td
    gathered = [None] * got_ws
    td.all_gather_object(gathered, [s.tolist() for s in shards])

    class A:
        steps, warmup, batch = 1, 0, 128
    ref = bench.run_reference(A, got_ws, got_rank) if got_rank != 0 else "rank0-skipped"
    dist.destroy_process_group()
    out.put((got_rank, t_max, gathered, ref))


@pytest.mark.timeout(300)
def test_two_gloo_ranks_shard_frequencies_and_take_max_time():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = [q.get(timeout=240) for _ in ps]
    for p in ps:
        p.join(60)
        assert p.exitcode == 0
    res.sort()
    for rank, t_max, gathered, ref in res:
        assert t_max == 2.0                                   # max over ranks, not the local time
        r0, r1 = gathered
        for s in range(4):                                    # disjoint shards per step
            assert not set(r0[s]) & set(r1[s])
        seen = set(f for g in gathered for s in g for f in s)
        assert len(seen) == 512                               # 4 steps x 2 ranks x 128 = the sweep
    assert res[1][3] is None                                  # reference arm: rank 1 does no work
