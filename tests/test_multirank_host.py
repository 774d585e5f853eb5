"""The multi-rank plumbing of bench.py on CPU (gloo, world size 2, 127.0.0.1):
replicas get distinct workloads (weak scaling, no collective on the data
path), timing reduces as the max over ranks and work as the sum, and the
reference arm runs on rank 0 only."""
import multiprocessing as mp
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    try:
        import bench
        w, r, local, pg = bench.dist_setup()
        assert (w, r, local) == (ws, rank, rank)
        t = bench.max_over_ranks(1.0 + rank, pg)        # per-rank step time
        n = bench.sum_over_ranks(10.0 * (rank + 1), pg)  # per-rank work
        bench.barrier(pg)
        fws = bench.make_workload(rank, n=3)
        sig = [round(float(f.abc[0]), 6) for f in fws]

        class A:
            steps, warmup = 1, 1
        ref = bench.run_reference(A, w, r) if rank != 0 else "skipped"
        pg.barrier()
        pg.destroy_process_group()
        q.put((rank, t, n, sig, ref is None if rank != 0 else None))
    except Exception as e:  # reported to the parent
        q.put((rank, "error", repr(e), None, None))


def test_two_ranks_reduce_and_shard():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in procs:
        rank, *rest = q.get(timeout=180)
        out[rank] = rest
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in (0, 1):
        assert out[r][0] != "error", out[r]
        t, n, sig, ref_none = out[r]
        assert t == 2.0          # max over ranks
        assert n == 30.0         # sum over ranks
    # each rank computes its own batch (weak scaling replicas)
    assert out[0][2] != out[1][2]
    # the reference arm does no work on ranks other than 0
    assert out[1][3] is True
