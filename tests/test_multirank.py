"""bench.py's multi-process plumbing on CPU: two gloo ranks (world size 2, one
process each, rendezvous on 127.0.0.1) go through bench.dist_init and the
reductions the replica bench uses -- the slowest rank's time (MAX) and the
whole job's terms (SUM) -- so value = all ranks' terms / the slowest rank's time."""
import multiprocessing as mp
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench
    try:
        w, r, _ = bench.dist_init("gloo")
        t = bench.reduce_max(1.5 + rank, w)          # per-rank step time: the job takes the slowest
        n = bench.reduce_sum(1e9 * (rank + 1), w)    # per-rank terms: the job did them all
        dist.barrier()
        q.put((r, w, t, n, n / t))
        dist.destroy_process_group()
    except Exception as e:   # report instead of hanging the parent
        q.put(("error", repr(e)))


def test_replica_reductions_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        res = [q.get(timeout=180) for _ in procs]
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(r[0] != "error" for r in res), res
    assert sorted(r[0] for r in res) == [0, 1]
    for _, w, t, n, v in res:
        assert w == 2
        assert t == 2.5
        assert n == 3e9
        assert v == 3e9 / 2.5


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_max(3.25, 1) == 3.25
    assert bench.reduce_sum(7.0, 1) == 7.0
