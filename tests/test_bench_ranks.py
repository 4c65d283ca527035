"""bench.py's multi-rank path (replicas, one process per GPU under
torchrun) on the host: two gloo ranks on the CPU join, pass the barrier and
agree on the maximum of their times, which is what the bench reports."""
import os
import socket
import sys

import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, out):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    import torch.distributed as dist
    import bench
    w, r, _ = bench.dist_init(backend="gloo", timeout_s=60)
    bench.barrier(w)
    m = bench.max_over_ranks(w, 10.0 + 3.5 * r)
    bench.barrier(w)
    out.put((r, w, m))
    dist.destroy_process_group()


def test_two_ranks_agree_on_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == [(0, 2, 13.5), (1, 2, 13.5)]
