"""The bench's multi-process plumbing on CPU (gloo, world size 2): every rank joins, the timing
is the max over ranks, and the barrier and shutdown complete (one process per GPU in the GPU
runs, replicas only: the path has no data-path collective)."""
import multiprocessing as mp
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    D = bench.Dist(world)
    D.barrier()
    m = D.max(10.0 * rank + 0.5)
    D.barrier()
    D.close()
    q.put((rank, D.world, m))


def test_two_rank_max_and_barrier():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in ps)
    got = sorted(q.get(timeout=5) for _ in ps)
    assert got == [(0, 2, 10.5), (1, 2, 10.5)]
