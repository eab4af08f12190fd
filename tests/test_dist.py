"""The multi-process plumbing of bench.py on CPU: world_size 2 over gloo.

The engine's multi-GPU form is replicas (one independent trajectory per GPU, no
data-path collective); what crosses ranks is the barrier around the timed region,
the max over ranks of the device time, and the per-rank input seed.
"""
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
    try:
        os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                           "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
        sys.path.insert(0, ROOT)
        import bench
        d = bench.Dist(world, backend="gloo", timeout_s=60)
        d.barrier()
        secs = 0.5 + rank  # rank 1 is the slow one
        m = d.max(secs)
        d.barrier()
        seed = bench.rank_seed(7, d.rank)
        d.close()
        q.put((rank, m, seed, bench.replica_value(3, world, m)))
    except Exception as e:  # report instead of hanging the parent
        q.put((rank, repr(e), None, None))


def test_two_gloo_ranks_time_by_the_slowest_and_run_distinct_inputs():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(2):
        r, m, seed, v = q.get(timeout=120)
        out[r] = (m, seed, v)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(2):
        assert out[r][0] == 1.5, out  # max over ranks, seen identically by both
        assert out[r][2] == 3 * 2 / 1.5  # whole-job steps / slowest rank's time
    assert out[0][1] != out[1][1]  # each replica its own molecule


def test_single_process_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        os.environ.pop(k, None)
    d = bench.Dist(1)
    assert d.pg is None and d.max(2.5) == 2.5
    d.barrier()
    d.close()
