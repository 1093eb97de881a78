"""bench.py with N > 1 ranks: one independent replica per GPU, timing taken as
the maximum over ranks (no data-path collective).  The host logic runs here as
two gloo ranks on the CPU."""
import multiprocessing as mp
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench

    w, r, local, pg = bench.dist_setup()
    mx = bench.max_over_ranks(10.0 * (rank + 1), pg)  # each rank's own step time
    bench.barrier(pg)
    q.put((r, w, local, mx))
    pg.destroy_process_group()


def test_two_ranks_take_the_max_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=5) for _ in range(2))
    assert [g[0] for g in got] == [0, 1]
    assert all(g[1] == 2 and g[3] == 20.0 for g in got)


def _ref_rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import contextlib
    import io

    import bench

    class A:
        steps, warmup = 1, 0

    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        if rank != 0:
            bench.run_reference_arm(A)  # ranks other than 0 exit without work
    q.put((rank, buf.getvalue()))


def test_reference_arm_prints_only_on_rank_zero():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    p = ctx.Process(target=_ref_rank_main, args=(1, 2, port, q))
    # rank 1 alone: it must not wait for rank 0 or print anything
    p.start()
    p.join(timeout=60)
    assert p.exitcode == 0
    rank, out = q.get(timeout=5)
    assert rank == 1 and out == ""
