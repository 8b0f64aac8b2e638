"""The multi-rank plumbing of bench.py on the CPU (gloo, two ranks, spawned).

`bench.py --gpus N` shards the cells (an independent field per rank, no
data-path collective) and reduces only the timing: every rank takes the same
barrier and the max over ranks of its time. Here: that reduction over two
gloo ranks; the per-rank fields (independent seeds, equal sizes); and a rank
that fails before the reduction, which the other rank learns of as an error
from its collective instead of waiting for good."""
import datetime
import multiprocessing as mp
import os
import socket


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _init(rank, world, port, timeout_s):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def _timing_worker(rank, world, port, q):
    dist = _init(rank, world, port, 60)
    import bench
    bench.barrier(world)
    t = bench.max_over_ranks(0.5 + rank, world)
    f = bench.head_field(4096, seed=bench.HEAD_SEED + rank)
    q.put((rank, t, f.n, float(f.T.sum())))
    dist.barrier()
    dist.destroy_process_group()


def _failing_worker(rank, world, port, q):
    dist = _init(rank, world, port, 10)
    import bench
    bench.barrier(world)
    if rank == 1:
        q.put((rank, "left"))
        q.close()
        q.join_thread()                   # the message is out before the process goes
        os._exit(3)                       # leaves between steps: no collective of its own in flight
    try:
        bench.max_over_ranks(1.0, world)
        q.put((rank, "no error"))
    except Exception as e:                # the dead peer surfaces as an error of the collective
        q.put((rank, type(e).__name__))


def _run(target, world=2, wait=90):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    ps = [ctx.Process(target=target, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    out = [q.get(timeout=wait) for _ in range(world)]
    for p in ps:
        p.join(timeout=wait)
        if p.is_alive():
            p.kill()
    return sorted(out), [p.exitcode for p in ps]


def test_max_over_ranks_and_per_rank_fields():
    out, codes = _run(_timing_worker)
    assert codes == [0, 0]
    assert [o[1] for o in out] == [1.5, 1.5]                 # max of 0.5 and 1.5 on both ranks
    assert out[0][2] == out[1][2] == 4096                     # weak scaling: equal work per rank
    assert out[0][3] != out[1][3]                             # independent fields


def test_a_rank_that_leaves_is_seen_by_the_other():
    out, codes = _run(_failing_worker)
    assert out[1] == (1, "left") and codes[1] == 3
    assert out[0][0] == 0 and out[0][1] != "no error"
