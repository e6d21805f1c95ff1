"""The N-rank path of bench.py on CPU: two gloo ranks on 127.0.0.1.

Ranks are replicas (views are independent), so the only collectives are the
barrier before the timed region and the max-over-ranks reduction of its
duration; whole-job throughput is the units all ranks processed over the
slowest rank's time, and the reference arm runs on rank 0 alone.
"""
import multiprocessing as mp
import os
import socket
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import bench
    r, w, _ = bench.dist_info()
    dist = bench.init_dist(w, backend="gloo")
    dist.barrier()
    slowest = bench.max_over_ranks(dist, 1.0 + r, device="cpu")
    value = bench.replica_throughput(1000, slowest, w)
    # the reference arm: rank 0 only; the others exit 0 without work
    ref = bench.main(["--impl", "reference", "--steps", "1", "--warmup", "0", "--cpu-rows", "1"]) if r != 0 else 0
    dist.barrier()
    dist.destroy_process_group()
    out.put((r, w, slowest, value, ref))


def test_two_gloo_ranks_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(out.get(timeout=5) for _ in procs)
    for r, (rank, world, slowest, value, ref) in enumerate(got):
        assert rank == r and world == 2
        assert slowest == 2.0          # max over ranks of 1.0 and 2.0
        assert value == 1000.0         # 2 ranks x 1000 units / 2.0 s
        assert ref == 0                # rank 1's reference arm returns at once


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.init_dist(1) is None
    assert bench.max_over_ranks(None, 3.5) == 3.5
    assert bench.replica_throughput(600, 2.0, 1) == 300.0
