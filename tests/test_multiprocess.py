"""The N>1 path of bench.py on CPU: two gloo ranks (127.0.0.1) run the
rank helpers the GPU run uses (independent box per rank, whole-job pairs
over the slowest rank's time, barrier), without a GPU."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import sys
    import pathlib
    root = pathlib.Path(__file__).resolve().parents[1]
    sys.path.insert(0, str(root))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import datetime
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        w = dict(bench.WORKLOADS["uniform64"])
        w["n_side"] = 16  # small box, same code path
        w["cpd"] = 5
        box = bench.make_box(w, seed_offset=bench.rank_seed_offset(rank))
        bench.barrier(world)
        # rank r "processes" (r+1) pairs in (10 r + 5) ms
        value, ms = bench.aggregate(rank + 1.0, 10.0 * rank + 5.0, world)
        q.put((rank, float(box.x[0]), value, ms))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    # independent boxes per rank
    assert res[0][1] != res[1][1]
    # whole-job rate = (1 + 2) pairs / max(5, 15) ms, identical on both ranks
    for _, _, value, ms in res:
        assert ms == pytest.approx(15.0)
        assert value == pytest.approx(3.0 / 0.015)
