"""Slab sharding of one box (abacus-public_b200/shard.py) on CPU: the
partition, the windows, and the halo exchange between gloo ranks
(127.0.0.1), checked against the whole box."""
import os
import socket

import numpy as np
import pytest


def test_partition_and_windows(synth):
    from abacus_public_b200 import shard
    for cpd, world in [(17, 1), (17, 2), (17, 3), (65, 8), (9, 4)]:
        parts = shard.partition(cpd, world)
        assert parts[0][0] == 0 and parts[-1][1] == cpd
        assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
        assert max(h - l for l, h in parts) - min(h - l for l, h in parts) <= 1
    assert shard.window_slabs(0, 3, 17) == [0, 1, 2, 3, 4, 15, 16]
    assert shard.window_slabs(5, 8, 17) == [3, 4, 5, 6, 7, 8, 9]
    assert shard.window_slabs(0, 14, 17) == list(range(17))  # window wraps onto itself
    with pytest.raises(ValueError):
        shard.partition(5, 6)
    with pytest.raises(ValueError):
        shard.halo_plan(0, 9, 17)  # a rank would own fewer than R slabs
    # weighted: a heavy slab pulls the cuts towards it, ranges stay >= min_slabs
    w = np.ones(17)
    w[3] = 40.0
    parts = shard.partition(17, 3, weights=w, min_slabs=2)
    assert parts[0][0] == 0 and parts[-1][1] == 17
    assert all(h - l >= 2 for l, h in parts)
    assert parts[0][1] <= 5  # the first range ends soon after the heavy slab


def test_window_box_matches_whole_box(synth):
    from abacus_public_b200 import shard
    box = synth.clustered_box(40000, 13, seed=5, n_clumps=20)
    lo, hi = 4, 8
    ws = shard.window_slabs(lo, hi, box.cpd)
    wb = shard.window_box(box.cpd, shard.extract(box, ws))
    c2 = box.cpd ** 2
    for s in range(box.cpd):
        if s in ws:
            assert np.array_equal(wb.counts[s * c2:(s + 1) * c2], box.counts[s * c2:(s + 1) * c2])
            a0, a1 = box.slab_range(s)
            b0, b1 = wb.slab_range(s)
            assert np.array_equal(wb.x[b0:b1], box.x[a0:a1])
            assert np.array_equal(wb.z[b0:b1], box.z[a0:a1])
        else:
            assert wb.counts[s * c2:(s + 1) * c2].sum() == 0
    assert wb.cell_start[-1] == wb.n


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime
    import pathlib
    import sys
    root = pathlib.Path(__file__).resolve().parents[1]
    sys.path.insert(0, str(root))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        bench._pkg()
        from abacus_public_b200 import shard, synth
        box = synth.clustered_box(30000, 11, seed=9, n_clumps=15)  # every rank: the same box
        lo, hi, left, right, lh, rh = shard.halo_plan(rank, world, box.cpd)
        owned = shard.extract(box, range(lo, hi))
        halo = shard.exchange(owned, rank, world, box.cpd)
        want = shard.extract(box, lh + rh)
        ok = sorted(halo) == sorted(want) and all(
            np.array_equal(halo[s].counts, want[s].counts) and np.array_equal(halo[s].x, want[s].x)
            and np.array_equal(halo[s].y, want[s].y) and np.array_equal(halo[s].z, want[s].z)
            for s in want)
        # the same exchange on tensors (the device-resident form; CPU tensors here)
        import torch
        owned_t = {s: (d.counts, torch.from_numpy(np.stack([d.x, d.y, d.z])))
                   for s, d in owned.items()}
        halo_t = shard.exchange_device(owned_t, rank, world, box.cpd)
        ok = ok and sorted(halo_t) == sorted(want) and all(
            np.array_equal(halo_t[s][0], want[s].counts)
            and np.array_equal(halo_t[s][1].numpy(), np.stack([want[s].x, want[s].y, want[s].z]))
            for s in want)
        # the bench's sharded arm: ranges cut by pair count (at least R slabs
        # each), the tensor exchange given those ranges
        parts = shard.partition(box.cpd, world, weights=shard.slab_pairs(box), min_slabs=2)
        plo, phi = parts[rank]
        owned_w = {s: (d.counts, torch.from_numpy(np.stack([d.x, d.y, d.z])))
                   for s, d in shard.extract(box, range(plo, phi)).items()}
        halo_w = shard.exchange_device(owned_w, rank, world, box.cpd, parts=parts)
        need = [s for s in shard.window_slabs(plo, phi, box.cpd) if not plo <= s < phi]
        want_w = shard.extract(box, need)
        ok = ok and sorted(halo_w) == sorted(want_w) and all(
            np.array_equal(halo_w[s][1].numpy(), np.stack([want_w[s].x, want_w[s].y, want_w[s].z]))
            for s in want_w)
        q.put((rank, ok, sorted(halo)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_halo_exchange_gloo(world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ok, got in res:
        assert ok, (rank, got)
