"""One box split over logical ranks, run one after another on one GPU (no
collective, nothing waits on another launch): each rank's window box (its
slabs plus a 2-slab halo, every other cell empty) gives, for the slabs it
owns, exactly the whole box's result."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("world", [2, 3])
def test_window_boxes_equal_whole_box(capi, synth, world):
    from abacus_public_b200 import shard
    box = synth.clustered_box(80000, 15, seed=21, n_clumps=30)
    eps = synth.kernel_eps(1, synth.plummer_eps(43))
    with capi.Context(softening=1, eps=eps, kernel_variant=0) as ctx:
        whole = ctx.box(box)
        for lo, hi in shard.partition(box.cpd, world):
            want = whole.forces(lo, hi)
            wb = shard.window_box(box.cpd, shard.extract(box, shard.window_slabs(lo, hi, box.cpd)))
            db = ctx.box(wb)
            got = db.forces(lo, hi)
            assert db.pair_count(lo, hi) == whole.pair_count(lo, hi)
            db.close()
            assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (lo, hi)
        whole.close()
