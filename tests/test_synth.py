"""Synthetic box generators (CPU only)."""
import numpy as np


def test_uniform_layout(synth):
    box = synth.uniform_box(20000, 9, seed=3)
    h = 1.0 / 9
    assert box.n == 20000 and box.cell_start[-1] == 20000
    for a in (box.x, box.y, box.z):
        assert a.dtype == np.float32
        assert a.min() >= -0.5 * h - 1e-9 and a.max() < 0.5 * h
    g = box.global_positions()
    c = np.floor((g + 0.5) * 9).astype(int)
    cid = (c[:, 0] * 9 + c[:, 1]) * 9 + c[:, 2]
    assert np.all(np.diff(cid) >= 0)
    assert np.array_equal(np.bincount(cid, minlength=729), box.counts)


def test_clustered_fraction_and_seed(synth):
    a = synth.clustered_box(50000, 11, seed=5, n_clumps=30)
    b = synth.clustered_box(50000, 11, seed=5, n_clumps=30)
    assert np.array_equal(a.x, b.x) and np.array_equal(a.cell_start, b.cell_start)
    assert a.counts.max() > 5 * a.counts.mean()


def test_kernel_eps(synth):
    e = synth.plummer_eps(64)
    assert abs(e - 1 / 64 / 40) < 1e-15
    assert synth.kernel_eps(0, e) == np.float32(e * e)
    assert synth.kernel_eps(1, e) == np.float32(1 / (e * 2.15517) ** 2)


def test_device_generator_layout(synth):
    """The GPU generator (run here on CPU tensors) keeps the box layout:
    cell order, counts summing to n, positions inside their cells, the
    clumped fraction visible as crowded cells, and a fixed seed."""
    x, y, z, cs = synth.clustered_box_device(60000, 13, seed=4, device="cpu", chunk=1 << 14)
    assert x.shape[0] == 60000 and cs[-1] == 60000 and cs[0] == 0
    assert np.all(np.diff(cs) >= 0)
    h = 0.5 / 13
    for a in (x, y, z):
        a = a.numpy()
        assert a.dtype == np.float32 and np.all(np.abs(a) <= h)
    counts = np.diff(cs)
    assert counts.max() > 5 * counts.mean()  # clumps
    x2, _, _, cs2 = synth.clustered_box_device(60000, 13, seed=4, device="cpu", chunk=1 << 14)
    assert np.array_equal(cs, cs2) and np.array_equal(x.numpy(), x2.numpy())
