"""nf_forces_noalloc: the allocation-free entry point, through the C ABI.

It serves callers that cannot call cudaMalloc (code living inside another
framework's device memory pool or caching allocator, or a process whose
device allocations are fixed after start-up): its only scratch is a static
device array inside the library.  Here it is checked against the regular
entry point (nf_box_forces) with the tolerance the other GPU tests use, on
two calls in a row, since every call reuses the same scratch.  The test
itself allocates its inputs and outputs with torch; the entry point does not.
This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_inputs(box):
    import torch
    rec = np.zeros((box.n, 4), np.float32)
    rec[:, 0], rec[:, 1], rec[:, 2] = box.x, box.y, box.z
    pos = torch.from_numpy(rec).cuda()
    cs = torch.from_numpy(np.ascontiguousarray(box.cell_start, dtype=np.int64)).cuda()
    return pos, cs


def _noalloc(capi, cfg, box, pos, cs, lo, hi, n_out):
    import torch
    width = 4 if cfg.out_kind == capi.OUT_FLOAT4 else 3
    out = torch.full((n_out, width), float("nan"), dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    capi.check(capi.lib().nf_forces_noalloc(ctypes.byref(cfg), box.cpd, pos.data_ptr(),
                                            cs.data_ptr(), lo, hi, out.data_ptr(),
                                            ctypes.c_void_p(stream.cuda_stream or 0)),
               "nf_forces_noalloc")
    torch.cuda.synchronize()
    return out.cpu().numpy()


# (softening, b2 > 0, output record): every softening with float4 records,
# the density channel (a fourth partial per sink in the shared scratch) for
# the two softenings with the fast path, and float3 records
CASES = [(0, False, "f4"), (1, False, "f4"), (2, False, "f4"), (3, False, "f4"),
         (0, True, "f4"), (1, True, "f4"), (1, False, "f3"), (0, False, "f3")]


@pytest.mark.parametrize("soft,dens,rec", CASES)
def test_noalloc_matches_regular_entry_point(capi, synth, soft, dens, rec):
    box = synth.clustered_box(60000, 13, seed=51, n_clumps=30)
    eps = synth.kernel_eps(soft, synth.plummer_eps(39))
    # density radius: a fifth of a cell, so that w sums over many neighbours
    b2 = float(np.float32((0.2 / box.cpd) ** 2)) if dens else 0.0
    kw = dict(softening=soft, eps=eps, b2=b2,
              out_kind=capi.OUT_FLOAT4 if rec == "f4" else capi.OUT_FLOAT3)
    with capi.Context(**kw) as ctx:
        db = ctx.box(box)
        ref = db.forces()
        ref_part = db.forces(3, 8)
        p0, p1 = db.slab_particles(3, 8)
        db.close()
    cfg = capi.default_config(**kw)
    pos, cs = _device_inputs(box)
    norm = np.linalg.norm(ref[:, :3].astype(np.float64), axis=1)
    for _ in range(2):  # two calls in a row share the static scratch
        a = _noalloc(capi, cfg, box, pos, cs, 0, box.cpd, box.n)
        assert a.shape == ref.shape
        assert np.isfinite(a).all()
        diff = np.abs(a[:, :3].astype(np.float64) - ref[:, :3])
        assert np.all(diff <= 1e-4 * norm[:, None] + 1e-30), float((diff / norm[:, None]).max())
        np.testing.assert_allclose(a[:, :3], ref[:, :3], rtol=0,
                                   atol=2e-6 * np.abs(ref[:, :3]).max())
        if rec == "f4":
            # w: the density sum (b2 > 0; 1e-5 relative, the density tolerance
            # of the other GPU tests) or exactly 0
            if dens:
                assert (ref[:, 3] > 0).mean() > 0.5
                np.testing.assert_allclose(a[:, 3], ref[:, 3], rtol=1e-5,
                                           atol=1e-5 * np.abs(ref[:, 3]).max())
            else:
                assert np.all(a[:, 3] == 0) and np.all(ref[:, 3] == 0)
        b = _noalloc(capi, cfg, box, pos, cs, 3, 8, p1 - p0)
        np.testing.assert_allclose(b[:, :3], ref_part[:, :3], rtol=0,
                                   atol=2e-6 * np.abs(ref_part[:, :3]).max())


def test_noalloc_rejects_sizes_beyond_its_scratch(capi, synth):
    box = synth.uniform_box(200000, 7, seed=52)
    cfg = capi.default_config(softening=0, eps=1e-6)
    pos, cs = _device_inputs(box)
    with pytest.raises(capi.NfError) as ei:
        _noalloc(capi, cfg, box, pos, cs, 0, box.cpd, box.n)
    assert ei.value.status == capi.NF_EINVAL
    assert "196608" in str(ei.value)
    # a slab range that fits is accepted
    c2 = box.cpd ** 2
    n1 = int(box.cell_start[c2] - box.cell_start[0])
    assert n1 <= 196608
    a = _noalloc(capi, cfg, box, pos, cs, 0, 1, n1)
    assert np.isfinite(a).all()
