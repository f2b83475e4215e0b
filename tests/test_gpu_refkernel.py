"""Against the reference's own GPU kernel: ComputeDirects
(singlestep/Direct/PencilKernel.cu) compiled from the reference sources for
sm_100a with its default GPU configuration (fast-math rsqrt without a
Newton step, BLOCK_ACCUM, float accumulation; oracle/_ref, built by
oracle/Makefile), driven on the reference's SIC layout for whole x-slabs.

* parity: this library's slab forces agree with the reference kernel's
  within the tolerance of the other tests (the reference kernel's own error
  is ~1e-6);
* the reference-kernel bar: pair interactions/s of the reference kernel on
  the same GPU next to this library's batched sweep (printed; run with -s).
  NF_REFKERNEL_WORKLOAD=clustered256 measures the default bench box.
"""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("softening", [0, 1])
def test_slabs_match_reference_gpu_kernel(capi, synth, oracle, softening):
    if not oracle.have_ref_gpu(softening):
        pytest.skip("reference GPU kernel not built (needs the reference sources)")
    box = synth.clustered_box(60000, 13, seed=71, n_clumps=20)
    eps = synth.kernel_eps(softening, synth.plummer_eps(39))
    with capi.Context(softening=softening, eps=eps) as ctx:
        db = ctx.box(box)
        for slab in (0, 6, 12):
            ref, _, pairs = oracle.ref_gpu_slab(box, softening, eps, slab)
            got = db.forces(slab, slab + 1)[:, :3]
            assert db.pair_count(slab, slab + 1) == pairs
            norm = np.linalg.norm(ref.astype(np.float64), axis=1)
            diff = np.abs(got.astype(np.float64) - ref)
            ok = norm > 0
            assert np.all(diff[ok] <= 1e-4 * norm[ok, None]), float((diff[ok] / norm[ok, None]).max())
        db.close()


@pytest.mark.parametrize("softening", [0, 1])
def test_2d_nodes_match_reference_gpu_kernel(capi, synth, oracle, softening):
    """2D z-split: the drop-in driver on each node of a z-partition against
    the reference kernel on the same nodes' SICs (sink pencils truncated to
    the node's cells, ghost cells as sources)."""
    if not oracle.have_ref_gpu(softening):
        pytest.skip("reference GPU kernel not built (needs the reference sources)")
    box = synth.clustered_box(50000, 13, seed=72, n_clumps=20)
    length = synth.plummer_eps(37)
    eps = synth.kernel_eps(softening, length)
    cpd = box.cpd
    cellz = np.repeat(np.arange(cpd ** 3) % cpd, np.diff(box.cell_start))
    for zs, zn in [(11, 5), (3, 4), (7, 4)]:
        drv = capi.Driver(box, softening=softening, softening_length=length, direct_bpd=2,
                          node_z=(zs, zn))
        try:
            got = drv.run_all()[:, :3]
        finally:
            drv.close()
        for slab in (0, 6, 12):
            p0, p1 = box.slab_range(slab)
            ref, _, _ = oracle.ref_gpu_slab(box, softening, eps, slab, node=(zs, zn))
            prim = (cellz[p0:p1] - zs) % cpd < zn
            r, g = ref[prim].astype(np.float64), got[p0:p1][prim].astype(np.float64)
            norm = np.linalg.norm(r, axis=1)
            ok = norm > 0
            diff = np.abs(g - r)
            assert np.all(diff[ok] <= 1e-4 * norm[ok, None]), \
                float((diff[ok] / norm[ok, None]).max())


def _check_xyzw(got, ref, b2, what):
    """Forces within 1e-4 |a_ref| per component; the density sum w within
    1e-4 relative as well: both sides add w as one plain FP32 running sum per
    pencil over up to thousands of terms (the reference kernel's a.w,
    PencilKernel.cu:115-183), whose own rounding reaches a few 1e-5 in the
    clumps."""
    r, g = ref.astype(np.float64), got.astype(np.float64)
    norm = np.linalg.norm(r[:, :3], axis=1)
    ok = norm > 0
    diff = np.abs(g[:, :3] - r[:, :3])
    assert np.all(diff[ok] <= 1e-4 * norm[ok, None]), (what, float((diff[ok] / norm[ok, None]).max()))
    # every sink's own pair adds b2 (r = 0 < b), so w >= b2
    assert np.all(r[:, 3] >= b2 * (1 - 1e-6)), what
    np.testing.assert_allclose(g[:, 3], r[:, 3], rtol=1e-4, atol=0, err_msg=what)


@pytest.mark.parametrize("softening", [0, 1])
def test_density_channel_matches_reference_gpu_kernel(capi, synth, oracle, softening):
    """The FOF density channel (b2 > 0): the reference kernel's
    direct_density (DirectGPUKernels.cuh, w += b2 - r^2 for r^2 < b2, built
    with COMPUTE_FOF_DENSITY) against the batched sweep, the drop-in driver
    and one node of a 2D z-split, x, y, z and w per sink."""
    if not oracle.have_ref_gpu(softening):
        pytest.skip("reference GPU kernel not built (needs the reference sources)")
    box = synth.clustered_box(60000, 13, seed=73, n_clumps=20)
    length = synth.plummer_eps(39)
    eps = synth.kernel_eps(softening, length)
    b2 = float(np.float32((0.2 / box.cpd) ** 2))  # a fifth of a cell width
    with capi.Context(softening=softening, eps=eps, b2=b2) as ctx:
        db = ctx.box(box)
        got_box = db.forces()
        db.close()
    drv = capi.Driver(box, softening=softening, softening_length=length, b2=b2, direct_bpd=2)
    try:
        got_drv = drv.run_all()
    finally:
        drv.close()
    zs, zn = 4, 5
    drv = capi.Driver(box, softening=softening, softening_length=length, b2=b2, direct_bpd=2,
                      node_z=(zs, zn))
    try:
        got_node = drv.run_all()
    finally:
        drv.close()
    cpd = box.cpd
    cellz = np.repeat(np.arange(cpd ** 3) % cpd, np.diff(box.cell_start))
    multi = 0
    for slab in (0, 6, 12):
        p0, p1 = box.slab_range(slab)
        ref, _, _ = oracle.ref_gpu_slab(box, softening, eps, slab, b2=b2, with_w=True)
        assert ref.shape == (p1 - p0, 4)
        multi += int((ref[:, 3] > 1.5 * b2).sum())  # sinks with neighbours inside b
        _check_xyzw(got_box[p0:p1], ref, b2, f"batched slab {slab}")
        _check_xyzw(got_drv[p0:p1], ref, b2, f"drop-in slab {slab}")
        refn, _, _ = oracle.ref_gpu_slab(box, softening, eps, slab, b2=b2, with_w=True,
                                         node=(zs, zn))
        prim = (cellz[p0:p1] - zs) % cpd < zn
        _check_xyzw(got_node[p0:p1][prim], refn[prim], b2, f"2D node slab {slab}")
        # both against the FP64 density sum: ours is no worse than the reference's
        sinks = np.arange(p0, p1, 7)
        w64 = oracle.fp64_density(box, b2, sinks)
        e_ours = np.abs(got_box[sinks, 3] - w64) / w64
        e_ref = np.abs(ref[sinks - p0, 3] - w64) / w64
        assert e_ours.max() <= 1e-4 and np.sqrt(np.mean(e_ours ** 2)) <= 2 * np.sqrt(np.mean(e_ref ** 2)) + 1e-7
    assert multi > 1000


def test_reference_kernel_bar(capi, synth, oracle):
    if not oracle.have_ref_gpu(1):
        pytest.skip("reference GPU kernel not built (needs the reference sources)")
    sys.path.insert(0, str(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
    import bench
    wl = os.environ.get("NF_REFKERNEL_WORKLOAD", "clustered128")
    w = bench.WORKLOADS[wl]
    box = bench.make_box(w)
    eps = bench.kernel_eps(w)
    soft = w["softening"]
    ref_ms, ref_pairs = 0.0, 0
    for slab in range(box.cpd):
        _, ms, pairs = oracle.ref_gpu_slab(box, soft, eps, slab, repeats=2)
        ref_ms += ms
        ref_pairs += pairs
    with capi.Context(softening=soft, eps=eps) as ctx:
        db = ctx.box(box)
        for _ in range(3):
            db.forces()
        ours_ms = min((db.forces(), ctx.last_timing().kernel_ms)[1] for _ in range(3))
        pairs = db.pair_count()
        db.close()
    assert pairs == ref_pairs
    ref_rate, ours_rate = ref_pairs / (ref_ms / 1e3), pairs / (ours_ms / 1e3)
    print(f"\n[reference-kernel bar] {wl}: reference ComputeDirects (sm_100a, one SIC per slab) "
          f"{ref_ms:.1f} ms = {ref_rate:.3e} pairs/s; this library's batched sweep "
          f"{ours_ms:.1f} ms = {ours_rate:.3e} pairs/s; ratio {ours_rate / ref_rate:.2f}")
    assert ours_rate > ref_rate
