"""The plain drop-in (NearFieldDriver -> SetInteractionCollection ->
nf_sic_execute) against the oracle, through the C ABI.

Same tolerances as test_gpu_box: |a_k - a_ref,k| <= 1e-4 |a_ref| per sink and
component against the reference CPU direct; RMS fractional error <= 2e-6
against FP64.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _check(oracle, box, soft, eps, a):
    ref = np.zeros((box.n, 3), np.float32)
    for s in range(box.cpd):
        oracle.ref32_slab(box, soft, eps, s, acc=ref)
    norm = np.linalg.norm(ref.astype(np.float64), axis=1)
    diff = np.abs(a[:, :3].astype(np.float64) - ref)
    ok = norm > 0
    assert np.all(diff[ok] <= 1e-4 * norm[ok, None]), float((diff[ok] / norm[ok, None]).max())
    sinks = np.arange(0, box.n, max(1, box.n // 3000))
    rms, mx, _ = oracle.frac_errors(a[sinks, :3], oracle.fp64_sinks(box, soft, eps, sinks))
    assert rms <= 2e-6 and mx <= 1e-4, (rms, mx)


@pytest.mark.parametrize("soft,blocking", [(0, 0), (0, 1), (1, 0), (1, 1), (2, 0), (3, 1)])
def test_driver_matches_oracle(capi, oracle, synth, soft, blocking):
    box = synth.clustered_box(50000, 13, seed=41, n_clumps=30)
    length = synth.plummer_eps(37)
    drv = capi.Driver(box, softening=soft, softening_length=length, direct_bpd=3)
    try:
        a = drv.run_all(blocking=blocking)
        st = drv.stats()
    finally:
        drv.close()
    eps = synth.kernel_eps(soft, length)
    assert np.float32(st.eps) == np.float32(eps)
    assert st.direct_interactions == oracle.pair_count(box)
    assert st.max_nsplits >= 3  # at least one SIC per buffer (MinSplits = NBuffers)
    _check(oracle, box, soft, eps, a)


def test_driver_small_buffers_split_more(capi, oracle, synth):
    """A small GPU buffer budget forces more y-splits; results do not change."""
    box = synth.uniform_box(80000, 15, seed=42)
    length = synth.plummer_eps(43)
    outs, splits = [], []
    for mem in (0.0, 0.0012):  # 1.2 MB: ~190 sink blocks per SIC
        drv = capi.Driver(box, softening=0, softening_length=length, direct_bpd=2, mem_gb=mem)
        try:
            outs.append(drv.run_all())
            splits.append(drv.stats().mean_splits_per_slab)
        finally:
            drv.close()
    assert splits[1] > splits[0]
    np.testing.assert_allclose(outs[1], outs[0], rtol=0, atol=1e-6 * np.abs(outs[0]).max())
    _check(oracle, box, 0, synth.kernel_eps(0, length), outs[1])


def test_driver_density_and_float3(capi, oracle, synth):
    box = synth.clustered_box(30000, 11, seed=43, n_clumps=20)
    length = synth.plummer_eps(31)
    b2 = float(np.float32((0.2 / 31) ** 2))
    drv = capi.Driver(box, softening=0, softening_length=length, b2=b2)
    try:
        a = drv.run_all()
    finally:
        drv.close()
    sinks = np.arange(0, box.n, 9)
    np.testing.assert_allclose(a[sinks, 3], oracle.fp64_density(box, b2, sinks), rtol=1e-5,
                               atol=1e-6 * b2)
    drv = capi.Driver(box, softening=1, softening_length=length, out_kind=capi.OUT_FLOAT3)
    try:
        a3 = drv.run_all()
    finally:
        drv.close()
    assert a3.shape[1] == 3
    _check(oracle, box, 1, synth.kernel_eps(1, length), a3)


def test_driver_errors(capi, synth):
    box = synth.uniform_box(5000, 7, seed=44)
    drv = capi.Driver(box, softening=0, softening_length=1e-3)
    try:
        drv.execute_slab(2)
        with pytest.raises(capi.NfError):
            drv.execute_slab(2)  # already in flight
        with pytest.raises(capi.NfError):
            drv.finalize(3)      # never executed
        drv.run_all_pending = None
        import time
        t0 = time.time()
        while drv.slab_done(2) != 1:
            assert time.time() - t0 < 60
            time.sleep(0.001)
        drv.finalize(2)
    finally:
        drv.close()


@pytest.mark.parametrize("soft,nodes,out_kind", [(0, [(0, 5), (5, 4), (9, 4)], 0),
                                                 (1, [(11, 5), (3, 4), (7, 4)], 0),
                                                 (2, [(2, 7), (9, 6)], 1)])
def test_driver_2d_z_split(capi, oracle, synth, soft, nodes, out_kind):
    """A 2D (x, z) split: each node runs the drop-in on its own z cells plus
    R ghost cells each side (MPI_size_z > 1 layout) and produces its primary
    particles; the nodes together match the one-domain drop-in and the
    oracle.  The second split puts a node's primary range across z = 0."""
    box = synth.clustered_box(50000, 13, seed=44, n_clumps=30)
    length = synth.plummer_eps(37)
    eps = synth.kernel_eps(soft, length)
    ok_kind = capi.OUT_FLOAT4 if out_kind == 0 else capi.OUT_FLOAT3
    a2 = np.zeros((box.n, 4 if out_kind == 0 else 3), np.float32)
    covered = np.zeros(box.n, int)
    for zs, zn in nodes:
        drv = capi.Driver(box, softening=soft, softening_length=length, direct_bpd=2,
                          node_z=(zs, zn), out_kind=ok_kind)
        try:
            a = drv.run_all()
            assert drv.stats().direct_interactions > 0
        finally:
            drv.close()
        m = drv.slabs.mask
        a2[m] = a[m]
        covered += m
    assert np.all(covered == 1)
    drv = capi.Driver(box, softening=soft, softening_length=length, direct_bpd=2,
                      out_kind=ok_kind)
    try:
        a1 = drv.run_all()
    finally:
        drv.close()
    norm = np.linalg.norm(a1[:, :3].astype(np.float64), axis=1)
    ok = norm > 0
    diff = np.abs(a2[:, :3].astype(np.float64) - a1[:, :3])
    assert np.all(diff[ok] <= 2e-6 * norm[ok, None]), float((diff[ok] / norm[ok, None]).max())
    _check(oracle, box, soft, eps, a2)


@pytest.mark.parametrize("node", [None, (4, 6)])
def test_every_record_written(capi, synth, node):
    """ForceOutputDebug's check (singlestep/Timestep/directdriver.cpp:344-356):
    AccSlab pre-filled with +inf, every sink record (of the node's primary
    cells for a 2D node) must come back finite; the batched form's output,
    pre-filled with NaN, likewise."""
    box = synth.clustered_box(40000, 13, seed=45, n_clumps=25)
    length = synth.plummer_eps(34)
    drv = capi.Driver(box, softening=1, softening_length=length, direct_bpd=2, node_z=node)
    try:
        for a in drv.slabs.acc:
            a[:] = np.inf
        acc = drv.run_all()
        mask = drv.slabs.mask if node else np.ones(box.n, bool)
    finally:
        drv.close()
    assert np.all(np.isfinite(acc[mask]))
    with capi.Context(softening=1, eps=synth.kernel_eps(1, length)) as ctx:
        db = ctx.box(box)
        out = np.full((box.n, db.record_width()), np.nan, np.float32)
        db.forces(0, box.cpd, out=out)
        db.close()
    assert np.all(np.isfinite(out))


def test_sic_timing_counts_every_sic(capi, synth, oracle):
    """nf_sic_timing: the summed pencil-kernel time of the SICs of a sweep,
    their count and their unpadded pairs (the sweep's DirectTotal); a reset
    zeroes the counters."""
    box = synth.clustered_box(40000, 11, seed=44, n_clumps=20)
    drv = capi.Driver(box, softening=1, softening_length=synth.plummer_eps(34), direct_bpd=2)
    try:
        drv.run_all()
        ms, n, pairs = drv.sic_timing(reset=True)
        st = drv.stats()
        assert n >= box.cpd and ms > 0.0
        assert pairs == st.direct_interactions == oracle.pair_count(box)
        assert drv.sic_timing() == (0.0, 0, 0)
        drv.run_all()
        ms2, n2, pairs2 = drv.sic_timing()
        assert n2 == n and pairs2 == pairs and ms2 > 0.0
    finally:
        drv.close()
