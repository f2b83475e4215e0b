"""The SetInteractionCollection planner and NearFieldDriver split planning
(CPU only: a planner-only driver, device = -1).

Invariants follow the reference planner (singlestep/Direct/PencilOnPencil.cc:
180-418): every sink cell lies in 2R+1 sink pencils, sink pencils are padded
to 64-particle blocks, each sink pencil meets 2R+1 source pencils, and
DirectTotal is the exact 5x5x5 pair count of the rows.
"""
import numpy as np
import pytest


def _rows_pairs(oracle, box, slab, jlow, jhigh, R=2):
    cpd = box.cpd
    c = box.counts.reshape(cpd, cpd, cpd)
    tot = 0
    for y in range(jlow, jhigh):
        for z in range(cpd):
            ns = int(c[slab, y, z])
            if not ns:
                continue
            xs = [(slab + d) % cpd for d in range(-R, R + 1)]
            ys = [(y + d) % cpd for d in range(-R, R + 1)]
            zs = [(z + d) % cpd for d in range(-R, R + 1)]
            tot += ns * int(c[np.ix_(xs, ys, zs)].sum())
    return tot


@pytest.fixture(scope="module")
def planner(capi, synth):
    box = synth.clustered_box(60000, 13, seed=31, n_clumps=30)
    drv = capi.Driver(box, softening=1, softening_length=1e-3, device=-1, mem_gb=0.05)
    yield box, drv
    drv.close()


@pytest.mark.parametrize("slab,jlow,jhigh", [(0, 0, 13), (5, 2, 7), (12, 11, 13), (6, 0, 1)])
def test_sic_counts(planner, oracle, slab, jlow, jhigh):
    box, drv = planner
    s, sink_count, parent, src_count = drv.plan_sic(slab, jlow, jhigh)
    cpd, R, W = box.cpd, 2, 5
    jw = jhigh - jlow
    assert s.nsinksets == jw * cpd
    assert s.nsourcesets == cpd * (jw + 2 * R)
    assert s.interaction_count == W * s.nsinksets
    c = box.counts.reshape(cpd, cpd, cpd)
    # each sink cell is counted once per pencil it lies in
    assert s.sink_total == W * int(c[slab, jlow:jhigh, :].sum())
    # pencil k is centred on z = (k + R) mod cpd (index_to_zcen)
    for j in range(jw):
        for k in range(cpd):
            zc = (k + R) % cpd
            want = sum(int(c[slab, jlow + j, (zc + a) % cpd]) for a in range(-R, R + 1))
            assert sink_count[j * cpd + k] == want
    # source pencils: rows jlow-R .. jhigh+R-1, cells slab-R .. slab+R at zc
    for j in range(jw + 2 * R):
        y = (jlow - R + j) % cpd
        for k in range(cpd):
            zc = (k + R) % cpd
            want = sum(int(c[(slab + a) % cpd, y, zc]) for a in range(-R, R + 1))
            assert src_count[j * cpd + k] == want
    blocks = (sink_count + 63) // 64
    assert s.nsinkblocks == int(blocks.sum())
    assert s.padded_sink_total == 64 * s.nsinkblocks
    assert np.array_equal(parent, np.repeat(np.arange(s.nsinksets), blocks))
    assert s.direct_total == _rows_pairs(oracle, box, slab, jlow, jhigh)
    assert s.padded_direct_total >= s.direct_total


def test_whole_box_direct_total(planner, oracle):
    box, drv = planner
    tot = sum(drv.plan_sic(s, 0, box.cpd)[0].direct_total for s in range(box.cpd))
    assert tot == oracle.pair_count(box)


def test_planner_limits_refuse_oversized_sics(capi, synth):
    box = synth.clustered_box(200000, 13, seed=32, n_clumps=10)
    drv = capi.Driver(box, softening=0, softening_length=1e-3, device=-1, mem_gb=0.0011)
    try:
        with pytest.raises(capi.NfError) as ei:
            drv.plan_sic(3, 0, 13)
        assert ei.value.status == capi.NF_EINVAL
    finally:
        drv.close()


def test_execute_without_gpu_is_an_error(planner, capi):
    box, drv = planner
    with pytest.raises(capi.NfError) as ei:
        drv.execute_slab(0)
    assert ei.value.status == capi.NF_EINVAL


def _zcen_2d(k, zs, zn, R, cpd):
    """index_to_zcen with the 2D pad (PencilOnPencil.cc:37-43)."""
    kk = k + zs + R
    if kk >= zs + zn + R:
        kk -= zn + 2 * R
    return kk % cpd


@pytest.mark.parametrize("zs,zn", [(3, 5), (10, 5), (0, 9)])
def test_sic_counts_2d_node(capi, synth, zs, zn):
    """One node of a 2D z-split: Nk = zn + 2R pencils centred from zs - R,
    sink pencils truncated to the primary cells, source pencils over ghost
    cells too (PencilOnPencil.cc:200-204, PencilPlan.cc:95-138, 260-279)."""
    box = synth.clustered_box(40000, 13, seed=33, n_clumps=20)
    cpd, R, W = box.cpd, 2, 5
    drv = capi.Driver(box, softening=1, softening_length=1e-3, device=-1, mem_gb=0.05,
                      node_z=(zs, zn))
    try:
        c = box.counts.reshape(cpd, cpd, cpd)
        primary = [(zs + i) % cpd for i in range(zn)]
        nk = zn + 2 * R
        for slab, jlow, jhigh in [(0, 0, 13), (7, 3, 8)]:
            s, sink_count, parent, src_count = drv.plan_sic(slab, jlow, jhigh)
            jw = jhigh - jlow
            assert s.nsinksets == jw * nk and s.nsourcesets == nk * (jw + 2 * R)
            assert s.sink_total == W * int(c[slab, jlow:jhigh][:, primary].sum())
            for j in range(jw):
                for k in range(nk):
                    zc = _zcen_2d(k, zs, zn, R, cpd)
                    want = sum(int(c[slab, jlow + j, (zc + a) % cpd]) for a in range(-R, R + 1)
                               if (zc + a - zs) % cpd < zn)
                    assert sink_count[j * nk + k] == want
            for j in range(jw + 2 * R):
                y = (jlow - R + j) % cpd
                for k in range(nk):
                    zc = _zcen_2d(k, zs, zn, R, cpd)
                    want = sum(int(c[(slab + a) % cpd, y, zc]) for a in range(-R, R + 1))
                    assert src_count[j * nk + k] == want
            blocks = (sink_count + 63) // 64
            assert np.array_equal(parent, np.repeat(np.arange(s.nsinksets), blocks))
    finally:
        drv.close()


def test_2d_nodes_cover_the_box(capi, oracle, synth):
    """Nodes that split z between them plan exactly the box's pair count."""
    box = synth.clustered_box(40000, 13, seed=34, n_clumps=20)
    tot = 0
    for zs, zn in [(0, 5), (5, 4), (9, 4)]:
        drv = capi.Driver(box, softening=0, softening_length=1e-3, device=-1, mem_gb=0.05,
                          node_z=(zs, zn))
        try:
            tot += sum(drv.plan_sic(s, 0, box.cpd)[0].direct_total for s in range(box.cpd))
        finally:
            drv.close()
    assert tot == oracle.pair_count(box)


@pytest.mark.parametrize("zs,zn", [(0, 10), (13, 3), (-1, 3)])
def test_2d_node_geometry_refused(capi, synth, zs, zn):
    box = synth.uniform_box(2000, 13, seed=35)
    with pytest.raises(capi.NfError) as ei:
        capi.Driver(box, softening=0, softening_length=1e-3, device=-1, node_z=(zs, zn))
    assert ei.value.status == capi.NF_EINVAL
