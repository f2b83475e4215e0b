"""The serving loop (nf_server_*): continuous admission of slab requests over
resident boxes, through the C ABI.

The key property: a request's result is the same alone and in a mix of
concurrent requests from several boxes (here bit for bit: each slab runs its
own cached plan in a fixed summation order; the stated tolerance, the one of
the other GPU tests, is checked as well).
"""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def two_boxes(synth):
    a = synth.clustered_box(60000, 13, seed=61, n_clumps=30)
    b = synth.clustered_box(90000, 17, seed=62, n_clumps=40)
    return a, b


def _slab_out(db, s):
    p0, p1 = db.slab_particles(s, s + 1)
    return np.full((p1 - p0, db.record_width()), np.nan, np.float32)


def test_alone_equals_in_the_mix(capi, synth, two_boxes):
    boxa, boxb = two_boxes
    eps = synth.kernel_eps(1, synth.plummer_eps(40))
    with capi.Context(softening=1, eps=eps) as ctx:
        da, db_ = ctx.box(boxa), ctx.box(boxb)
        ref_a = da.forces()  # the sweep API, for the tolerance check
        with capi.Server(ctx, max_inflight=6) as srv:
            s0 = 5
            alone = _slab_out(da, s0)
            srv.wait(srv.submit(da, s0, alone))
            # the mix: every slab of both boxes, interleaved, from two threads
            outs, tickets = {}, []
            lock = threading.Lock()

            def feed(box, nslab, tag):
                for s in range(nslab):
                    o = _slab_out(box, s)
                    t = srv.submit(box, s, o)
                    with lock:
                        outs[(tag, s)] = o
                        tickets.append(t)

            th = [threading.Thread(target=feed, args=(da, boxa.cpd, "a")),
                  threading.Thread(target=feed, args=(db_, boxb.cpd, "b"))]
            for t in th:
                t.start()
            for t in th:
                t.join()
            for t in tickets:
                srv.wait(t)
            st = srv.stats()
            infos = [srv.info(t) for t in tickets]
        da.close()
        db_.close()
    mixed = outs[("a", s0)]
    assert np.array_equal(alone.view(np.uint32), mixed.view(np.uint32))
    p0, p1 = boxa.slab_range(s0)
    ref = ref_a[p0:p1]
    np.testing.assert_allclose(mixed, ref, rtol=0, atol=2e-6 * np.abs(ref).max())
    full = np.concatenate([outs[("a", s)] for s in range(boxa.cpd)])
    np.testing.assert_allclose(full, ref_a, rtol=0, atol=2e-6 * np.abs(ref_a).max())
    assert st.completed == 1 + boxa.cpd + boxb.cpd
    assert st.failed == 0 and st.rejected == 0
    assert st.max_concurrent >= 2  # requests overlapped on the device
    assert 0 < st.p50_ms <= st.p99_ms <= st.max_ms
    # per-request records: completed, on a valid slot, latency = queue + run
    for inf in infos:
        assert inf.state == 2 and inf.status == 0 and 0 <= inf.slot < 6 and inf.pairs > 0
        assert inf.queue_ms >= 0 and inf.run_ms > 0
        assert inf.total_ms == pytest.approx(inf.queue_ms + inf.run_ms, abs=1e-6)
    assert max(i.total_ms for i in infos) <= st.max_ms + 1e-9


def test_device_output_and_admission_limits(capi, synth, two_boxes):
    import torch
    boxa, _ = two_boxes
    eps = synth.kernel_eps(0, synth.plummer_eps(40))
    with capi.Context(softening=0, eps=eps) as ctx:
        da = ctx.box(boxa)
        ref = da.forces()
        p0, p1 = da.slab_particles(3, 4)
        # a budget that fits about one slab request at a time: all still complete
        nmax = max(boxa.slab_range(s)[1] - boxa.slab_range(s)[0] for s in range(boxa.cpd))
        need = (5 * 3 * 8 + 16) * nmax + 2048
        with capi.Server(ctx, hbm_budget_bytes=need, max_inflight=4) as srv:
            dev = torch.empty((p1 - p0, 4), dtype=torch.float32, device="cuda")
            srv.wait(srv.submit(da, 3, dev.data_ptr(), out_on_device=True))
            got = dev.cpu().numpy()
            np.testing.assert_allclose(got, ref[p0:p1], rtol=0, atol=2e-6 * np.abs(ref).max())
            outs = [_slab_out(da, s) for s in range(boxa.cpd)]
            tk = [srv.submit(da, s, outs[s]) for s in range(boxa.cpd)]
            for t in tk:
                srv.wait(t)
            st = srv.stats()
            assert st.completed == 1 + boxa.cpd and st.hbm_peak_bytes <= need
        # a budget smaller than one request: refused at submission
        with capi.Server(ctx, hbm_budget_bytes=4096) as srv:
            with pytest.raises(capi.NfError) as ei:
                srv.submit(da, 0, _slab_out(da, 0))
            assert ei.value.status == capi.NF_EADMISSION
            assert srv.stats().rejected == 1
        da.close()


def test_cancel_and_stop(capi, synth, two_boxes):
    _, boxb = two_boxes
    eps = synth.kernel_eps(1, synth.plummer_eps(45))
    with capi.Context(softening=1, eps=eps) as ctx:
        db_ = ctx.box(boxb)
        db_.forces(0, 1)  # plans and tuning done before serving
        with capi.Server(ctx, max_inflight=1) as srv:
            outs = [_slab_out(db_, s % boxb.cpd) for s in range(40)]
            tk = [srv.submit(db_, s % boxb.cpd, outs[s]) for s in range(40)]
            cancelled = 0
            for t in tk[20:]:
                try:
                    srv.cancel(t)
                    cancelled += 1
                except capi.NfError:
                    pass  # already admitted
            assert cancelled > 0
            for t in tk:
                try:
                    srv.wait(t)
                except capi.NfError as e:
                    assert e.status == capi.NF_ECANCELLED
            st = srv.stats()
            assert st.cancelled == cancelled and st.completed == 40 - cancelled
            states = [srv.info(t) for t in tk]
            assert sum(i.state == -2 for i in states) == cancelled
            assert all(i.queue_ms == -1.0 and i.slot == -1 for i in states if i.state == -2)
            with pytest.raises(capi.NfError):
                srv.wait(123456789)  # unknown ticket
        db_.close()


def test_per_box_softening(capi, synth, two_boxes):
    """Boxes of different spacing under one context and one server: a box
    given its own eps (nf_box_set_eps) computes exactly what a context with
    that eps computes, in sweeps and in served slab requests."""
    boxa, boxb = two_boxes
    eps_a = synth.kernel_eps(1, synth.plummer_eps(40))
    eps_b = synth.kernel_eps(1, synth.plummer_eps(45))
    with capi.Context(softening=1, eps=eps_b, kernel_variant=0) as ctx_b:
        db_only = ctx_b.box(boxb)
        want = db_only.forces()
        # single-slab plans (what the server runs) sum in their own fixed order
        want_slabs = np.concatenate([db_only.forces(s, s + 1) for s in range(boxb.cpd)])
        db_only.close()
    with capi.Context(softening=1, eps=eps_a, kernel_variant=0) as ctx:
        da, db_ = ctx.box(boxa), ctx.box(boxb)
        before = db_.forces()  # with the context's eps: differs
        db_.set_eps(eps_b)
        got = db_.forces()
        with capi.Server(ctx, max_inflight=4) as srv:
            outs = [_slab_out(db_, s) for s in range(boxb.cpd)]
            tk = [srv.submit(db_, s, outs[s]) for s in range(boxb.cpd)]
            tka = srv.submit(da, 2, _slab_out(da, 2))
            for t in tk + [tka]:
                srv.wait(t)
        with pytest.raises(capi.NfError):
            db_.set_eps(float("nan"))
        da.close()
        db_.close()
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert not np.array_equal(before, want)
    served = np.concatenate(outs)
    assert np.array_equal(served.view(np.uint32), want_slabs.view(np.uint32))
    np.testing.assert_allclose(served, want, rtol=0, atol=2e-6 * np.abs(want).max())
