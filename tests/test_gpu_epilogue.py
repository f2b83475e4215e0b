"""The steps either side of the near field, on the device: positions given
as (x, y, z) records (nf_box_update_aos), and the near field fused with the
rescale / co-add with the far field and the two half kicks (nf_box_kick),
checked against the sweep plus the oracle's restatement of
singlestep/Timestep/kick.cpp."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def kbox(synth):
    return synth.clustered_box(70000, 15, seed=33, n_clumps=25)


def test_aos_upload_equals_soa(capi, synth, kbox):
    eps = synth.kernel_eps(1, synth.plummer_eps(41))
    with capi.Context(softening=1, eps=eps, kernel_variant=0) as ctx:
        a = ctx.box(kbox)
        want = a.forces()
        b = ctx.box(kbox)
        b.update_aos(np.stack([kbox.x, kbox.y, kbox.z], axis=1))
        got = b.forces()
        a.close()
        b.close()
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("softening,dens", [(0, False), (1, False), (1, True)])
def test_kick_matches_sweep_plus_reference_kick(capi, synth, oracle, kbox, softening, dens):
    """nf_box_kick against the sweep followed by the oracle's restatement of
    kick.cpp and, where it is built, by the reference's own kick.cpp
    (RescaleAndCoAddAcceleration + KickSlab, compiled unmodified): a, w and
    v bit for bit, the cell maxima exactly, the mean square velocity to
    1e-5 (summation order)."""
    import torch
    lo, hi = 3, 11
    length = synth.plummer_eps(41)
    eps = synth.kernel_eps(softening, length)
    L_int = length * (synth.SINGLE_SPLINE_FACTOR if softening == 1 else 1.0)
    cosmo = (0.31, 0.0, kbox.n, 0, L_int)  # Omega_M, Omega_Smooth, np, MakeGlass, L
    rescale, inv_eps3 = oracle.kick_constants(*cosmo)
    near_scale = inv_eps3 if softening == 1 else np.float32(1.0)
    b2 = np.float32((0.2 / kbox.cpd) ** 2) if dens else np.float32(0.0)
    k1, k2 = np.float32(0.013), np.float32(0.011)
    p0, p1 = kbox.slab_range(lo)[0], kbox.slab_range(hi - 1)[1]
    n = p1 - p0
    rng = np.random.default_rng(4)
    far = (rng.standard_normal((n, 3)) * 1e3).astype(np.float32)
    vel = (rng.standard_normal((n, 3)) * 1e-2).astype(np.float32)
    c2 = kbox.cpd ** 2
    counts = kbox.counts[lo * c2:hi * c2]
    ref_kick = oracle.have_ref_kick(softening)
    with capi.Context(softening=softening, eps=eps, b2=float(b2)) as ctx:
        db = ctx.box(kbox)
        nacc = db.forces(lo, hi)
        if dens:
            assert np.all(nacc[:, 3] >= b2 * (1 - 1e-6))
        d_far = torch.from_numpy(far).cuda()
        d_vel = torch.from_numpy(vel).cuda()
        d_acc = torch.empty((n, 4), dtype=torch.float32, device="cuda")
        d_st = torch.empty(((hi - lo) * c2, 3), dtype=torch.float32, device="cuda")
        for rep in range(2):  # twice: the second call starts from the kicked velocities
            v_in = d_vel.cpu().numpy()
            db.kick(lo, hi, d_vel.data_ptr(), d_far.data_ptr(), d_acc.data_ptr(), d_st.data_ptr(),
                    near_scale=float(near_scale), rescale=float(rescale), kick1=float(k1),
                    kick2=float(k2), b2=float(b2))
            got = (d_acc.cpu().numpy(), d_vel.cpu().numpy(), d_st.cpu().numpy())
            wants = [oracle.rescale_and_kick(nacc, far, v_in, counts, near_scale, rescale, k1,
                                             k2, b2=b2)]
            if ref_kick:
                wants.append(oracle.ref_rescale_and_kick(softening, nacc, far, v_in, counts,
                                                         kbox.cpd, *cosmo, k1, k2, b2)[:3])
            for acc_w, v_w, st_w in wants:
                assert np.array_equal(got[0].view(np.uint32), acc_w.view(np.uint32))
                assert np.array_equal(got[1].view(np.uint32), v_w.view(np.uint32))
                assert np.array_equal(got[2][:, 1:], st_w[:, 1:])  # maxima: exact
                np.testing.assert_allclose(got[2][:, 0], st_w[:, 0], rtol=1e-5, atol=0)
        db.close()


@pytest.mark.parametrize("chunks", [1, 2, 3, 5])
def test_pipelined_step_equals_chunked_sweeps(capi, synth, kbox, chunks):
    """nf_box_step (upload + sweep + download overlapped over slab chunks)
    returns, bit for bit, what nf_box_update + nf_box_forces over the same
    chunk ranges return, from fresh positions each call."""
    eps = synth.kernel_eps(1, synth.plummer_eps(41))
    rng = np.random.default_rng(chunks)
    with capi.Context(softening=1, eps=eps, kernel_variant=0) as ctx:
        db = ctx.box(kbox)
        for rep in range(2):
            # positions moved inside their cells (same cell counts)
            h = np.float32(0.5 / kbox.cpd)
            x = np.clip(kbox.x + rng.normal(0, 1e-3 * h, kbox.n).astype(np.float32), -h * 0.999, h * 0.999)
            y, z = kbox.y.copy(), kbox.z.copy()
            x = np.ascontiguousarray(x, dtype=np.float32)
            out = np.full((kbox.n, 4), np.nan, np.float32)
            db.step(x, y, z, out, chunks)
            db.update(x, y, z)
            bnd = [kbox.cpd * k // chunks for k in range(chunks + 1)]
            want = np.concatenate([db.forces(bnd[k], bnd[k + 1]) for k in range(chunks)])
            assert np.array_equal(out.view(np.uint32), want.view(np.uint32)), (chunks, rep)
        with pytest.raises(capi.NfError):
            db.step(x, y, z, out, kbox.cpd)  # chunks of fewer than R slabs
        db.close()


def test_new_entry_points_reject_bad_arguments(capi, synth, kbox):
    import ctypes
    lib = capi.lib()
    eps = synth.kernel_eps(1, synth.plummer_eps(41))
    with capi.Context(softening=1, eps=eps) as ctx:
        db = ctx.box(kbox)
        k = capi.KickParams(1.0, 1.0, 0.0, 0.0, 0.0)
        vel = np.zeros((kbox.n, 3), np.float32)
        assert lib.nf_box_kick(ctx.h, db.h, 0, kbox.cpd, ctypes.byref(k), None, None, None,
                               None) == capi.NF_EINVAL                      # no velocities
        assert lib.nf_box_kick(ctx.h, db.h, 3, 3, ctypes.byref(k), None, vel.ctypes.data, None,
                               None) == capi.NF_EINVAL                      # empty range
        assert lib.nf_box_kick(ctx.h, db.h, 0, kbox.cpd + 1, ctypes.byref(k), None,
                               vel.ctypes.data, None, None) == capi.NF_EINVAL
        assert lib.nf_box_update_aos(ctx.h, db.h, None) == capi.NF_EINVAL
        out = np.zeros((kbox.n, 4), np.float32)
        assert lib.nf_box_step(ctx.h, db.h, None, None, None, out.ctypes.data, 0) == capi.NF_EINVAL
        # still usable afterwards
        a = db.forces(0, 1)
        assert np.all(np.isfinite(a))
        db.close()
