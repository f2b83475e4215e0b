"""Known answers on the GPU path (pair-kernel checks at the softening edges):
two bodies at r = 0, r < eps (the single spline's near branch), r = eps,
r > eps and one cell apart, against the softening formulas evaluated in
double; and the cubic lattice, whose symmetric 5x5x5 neighbourhoods cancel
(the idea of Tests/CheckForces/check_forces.py)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _two_body_box(synth, cpd, p0, p1):
    """Two particles (cell-relative positions p0 in the centre cell, p1 in
    the centre cell shifted by p1's cell offset)."""
    c = (cpd - 1) // 2
    (x0, y0, z0), (x1, y1, z1, dcx) = p0, p1
    cid0 = (c * cpd + c) * cpd + c
    cid1 = ((c + dcx) * cpd + c) * cpd + c
    counts = np.zeros(cpd ** 3, np.int64)
    counts[cid0] += 1
    counts[cid1] += 1
    cs = np.zeros(cpd ** 3 + 1, np.int64)
    np.cumsum(counts, out=cs[1:])
    order = [(cid0, (x0, y0, z0)), (cid1, (x1, y1, z1))]
    order.sort(key=lambda t: t[0])
    xyz = np.array([p for _, p in order], np.float32)
    return synth.Box(cpd, xyz[:, 0].copy(), xyz[:, 1].copy(), xyz[:, 2].copy(), cs), \
        [i for i, (cid, _) in enumerate(order) if cid == cid0][0]


def _f_ref(soft, r2, eps_param):
    """g with a = -g d, raw reference units (double)."""
    if soft == 0:
        return (r2 + eps_param) ** -1.5
    inv_eps2 = eps_param  # single spline: 1/eps_int^2
    u2 = r2 * inv_eps2 + 1e-32
    f = u2 ** -0.5
    return f ** 3 if u2 > 1 else (-15 * f + 6) * u2 + 10


@pytest.mark.parametrize("soft", [0, 1])
@pytest.mark.parametrize("r_over_eps, cells", [(0.0, 0), (0.5, 0), (1.0, 0), (2.0, 0), (9.0, 0),
                                                (None, 1)])
def test_two_body(capi, synth, soft, r_over_eps, cells):
    cpd = 7
    h = 1.0 / cpd
    eps_len = 0.02 * h
    eps_param = synth.kernel_eps(soft, eps_len / (synth.SINGLE_SPLINE_FACTOR if soft == 1 else 1.0))
    eps_int = eps_len
    if cells == 0:
        r = r_over_eps * eps_int
        box, i0 = _two_body_box(synth, cpd, (0.1 * h, -0.05 * h, 0.02 * h),
                                (0.1 * h + r, -0.05 * h, 0.02 * h, 0))
    else:  # adjacent cells along x
        box, i0 = _two_body_box(synth, cpd, (0.3 * h, 0.0, 0.0), (-0.3 * h, 0.01 * h, 0.0, 1))
    with capi.Context(softening=soft, eps=eps_param) as ctx:
        db = ctx.box(box)
        got = db.forces()[:, :3].astype(np.float64)
        db.close()
    # separation from particle i0 to the other one, in double, box frame
    j = 1 - i0
    gp = box.global_positions()
    d = gp[j] - gp[i0]
    r2 = float(d @ d)
    g = _f_ref(soft, r2, float(np.float32(eps_param)))
    want0 = -g * d  # the library's output is in the reference's raw units
    assert np.all(np.isfinite(got))
    if r2 == 0.0:
        assert np.all(got == 0.0)
        return
    np.testing.assert_allclose(got[i0], want0, rtol=2e-6, atol=1e-7 * np.abs(want0).max())
    np.testing.assert_allclose(got[j], -want0, rtol=2e-6, atol=1e-7 * np.abs(want0).max())


def test_lattice_cancels(capi, synth):
    cpd = 9
    n = cpd ** 3
    cs = np.arange(n + 1, dtype=np.int64)
    zero = np.zeros(n, np.float32)
    box = synth.Box(cpd=cpd, x=zero, y=zero.copy(), z=zero.copy(), cell_start=cs)
    for soft in (0, 1):
        eps = synth.kernel_eps(soft, 0.01 / cpd)
        with capi.Context(softening=soft, eps=eps) as ctx:
            db = ctx.box(box)
            a = db.forces()[:, :3]
            db.close()
        one = (1.0 / cpd) ** -2 if soft == 0 else (1.0 / cpd) ** -2 * float(eps) ** -1.5
        assert np.abs(a).max() < 1e-6 * one, (soft, float(np.abs(a).max()), one)


@pytest.mark.parametrize("soft", [0, 1])
def test_cell_faces_and_periodic_corner(capi, oracle, synth, soft):
    """Particles exactly on cell faces (cell-relative -h/2, one ulp inside
    either face, and 0 on each axis: 64 per cell) in the periodic corner
    cell (0,0,0), an interior cell and a cell on the x = cpd-1 face, over a
    random background.  The three face cells are not neighbours of each other,
    so no two particles sit an ulp apart across a face, where any two FP32
    implementations round the cell shift differently; inside a cell the
    separations are exact.  Checked against the reference CPU restatement
    (per component 1e-4 |a|) and the FP64 oracle (RMS 2e-6, max 1e-4)."""
    cpd = 7
    h = 1.0 / cpd
    rng = np.random.default_rng(71)
    n_bg = 3000
    gpos = rng.random((n_bg, 3))
    cell = np.floor(gpos * cpd).astype(np.int64) % cpd
    local = (gpos - (cell + 0.5) * h).astype(np.float32)
    lo = np.float32(-0.5 * h)
    vals = np.array([lo, np.nextafter(lo, np.float32(1)),
                     np.nextafter(np.float32(0.5 * h), np.float32(0)), np.float32(0)], np.float32)
    face = np.array(np.meshgrid(vals, vals, vals, indexing="ij")).reshape(3, -1).T
    cells, locs = [cell], [local]
    for c in [(0, 0, 0), (3, 3, 3), (6, 3, 0)]:
        cells.append(np.tile(np.array(c, np.int64), (len(face), 1)))
        locs.append(face)
    cell = np.concatenate(cells)
    local = np.concatenate(locs)
    cid = (cell[:, 0] * cpd + cell[:, 1]) * cpd + cell[:, 2]
    order = np.argsort(cid, kind="stable")
    cid, local = cid[order], local[order]
    cs = np.zeros(cpd ** 3 + 1, np.int64)
    np.cumsum(np.bincount(cid, minlength=cpd ** 3), out=cs[1:])
    box = synth.Box(cpd=cpd, x=local[:, 0].copy(), y=local[:, 1].copy(), z=local[:, 2].copy(),
                    cell_start=cs)
    eps = synth.kernel_eps(soft, 0.05 * h)
    with capi.Context(softening=soft, eps=eps) as ctx:
        db = ctx.box(box)
        a = db.forces()[:, :3].astype(np.float64)
        db.close()
    assert np.all(np.isfinite(a))
    ref = np.zeros((box.n, 3), np.float32)
    for s in range(cpd):
        oracle.ref32_slab(box, soft, eps, s, acc=ref)
    norm = np.linalg.norm(ref.astype(np.float64), axis=1)
    assert np.all(norm > 0)
    diff = np.abs(a - ref)
    assert np.all(diff <= 1e-4 * norm[:, None]), float((diff / norm[:, None]).max())
    rms, mx, _ = oracle.frac_errors(a, oracle.fp64_sinks(box, soft, eps, np.arange(box.n)))
    assert rms <= 2e-6 and mx <= 1e-4, (rms, mx)
