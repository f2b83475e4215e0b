"""The oracle, pinned against the reference's own CPU kernel (CPU only)."""
import pathlib

import numpy as np
import pytest

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"
FIXTURES = sorted(p for p in GOLDEN.glob("*.npz") if not p.stem.startswith("kick_"))


class _Box:
    def __init__(self, f):
        self.cpd = int(f["cpd"])
        self.x, self.y, self.z = f["x"], f["y"], f["z"]
        self.cell_start = f["cell_start"]
        self.n = self.x.size

    def slab_range(self, s):
        c2 = self.cpd ** 2
        return int(self.cell_start[s * c2]), int(self.cell_start[(s + 1) * c2])


def load_fixture(path):
    f = np.load(path)
    return _Box(f), int(f["softening"]), float(f["eps"]), list(f["slabs"]), f["rows"], f["acc"]


def test_fixtures_present():
    assert len(FIXTURES) == 12


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: p.stem)
def test_restatement_matches_golden_bitwise(oracle, path):
    """nf_oracle.c reproduces singlestep/Direct/direct.cpp bit for bit."""
    box, soft, eps, slabs, rows, acc = load_fixture(path)
    out = np.zeros((box.n, 3), dtype=np.float32)
    for s in slabs:
        oracle.ref32_slab(box, soft, np.float32(eps), s, acc=out)
    assert np.array_equal(out[rows].view(np.uint32), acc.view(np.uint32))


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: p.stem)
def test_fp64_oracle_agrees_with_reference(oracle, path):
    """The FP64 sum agrees with the reference FP32 result to FP32 accuracy."""
    box, soft, eps, slabs, rows, acc = load_fixture(path)
    a64 = oracle.fp64_sinks(box, soft, eps, rows)
    rms, mx, _ = oracle.frac_errors(acc, a64)
    assert rms < 2e-6 and mx < 1e-4, (rms, mx)


@pytest.mark.skipif(not (pathlib.Path(__file__).resolve().parents[1] / "oracle" / "_ref").exists(),
                    reason="reference build not present")
@pytest.mark.parametrize("soft", [0, 1, 2, 3])
def test_restatement_matches_reference_build(oracle, synth, soft):
    if not oracle.have_ref(soft):
        pytest.skip("reference build not present")
    box = synth.clustered_box(5000, 7, seed=99, n_clumps=5)
    eps = synth.kernel_eps(soft, synth.plummer_eps(17))
    a = oracle.ref32_slab(box, soft, eps, 2)
    b = oracle.ref_slab(box, soft, eps, 2)
    lo, hi = box.slab_range(2)
    assert np.array_equal(a[lo:hi].view(np.uint32), b[lo:hi].view(np.uint32))


def test_two_body_known_answer(oracle, synth):
    """Two particles in one periodic box: a = -d / (r^2 + eps^2)^{3/2}."""
    cpd = 5
    h = 1.0 / cpd
    x = np.array([0.01, -0.02], np.float32)
    y = np.array([0.0, 0.015], np.float32)
    z = np.array([0.0, 0.0], np.float32)
    # both in the centre cell (2,2,2) -> id 62
    cs = np.zeros(cpd ** 3 + 1, np.int64)
    cs[63:] = 2
    box = synth.Box(cpd=cpd, x=x, y=y, z=z, cell_start=cs)
    eps2 = 1e-4
    a = oracle.fp64_sinks(box, 0, eps2, np.array([0, 1]))
    d = np.array([x[1] - x[0], y[1] - y[0], 0.0], np.float64)
    g = (d @ d + np.float64(np.float32(eps2))) ** -1.5
    np.testing.assert_allclose(a[0], -g * d, rtol=1e-12)
    np.testing.assert_allclose(a[1], g * d, rtol=1e-12)
    assert h > 0


def test_lattice_symmetry(oracle, synth):
    """A cubic lattice, one particle per cell at the centre: the 5x5x5 sum
    cancels (the CheckForces idea, Tests/CheckForces/check_forces.py)."""
    cpd = 7
    n = cpd ** 3
    cs = np.arange(n + 1, dtype=np.int64)
    zero = np.zeros(n, np.float32)
    box = synth.Box(cpd=cpd, x=zero, y=zero.copy(), z=zero.copy(), cell_start=cs)
    for soft in (0, 1):
        eps = synth.kernel_eps(soft, 0.01)
        a64 = oracle.fp64_sinks(box, soft, eps, np.arange(0, n, 17))
        assert np.abs(a64).max() < 1e-9
        a32 = oracle.ref32_slab(box, soft, eps, 3)
        lo, hi = box.slab_range(3)
        scale = (1.0 / cpd) ** -2 if soft == 0 else 1.0
        assert np.abs(a32[lo:hi]).max() < 1e-4 * scale


def test_pair_count_formula(oracle, synth):
    box = synth.clustered_box(4000, 9, seed=4, n_clumps=4)
    counts = box.counts.reshape(9, 9, 9)
    tot = 0
    for dx in range(-2, 3):
        for dy in range(-2, 3):
            for dz in range(-2, 3):
                tot += int((counts * np.roll(counts, (-dx, -dy, -dz), axis=(0, 1, 2))).sum())
    assert oracle.pair_count(box) == tot


@pytest.mark.parametrize("kind", ["uniform", "clustered"])
def test_cpu_execute_pins_pencil_layout(oracle, synth, kind):
    """SetInteractionCollection::CPUExecute restated on SIC arrays built in
    the reference's pencil layout (sink z shifts, source x shifts, y offsets,
    64-slot padding, 2R+1 partials co-added in float32) reproduces the
    cell-loop reference direct: per component within 1e-4 |a|, and within the
    reference's own FP32 error of FP64 (RMS 5e-6; its cell shifts are added
    in float, where the cell loop forms them in double)."""
    if kind == "uniform":
        box = synth.uniform_box(20000, 9, seed=81)
    else:
        box = synth.clustered_box(30000, 11, seed=82, n_clumps=20)
    eps = synth.kernel_eps(0, synth.plummer_eps(round(box.n ** (1 / 3))))
    pen = np.zeros((box.n, 3), np.float32)
    ref = np.zeros((box.n, 3), np.float32)
    for s in range(box.cpd):
        p0, p1 = box.slab_range(s)
        pen[p0:p1] = oracle.cpu_execute_slab(box, eps, s)
        oracle.ref32_slab(box, 0, eps, s, acc=ref)
    norm = np.linalg.norm(ref.astype(np.float64), axis=1)
    assert np.all(norm > 0)
    diff = np.abs(pen.astype(np.float64) - ref)
    assert np.all(diff <= 1e-4 * norm[:, None]), float((diff / norm[:, None]).max())
    rms, mx, _ = oracle.frac_errors(pen.astype(np.float64),
                                    oracle.fp64_sinks(box, 0, eps, np.arange(box.n)))
    assert rms <= 5e-6 and mx <= 1e-4, (rms, mx)


def test_cpu_execute_2d_nodes_cover_the_box(oracle, synth):
    """The 2D z-split on the reference's own pencil arithmetic: SICs of the
    nodes of a z-partition (pencils centred over each node's cells and R
    ghost cells each side, sink pencils truncated to its primary cells)
    give every particle exactly once, and the same accelerations as one
    z-domain up to the float32 order of the pencil co-add."""
    box = synth.clustered_box(30000, 13, seed=83, n_clumps=20)
    eps = synth.kernel_eps(0, synth.plummer_eps(31))
    cpd = box.cpd
    cellz = np.repeat(np.arange(cpd ** 3) % cpd, np.diff(box.cell_start))
    one = np.zeros((box.n, 3), np.float32)
    two = np.zeros((box.n, 3), np.float32)
    cover = np.zeros(box.n, int)
    for s in range(cpd):
        p0, p1 = box.slab_range(s)
        one[p0:p1] = oracle.cpu_execute_slab(box, eps, s)
        for zs, zn in [(11, 5), (3, 4), (7, 4)]:
            r = oracle.cpu_execute_slab(box, eps, s, node=(zs, zn))
            prim = (cellz[p0:p1] - zs) % cpd < zn
            assert np.all(r[~prim] == 0)
            two[p0:p1][prim] = r[prim]
            cover[p0:p1][prim] += 1
    assert np.all(cover == 1)
    norm = np.linalg.norm(one.astype(np.float64), axis=1)
    assert np.all(np.abs(two.astype(np.float64) - one) <= 1e-5 * norm[:, None])


@pytest.mark.parametrize("name", ["kick_plummer", "kick_single_spline"])
def test_kick_restatement_matches_reference_golden(oracle, name):
    """oracle.rescale_and_kick against the golden output of the reference's
    own kick.cpp (RescaleAndCoAddAcceleration + KickSlab/KickCell, compiled
    unmodified): accelerations, w, velocities and the three cell statistics
    bit for bit."""
    g = np.load(GOLDEN / f"{name}.npz")
    soft = int(g["softening"])
    rescale, inv_eps3 = oracle.kick_constants(float(g["omega_m"]), float(g["omega_smooth"]),
                                              int(g["np_total"]), int(g["make_glass"]),
                                              float(g["softening_length_internal"]))
    near_scale = inv_eps3 if soft == 1 else np.float32(1.0)
    acc, v, st = oracle.rescale_and_kick(g["nacc"], g["far"], g["vel"], g["counts"], near_scale,
                                         rescale, np.float32(g["kick1"]), np.float32(g["kick2"]),
                                         b2=np.float32(g["b2"]))
    assert np.array_equal(acc.view(np.uint32), g["acc_out"].view(np.uint32))
    assert np.array_equal(v.view(np.uint32), g["vel_out"].view(np.uint32))
    assert np.array_equal(st.view(np.uint32), g["stats_out"].view(np.uint32))
    assert np.array_equal(g["dens_out"], g["acc_out"][:, 3])  # set_density(acc.w)


@pytest.mark.parametrize("soft", [0, 1])
def test_kick_restatement_matches_compiled_reference(oracle, soft):
    if not oracle.have_ref_kick(soft):
        pytest.skip("reference kick not built (needs the reference sources)")
    rng = np.random.default_rng(40 + soft)
    cpd = 7
    counts = rng.integers(0, 30, size=3 * cpd * cpd)
    n = int(counts.sum())
    nacc = rng.standard_normal((n, 4)).astype(np.float32) * np.float32(1e3)
    far = (rng.standard_normal((n, 3)) * 1e2).astype(np.float32)
    vel = (rng.standard_normal((n, 3)) * 1e-1).astype(np.float32)
    sli = 3e-4
    args = (0.27, 0.01, 512 ** 3, 1, sli)  # with the glass sign flip
    rescale, inv_eps3 = oracle.kick_constants(*args)
    ref = oracle.ref_rescale_and_kick(soft, nacc, far, vel, counts, cpd, *args,
                                      np.float32(0.02), np.float32(0.03), np.float32(1e-3))
    got = oracle.rescale_and_kick(nacc, far, vel, counts,
                                  inv_eps3 if soft == 1 else np.float32(1.0), rescale,
                                  np.float32(0.02), np.float32(0.03), b2=np.float32(1e-3))
    for a, b in zip(got, ref[:3]):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
