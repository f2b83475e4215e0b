"""ctypes front end of the oracle (TEST INFRASTRUCTURE ONLY).

Loads oracle/liboracle.so (the C restatement in nf_oracle.c) and, when it was
built, oracle/_ref/libnfref_<softening>.so (the reference's own
singlestep/Direct/direct.cpp + DirectCPUKernels.cc compiled unmodified from
its sources, driven by the ExecuteSlabCPU cell loop in ref_shim.cpp).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module; the product library never does.
"""
from __future__ import annotations

import ctypes
import os
import pathlib
from types import SimpleNamespace

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF_DIR = HERE / "_ref"
SOFTENING_NAMES = {0: "plummer", 1: "single_spline", 2: "cubic_spline", 3: "cubic_plummer"}

_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")

_lib = None
_ref = {}


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            raise FileNotFoundError(f"{LIB} is not built (run __graft_entry__.build())")
        L = ctypes.CDLL(str(LIB))
        L.nfo_ref32_slab.argtypes = [ctypes.c_int, ctypes.c_int, _i64p, _f32p, _f32p, _f32p,
                                     ctypes.c_int, ctypes.c_float, ctypes.c_int, _f32p]
        L.nfo_ref32_cells.argtypes = [ctypes.c_int, ctypes.c_int, _i64p, _f32p, _f32p, _f32p,
                                      ctypes.c_int, ctypes.c_float, _i64p, ctypes.c_int64, _f32p]
        L.nfo_fp64_sinks.argtypes = [ctypes.c_int, ctypes.c_int, _i64p, _f32p, _f32p, _f32p,
                                     ctypes.c_int, ctypes.c_double, _i64p, ctypes.c_int64, _f64p]
        L.nfo_frame32_sinks.argtypes = [ctypes.c_int, ctypes.c_int, _i64p, _f32p, _f32p, _f32p,
                                        ctypes.c_int, ctypes.c_float, ctypes.c_int, _i64p,
                                        ctypes.c_int64, _f32p]
        L.nfo_fp64_density.argtypes = [ctypes.c_int, ctypes.c_int, _i64p, _f32p, _f32p, _f32p,
                                       ctypes.c_double, _i64p, ctypes.c_int64, _f64p]
        L.nfo_fp64_density.restype = ctypes.c_int
        L.nfo_cpu_execute.argtypes = [ctypes.c_int, ctypes.c_int, _f32p,
                                      np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS"),
                                      _i32p, ctypes.c_int, _f32p, _i32p, _i32p, _i32p, _f32p,
                                      ctypes.c_int, ctypes.c_float, _f32p]
        L.nfo_cpu_execute.restype = ctypes.c_int
        L.nfo_pair_count.argtypes = [ctypes.c_int, ctypes.c_int, _i64p]
        L.nfo_pair_count.restype = ctypes.c_uint64
        for f in (L.nfo_ref32_slab, L.nfo_ref32_cells, L.nfo_fp64_sinks, L.nfo_frame32_sinks):
            f.restype = ctypes.c_int
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise ValueError(f"oracle call failed with {rc}")


def ref32_slab(box, softening, eps, slab, R=2, acc=None):
    """Reference CPU direct (restated) for every sink of one x-slab.
    Returns float32[N,3] with only the slab's rows written."""
    if acc is None:
        acc = np.zeros((box.n, 3), dtype=np.float32)
    _check(lib().nfo_ref32_slab(box.cpd, R, box.cell_start, box.x, box.y, box.z,
                                softening, eps, slab, acc.reshape(-1)))
    return acc


def ref32_cells(box, softening, eps, cells, R=2, acc=None):
    if acc is None:
        acc = np.zeros((box.n, 3), dtype=np.float32)
    cells = np.ascontiguousarray(cells, dtype=np.int64)
    _check(lib().nfo_ref32_cells(box.cpd, R, box.cell_start, box.x, box.y, box.z,
                                 softening, eps, cells, cells.size, acc.reshape(-1)))
    return acc


def fp64_sinks(box, softening, eps, sinks, R=2):
    sinks = np.ascontiguousarray(sinks, dtype=np.int64)
    out = np.zeros((sinks.size, 3), dtype=np.float64)
    _check(lib().nfo_fp64_sinks(box.cpd, R, box.cell_start, box.x, box.y, box.z, softening,
                                float(np.float32(eps)), sinks, sinks.size, out.reshape(-1)))
    return out


def fp64_density(box, b2, sinks, R=2):
    sinks = np.ascontiguousarray(sinks, dtype=np.int64)
    out = np.zeros(sinks.size, dtype=np.float64)
    _check(lib().nfo_fp64_density(box.cpd, R, box.cell_start, box.x, box.y, box.z,
                                  float(np.float32(b2)), sinks, sinks.size, out))
    return out


def frame32_sinks(box, softening, eps, sinks, compensated=True, R=2):
    sinks = np.ascontiguousarray(sinks, dtype=np.int64)
    out = np.zeros((sinks.size, 3), dtype=np.float32)
    _check(lib().nfo_frame32_sinks(box.cpd, R, box.cell_start, box.x, box.y, box.z, softening,
                                   eps, int(compensated), sinks, sinks.size, out.reshape(-1)))
    return out


def pair_count(box, R=2) -> int:
    return int(lib().nfo_pair_count(box.cpd, R, box.cell_start))


def frac_errors(a, a64):
    """Per-sink fractional force error |a - a64| / |a64| (as in
    Tests/Ewald/run_ewald.py:268) -> (rms, max, per-sink array)."""
    a = np.asarray(a, dtype=np.float64)
    num = np.linalg.norm(a - a64, axis=1)
    den = np.linalg.norm(a64, axis=1)
    ok = den > 0
    e = np.zeros_like(num)
    e[ok] = num[ok] / den[ok]
    return float(np.sqrt(np.mean(e[ok] ** 2))) if ok.any() else 0.0, float(e.max()), e


# ---------------------------------------------------------------------------
# the reference's own kernel, compiled from its sources (oracle/_ref)
# ---------------------------------------------------------------------------

def ref_lib_path(softening: int, flavour: str = "strict") -> pathlib.Path:
    return REF_DIR / f"libnfref_{SOFTENING_NAMES[softening]}_{flavour}.so"


def have_ref(softening: int, flavour: str = "strict") -> bool:
    return ref_lib_path(softening, flavour).exists()


def ref_lib(softening: int, flavour: str = "strict"):
    key = (softening, flavour)
    if key not in _ref:
        L = ctypes.CDLL(str(ref_lib_path(softening, flavour)))
        L.nfref_execute_slab.argtypes = [ctypes.c_int, ctypes.c_int, _i64p, _f32p, _f32p, _f32p,
                                         ctypes.c_float, ctypes.c_int, _f32p, ctypes.c_int]
        L.nfref_execute_slab.restype = ctypes.c_int
        L.nfref_execute_cells.argtypes = [ctypes.c_int, ctypes.c_int, _i64p, _f32p, _f32p, _f32p,
                                          ctypes.c_float, _i64p, ctypes.c_int64, _f32p,
                                          ctypes.c_int]
        L.nfref_execute_cells.restype = ctypes.c_int
        L.nfref_max_threads.restype = ctypes.c_int
        _ref[key] = L
    return _ref[key]


def ref_slab(box, softening, eps, slab, R=2, flavour="strict", threads=0, acc=None):
    """The reference's Direct::Execute over one slab (ExecuteSlabCPU loop)."""
    if acc is None:
        acc = np.zeros((box.n, 3), dtype=np.float32)
    _check(ref_lib(softening, flavour).nfref_execute_slab(
        box.cpd, R, box.cell_start, box.x, box.y, box.z, eps, slab, acc.reshape(-1), threads))
    return acc


def ref_cells(box, softening, eps, cells, R=2, flavour="strict", threads=0, acc=None):
    if acc is None:
        acc = np.zeros((box.n, 3), dtype=np.float32)
    cells = np.ascontiguousarray(cells, dtype=np.int64)
    _check(ref_lib(softening, flavour).nfref_execute_cells(
        box.cpd, R, box.cell_start, box.x, box.y, box.z, eps, cells, cells.size,
        acc.reshape(-1), threads))
    return acc


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:  # pragma: no cover
        return os.cpu_count() or 1


# ---------------------------------------------------------------------------
# the step after the near field (test restatement of the reference's kick)
# ---------------------------------------------------------------------------

def rescale_and_kick(nacc, far, vel, counts, near_scale, rescale, kick1, kick2, b2=0.0):
    """RescaleAndCoAddAcceleration (singlestep/Timestep/kick.cpp:72-107) then
    KickCell (kick.cpp:30-56), in float32 and in the reference's operation
    order, on particles in cell order (counts: particles per cell).

    Returns (acc (N, 4): a and w = nacc.w - b2, the velocities after both half
    kicks, per-cell stats (ncell, 3): mean square velocity after the first
    half kick, max |v| component, max |a| component)."""
    f = np.float32
    nacc = np.asarray(nacc, np.float32)
    a = (nacc[:, :3] * f(near_scale) + np.asarray(far, np.float32)) * f(rescale)
    w = nacc[:, 3] - f(b2) if nacc.shape[1] == 4 else np.zeros(len(nacc), np.float32)
    v1 = np.asarray(vel, np.float32) + a * f(kick1)
    v2 = v1 + a * f(kick2)
    counts = np.asarray(counts, np.int64)
    ncell = counts.size
    stats = np.zeros((ncell, 3), np.float32)
    nz = counts > 0
    starts = np.concatenate([[0], np.cumsum(counts)[:-1]])[nz]
    n2 = (v1[:, 0] * v1[:, 0] + v1[:, 1] * v1[:, 1]) + v1[:, 2] * v1[:, 2]
    # each cell's sum in float32, particle by particle in order (the loop of
    # KickCell without OpenMP SIMD): step k adds every cell's k-th particle
    cnt = counts[nz]
    acc2 = np.zeros(cnt.size, np.float32)
    for k in range(int(cnt.max()) if cnt.size else 0):
        live = cnt > k
        acc2[live] += n2[starts[live] + k]
    stats[nz, 0] = acc2 / cnt.astype(np.float32)
    stats[nz, 1] = np.maximum.reduceat(np.abs(v1).max(axis=1), starts)
    stats[nz, 2] = np.maximum.reduceat(np.abs(a).max(axis=1), starts)
    return np.concatenate([a, w[:, None]], axis=1), v2, stats


def kick_constants(omega_m, omega_smooth, np_total, make_glass, softening_length_internal):
    """The two float factors RescaleAndCoAddAcceleration forms
    (singlestep/Timestep/kick.cpp:75-92), computed in double and rounded to
    float as there: rescale = -3 (Omega_M - Omega_Smooth) / (8 pi np) (negated
    for glass) and the single spline's inv_eps3 = 1 / L^3."""
    import math
    rescale = np.float32(-3.0 * (omega_m - omega_smooth) / (8.0 * math.pi * np_total))
    if make_glass:
        rescale = np.float32(rescale * np.float32(-1))
    L = float(softening_length_internal)
    inv_eps3 = np.float32(1.0 / (L * L * L))
    return rescale, inv_eps3


# ---------------------------------------------------------------------------
# the reference's own kick (oracle/_ref/libnfref_kick_*.so: kick.cpp compiled
# unmodified by the Makefile with its FLOAT3p1 / ThreeVector types)
# ---------------------------------------------------------------------------

def have_ref_kick(softening: int) -> bool:
    return softening in _GPU_SOFT and (REF_DIR / f"libnfref_kick_{_GPU_SOFT[softening]}.so").exists()


_kick_libs = {}


def ref_kick_lib(softening: int):
    if softening not in _kick_libs:
        L = ctypes.CDLL(str(REF_DIR / f"libnfref_kick_{_GPU_SOFT[softening]}.so"))
        L.nfrefkick_rescale.argtypes = [ctypes.c_int64, _f32p, _f32p, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_int64, ctypes.c_int,
                                        ctypes.c_double, ctypes.c_float]
        L.nfrefkick_rescale.restype = ctypes.c_int
        L.nfrefkick_kick_slab.argtypes = [ctypes.c_int, _i64p, _f32p, _f32p, ctypes.c_float,
                                          ctypes.c_float, _f32p, ctypes.c_void_p]
        L.nfrefkick_kick_slab.restype = ctypes.c_int
        L.nfrefkick_acc_floats.restype = ctypes.c_int
        _kick_libs[softening] = L
    return _kick_libs[softening]


def ref_rescale_and_kick(softening, nacc, far, vel, counts, cpd, omega_m, omega_smooth, np_total,
                         make_glass, softening_length_internal, kick1, kick2, b2=0.0):
    """The reference's RescaleAndCoAddAcceleration then KickSlab (kick.cpp),
    slab by slab, on particles in cell order; counts: particles per cell of
    whole slabs (a multiple of cpd^2 cells).  Same returns as
    rescale_and_kick: (acc (N, 4), velocities after both half kicks, per-cell
    stats (ncell, 3)) plus the aux density each particle was given."""
    L = ref_kick_lib(softening)
    assert L.nfrefkick_acc_floats() == 4
    nacc = np.asarray(nacc, np.float32)
    n = len(nacc)
    acc = np.zeros((n, 4), np.float32)
    acc[:, :nacc.shape[1]] = nacc
    far = np.ascontiguousarray(far, np.float32)
    v = np.array(vel, np.float32, copy=True)
    counts = np.asarray(counts, np.int64)
    c2 = cpd * cpd
    assert counts.size % c2 == 0 and counts.sum() == n
    stats = np.zeros((counts.size, 3), np.float32)
    dens = np.zeros(n, np.float32)
    p = 0
    for s in range(counts.size // c2):
        cnt = counts[s * c2:(s + 1) * c2]
        m = int(cnt.sum())
        a_s = np.ascontiguousarray(acc[p:p + m])
        f_s = np.ascontiguousarray(far[p:p + m])
        _check(L.nfrefkick_rescale(m, a_s.reshape(-1), f_s.reshape(-1), omega_m, omega_smooth,
                                   int(np_total), int(make_glass),
                                   float(softening_length_internal), b2))
        v_s = np.ascontiguousarray(v[p:p + m])
        st = np.zeros((c2, 3), np.float32)
        d_s = np.zeros(m, np.float32)
        cs = np.concatenate([[0], np.cumsum(cnt)]).astype(np.int64)
        _check(L.nfrefkick_kick_slab(cpd, cs, v_s.reshape(-1), a_s.reshape(-1), kick1, kick2,
                                     st.reshape(-1), d_s.ctypes.data_as(ctypes.c_void_p)))
        acc[p:p + m], v[p:p + m], dens[p:p + m] = a_s, v_s, d_s
        stats[s * c2:(s + 1) * c2] = st
        p += m
    return acc, v, stats, dens


# ---------------------------------------------------------------------------
# the reference's own GPU pencil kernel (oracle/_ref/libnfref_gpu_*.so,
# compiled from singlestep/Direct/PencilKernel.cu by the Makefile), driven on
# the reference's SIC layout (PencilOnPencil.cc:254-416, PencilPlan.cc:22-90,
# 214-255) for one whole x-slab; a checker for the GPU tests
# ---------------------------------------------------------------------------

_GPU_SOFT = {0: "plummer", 1: "single_spline"}


def have_ref_gpu(softening: int) -> bool:
    return softening in _GPU_SOFT and (REF_DIR / f"libnfref_gpu_{_GPU_SOFT[softening]}.so").exists()


_ref_gpu_libs = {}


def ref_gpu_lib(softening: int):
    if softening not in _ref_gpu_libs:
        L = ctypes.CDLL(str(REF_DIR / f"libnfref_gpu_{_GPU_SOFT[softening]}.so"))
        p = ctypes.c_void_p
        i = ctypes.c_int
        f = ctypes.c_float
        L.nfrefgpu_run.argtypes = [i, i, p, p, p, i, p, i, p, p, i, p, p, f, f, i, p, p]
        L.nfrefgpu_run.restype = i
        L.nfrefgpu_accstruct_floats.restype = i
        _ref_gpu_libs[softening] = L
    return _ref_gpu_libs[softening]


def _fill(box, cid, shift_col, sx, sy, sz, starts, shift, keep=None):
    """Copy the particles of cells cid[p, c] into slots starts[p] + running
    offset, adding shift[c] to the coordinate shift_col (0: x, 2: z); cells
    with keep[p, c] False contribute nothing."""
    cs = box.cell_start
    n = (cs[cid + 1] - cs[cid]).astype(np.int64)
    if keep is not None:
        n = np.where(keep, n, 0)
    P, W = cid.shape
    off = np.zeros_like(n)
    off[:, 1:] = np.cumsum(n, axis=1)[:, :-1]
    dst0 = (starts[:, None] + off).ravel()
    src0 = cs[cid].ravel()
    nf = n.ravel()
    tot = int(nf.sum())
    pair = np.repeat(np.arange(nf.size), nf)
    within = np.arange(tot) - np.repeat(np.cumsum(nf) - nf, nf)
    src = src0[pair] + within
    dst = dst0[pair] + within
    sh = np.repeat(np.tile(shift, P), nf)
    comp = [box.x, box.y, box.z]
    for k, out in enumerate((sx, sy, sz)):
        v = comp[k][src]
        out[dst] = v + sh if k == shift_col else v
    return src, dst


def sic_arrays(box, slab, R=2, node=None):
    """The arrays of one whole x-slab as one SIC (PencilOnPencil.cc:254-416,
    PencilPlan.cc:22-90, 214-255).  Sink pencil (y=j, z centre k): cells
    (slab, j, k-R..k+R) with z shifted by (c-R) h, padded to 64-slot blocks;
    source pencil (j', k): cells (slab-R..slab+R, j', k) with x shifted by
    (c-R) h; sink pencil (j, k) meets source pencils (j+y-R, k), y = 0..2R,
    with y offset (y-R) h.  s_src / s_dst map each sink's particle index to
    its slot in each of its 2R+1 sink pencils.
    node = (node_z_start, node_z_size): one node of a 2D z-split -- centres
    node_z_start-R .. node_z_start+node_z_size+R-1 (index_to_zcen with its
    pad, PencilOnPencil.cc:37-43) and sink pencils truncated to the node's
    primary cells (PencilPlan.cc:110-116)."""
    f32 = np.float32
    cpd, W = box.cpd, 2 * R + 1
    h = f32(1.0 / cpd)
    shift = np.array([f32(c - R) * h for c in range(W)], dtype=np.float32)
    cs = box.cell_start
    counts = np.diff(cs)
    centres = np.arange(cpd) if node is None else (node[0] + np.arange(-R, node[1] + R)) % cpd
    nk = len(centres)
    j = np.repeat(np.arange(cpd), nk)
    kidx = np.tile(np.arange(nk), cpd)
    k = centres[kidx]
    P = cpd * nk
    cells = np.arange(W)
    sink_z = (k[:, None] + cells[None, :] - R) % cpd
    sink_cid = (slab * cpd + j[:, None]) * cpd + sink_z
    keep = None if node is None else (sink_z - node[0]) % cpd < node[1]
    n_p = np.where(keep, counts[sink_cid], 0).sum(axis=1) if keep is not None \
        else counts[sink_cid].sum(axis=1)
    padded = (n_p + 63) // 64 * 64
    s_start = np.concatenate([[0], np.cumsum(padded)[:-1]]).astype(np.int64)
    nslots = int(padded.sum())
    sx = np.zeros(nslots, f32)
    sy = np.zeros(nslots, f32)
    sz = np.zeros(nslots, f32)
    s_src, s_dst = _fill(box, sink_cid, 2, sx, sy, sz, s_start, shift, keep)
    id_max = (s_start + n_p).astype(np.uint32)
    nblk = padded // 64
    parent = np.repeat(np.arange(P), nblk).astype(np.int32)
    src_cid = (((slab + cells[None, :] - R) % cpd) * cpd + j[:, None]) * cpd + k[:, None]
    n_q = counts[src_cid].sum(axis=1)
    q_start = np.concatenate([[0], np.cumsum(n_q)[:-1]]).astype(np.int64)
    nsrc = int(n_q.sum())
    tx = np.zeros(nsrc, f32)
    ty = np.zeros(nsrc, f32)
    tz = np.zeros(nsrc, f32)
    _fill(box, src_cid, 0, tx, ty, tz, q_start, shift)
    ys = np.arange(W)
    ilist = (((j[:, None] + ys[None, :] - R) % cpd) * nk + kidx[:, None]).astype(np.int32)
    yoff = np.tile(shift, (P, 1)).astype(np.float32)
    # every index a kernel will use, checked on the host
    assert parent.size == nslots // 64
    assert np.all(id_max <= nslots) and np.all(s_start % 64 == 0)
    assert np.all((ilist >= 0) & (ilist < P))
    assert np.all(q_start + n_q <= nsrc)
    assert nslots < 2 ** 31 and nsrc < 2 ** 31
    return SimpleNamespace(P=P, W=W, nblk=nblk, nslots=nslots, nsrc=nsrc, sx=sx, sy=sy, sz=sz,
                           tx=tx, ty=ty, tz=tz, id_max=id_max, parent=parent, q_start=q_start,
                           n_q=n_q, ilist=ilist, yoff=yoff, s_src=s_src, s_dst=s_dst, n_p=n_p)


def _coadd(box, slab, a, acc, nc=3):
    """Each sink's 2R+1 pencil partials summed in float32, in pencil order
    (the first nc components of the records)."""
    p0, p1 = box.slab_range(slab)
    out = np.zeros((p1 - p0, nc), np.float32)
    np.add.at(out, a.s_src - p0, acc[a.s_dst, :nc])
    return out


def cpu_execute_slab(box, eps, slab, R=2, node=None):
    """SetInteractionCollection::CPUExecute (Plummer) on one whole x-slab as
    one SIC: float32[n_slab, 3] in particle order (a 2D node: its primary
    particles only, the rest zero)."""
    a = sic_arrays(box, slab, R, node)
    acc = np.zeros((max(a.nslots, 1), 3), np.float32)
    sink_xyz = np.ascontiguousarray(np.concatenate([a.sx, a.sy, a.sz]))
    src_xyz = np.ascontiguousarray(np.concatenate([a.tx, a.ty, a.tz]))
    _check(lib().nfo_cpu_execute(int(a.nblk.sum()), a.nslots, sink_xyz, a.id_max, a.parent,
                                 a.nsrc, src_xyz, a.q_start.astype(np.int32),
                                 a.n_q.astype(np.int32),
                                 np.ascontiguousarray(a.ilist.ravel()),
                                 np.ascontiguousarray(a.yoff.ravel()), a.W, float(np.float32(eps)),
                                 acc.reshape(-1)))
    return _coadd(box, slab, a, acc)


def ref_gpu_slab(box, softening, eps, slab, repeats=1, b2=0.0, R=2, node=None, with_w=False):
    """The reference GPU kernel on one whole x-slab as one SIC (the arrays of
    sic_arrays; node: one node of a 2D z-split): returns (acc float32[n_slab,
    3] in particle order -- [n_slab, 4] with the density sum w when with_w --,
    mean launch ms, DirectTotal pairs).  The y shift is applied on the
    device; the five pencil partials of each sink are co-added in float32."""
    return ref_gpu_run(box, softening, eps, slab, sic_arrays(box, slab, R, node), repeats=repeats,
                       b2=b2, with_w=with_w)


def ref_gpu_run(box, softening, eps, slab, a, repeats=1, b2=0.0, with_w=False):
    """ref_gpu_slab on arrays already laid out by sic_arrays (so that a caller
    can lay out the next slab while this one runs)."""
    P, nblk, nslots, nsrc = a.P, a.nblk, a.nslots, a.nsrc
    sx, sy, sz, tx, ty, tz = a.sx, a.sy, a.sz, a.tx, a.ty, a.tz
    id_max, parent, q_start, n_q, ilist, yoff = a.id_max, a.parent, a.q_start, a.n_q, a.ilist, a.yoff
    L = ref_gpu_lib(softening)
    nf4 = L.nfrefgpu_accstruct_floats()
    if with_w and nf4 < 4:
        raise ValueError("the reference kernel was built without COMPUTE_FOF_DENSITY")
    acc = np.zeros((max(nslots, 1), nf4), np.float32)
    sink_xyz = np.ascontiguousarray(np.concatenate([sx, sy, sz]))
    src_xyz = np.ascontiguousarray(np.concatenate([tx, ty, tz]))
    q_start32 = q_start.astype(np.int32)
    n_q32 = n_q.astype(np.int32)
    ms = ctypes.c_float(0)
    ptr = lambda v: v.ctypes.data_as(ctypes.c_void_p)
    rc = L.nfrefgpu_run(int(nblk.sum()), nslots, ptr(sink_xyz), ptr(id_max), ptr(parent), nsrc,
                        ptr(src_xyz), P, ptr(q_start32), ptr(n_q32), int(ilist.size),
                        ptr(np.ascontiguousarray(ilist.ravel())),
                        ptr(np.ascontiguousarray(yoff.ravel())), float(np.float32(eps)),
                        float(np.float32(b2)), int(repeats), ptr(acc), ctypes.byref(ms))
    if rc != 0:
        raise RuntimeError(f"reference GPU kernel failed: cudaError {rc}")
    pairs = int((a.n_p[:, None] * n_q[ilist]).sum())
    return _coadd(box, slab, a, acc, 4 if with_w else 3), ms.value, pairs
