"""One box over several GPUs: contiguous x-slab ranges plus a position halo.

The near-field force of a sink depends only on the particles of the 2R+1
slabs around its own, so a box splits into contiguous x-slab ranges with no
data-path collective.  Each rank owns the particles of its range and, per
step, receives the R boundary slabs of each neighbour (periodic in x): its
"window" of owned + halo slabs.  A window is uploaded as an ordinary
resident box whose cells outside the window are empty (nf_box_create with
the full cell_start), and the rank computes its own slabs only
(nf_box_forces(lo, hi)); those pencils read nothing outside the window, so
the result equals the whole box's for the same slabs.

This is the multi-GPU layout of the reference's slab pipeline
(singlestep/Timestep/pipeline.cpp: slabs of a step are processed in x
order; the GPU near field of slab x reads PosXYZ slabs x-R .. x+R,
singlestep/Direct/PencilPlan.cc:95-138), with device-resident slabs: the
halo crosses NVLink once per step as plain NCCL point-to-point messages
(gloo on CPU), every rank posting the same operations in the same order.
"""
from __future__ import annotations

import dataclasses

import numpy as np


def partition(cpd: int, world: int, weights=None, min_slabs: int = 1) -> list[tuple[int, int]]:
    """Contiguous x-slab ranges [lo, hi).  Without weights: sizes differing
    by at most one.  With per-slab weights (e.g. pair counts of a clustered
    box): cuts placed so that each range's weight is close to 1/world of the
    total, every range keeping at least min_slabs slabs."""
    if world < 1 or world * min_slabs > cpd:
        raise ValueError(f"cannot split {cpd} slabs over {world} ranks")
    if weights is None:
        base, extra = divmod(cpd, world)
        out, lo = [], 0
        for r in range(world):
            hi = lo + base + (1 if r < extra else 0)
            out.append((lo, hi))
            lo = hi
        return out
    w = np.asarray(weights, dtype=np.float64)
    cum = np.concatenate([[0.0], np.cumsum(w)])
    cuts = [0]
    for r in range(1, world):
        target = cum[-1] * r / world
        c = int(np.searchsorted(cum, target))
        c = max(c, cuts[-1] + min_slabs)            # room for this range
        c = min(c, cpd - (world - r) * min_slabs)   # and for the ones after it
        cuts.append(c)
    cuts.append(cpd)
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


def slab_pairs(box, R: int = 2) -> np.ndarray:
    """Pair count of every x-slab as sinks (sum over its cells of count times
    the 5x5x5 neighbourhood count), for a balanced partition."""
    cpd = box.cpd
    c = box.counts.reshape(cpd, cpd, cpd).astype(np.float64)
    nb = np.zeros_like(c)
    for dx in range(-R, R + 1):
        for dy in range(-R, R + 1):
            for dz in range(-R, R + 1):
                nb += np.roll(c, (dx, dy, dz), axis=(0, 1, 2))
    return (c * nb).sum(axis=(1, 2))


def window_slabs(lo: int, hi: int, cpd: int, R: int = 2) -> list[int]:
    """Global ids of the slabs a rank owning [lo, hi) needs: owned plus R on
    each side (periodic), each once, in increasing id order (the order of
    the slabs in a box's cell-ordered particle arrays)."""
    if hi - lo + 2 * R >= cpd:
        return list(range(cpd))
    return sorted({(s + cpd) % cpd for s in range(lo - R, hi + R)})


@dataclasses.dataclass
class SlabData:
    """The particles of one x-slab: per-cell counts (cpd^2, cell order within
    the slab) and cell-relative float32 positions in cell order."""
    counts: np.ndarray
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray


def extract(box, slabs) -> dict[int, SlabData]:
    """The given slabs of a box (what a rank owns)."""
    c2 = box.cpd * box.cpd
    cnt = box.counts
    out = {}
    for s in slabs:
        p0, p1 = box.slab_range(s)
        out[s] = SlabData(cnt[s * c2:(s + 1) * c2].astype(np.int64), box.x[p0:p1], box.y[p0:p1],
                          box.z[p0:p1])
    return out


def window_box(cpd: int, slabs: dict[int, SlabData], name: str = "window"):
    """A box holding only the given slabs (all other cells empty)."""
    from . import synth
    c2 = cpd * cpd
    counts = np.zeros(cpd ** 3, dtype=np.int64)
    xs, ys, zs = [], [], []
    for s in sorted(slabs):
        d = slabs[s]
        counts[s * c2:(s + 1) * c2] = d.counts
        xs.append(d.x)
        ys.append(d.y)
        zs.append(d.z)
    cs = np.zeros(cpd ** 3 + 1, dtype=np.int64)
    np.cumsum(counts, out=cs[1:])
    cat = (lambda a: np.ascontiguousarray(np.concatenate(a), dtype=np.float32)
           if a else np.zeros(0, np.float32))
    return synth.Box(cpd, cat(xs), cat(ys), cat(zs), cs, name)


def halo_plan(rank: int, world: int, cpd: int, R: int = 2, parts=None):
    """(lo, hi, left, right, left_halo, right_halo): this rank's range, its
    neighbours, and the slabs it receives from each (the left neighbour's
    last R slabs, the right neighbour's first R slabs)."""
    parts = partition(cpd, world) if parts is None else parts
    lo, hi = parts[rank]
    if world > 1 and min(h - l for l, h in parts) < R:
        raise ValueError(f"every rank must own at least R={R} slabs")
    left, right = (rank - 1) % world, (rank + 1) % world
    left_halo = [(s + cpd) % cpd for s in range(lo - R, lo)]
    right_halo = [s % cpd for s in range(hi, hi + R)]
    return lo, hi, left, right, left_halo, right_halo


def _pack(slabs: dict[int, SlabData], ids) -> tuple[np.ndarray, np.ndarray]:
    cnt = np.concatenate([slabs[s].counts for s in ids])
    xyz = np.concatenate([np.stack([slabs[s].x, slabs[s].y, slabs[s].z]) for s in ids], axis=1)
    return cnt, np.ascontiguousarray(xyz, dtype=np.float32)


def _unpack(ids, cnt: np.ndarray, xyz: np.ndarray, cpd: int) -> dict[int, SlabData]:
    c2 = cpd * cpd
    out, p = {}, 0
    for k, s in enumerate(ids):
        c = cnt[k * c2:(k + 1) * c2].astype(np.int64)
        n = int(c.sum())
        out[s] = SlabData(c, xyz[0, p:p + n].copy(), xyz[1, p:p + n].copy(), xyz[2, p:p + n].copy())
        p += n
    return out


def exchange_device(owned: dict, rank: int, world: int, cpd: int, R: int = 2, parts=None) -> dict:
    """The halo exchange on device-resident slabs: owned maps slab ->
    (counts as a numpy array, positions as a (3, n) float32 torch tensor on
    this rank's GPU); returns the received halo slabs in the same form.
    Message order as in exchange()."""
    if world == 1:
        return {}
    import torch
    import torch.distributed as dist
    lo, hi, left, right, lh, rh = halo_plan(rank, world, cpd, R, parts)
    dev = next(iter(owned.values()))[1].device
    cnt = lambda ids: torch.from_numpy(np.concatenate([owned[s][0] for s in ids])).to(dev)
    pos = lambda ids: torch.cat([owned[s][1] for s in ids], dim=1).contiguous()
    to_right, to_left = list(range(hi - R, hi)), list(range(lo, lo + R))
    n = R * cpd * cpd
    recv_cl = torch.empty(n, dtype=torch.int64, device=dev)
    recv_cr = torch.empty(n, dtype=torch.int64, device=dev)
    ops = [dist.P2POp(dist.isend, cnt(to_right), right), dist.P2POp(dist.isend, cnt(to_left), left),
           dist.P2POp(dist.irecv, recv_cl, left), dist.P2POp(dist.irecv, recv_cr, right)]
    for q in dist.batch_isend_irecv(ops):
        q.wait()
    cl, cr = recv_cl.cpu().numpy(), recv_cr.cpu().numpy()
    recv_xl = torch.empty((3, int(cl.sum())), dtype=torch.float32, device=dev)
    recv_xr = torch.empty((3, int(cr.sum())), dtype=torch.float32, device=dev)
    ops = [dist.P2POp(dist.isend, pos(to_right), right), dist.P2POp(dist.isend, pos(to_left), left),
           dist.P2POp(dist.irecv, recv_xl, left), dist.P2POp(dist.irecv, recv_xr, right)]
    for q in dist.batch_isend_irecv(ops):
        q.wait()
    out, c2 = {}, cpd * cpd
    for ids, c, x in ((lh, cl, recv_xl), (rh, cr, recv_xr)):
        p = 0
        for k, s in enumerate(ids):
            ck = c[k * c2:(k + 1) * c2]
            m = int(ck.sum())
            out[s] = (ck, x[:, p:p + m])
            p += m
    return out


def exchange(owned: dict[int, SlabData], rank: int, world: int, cpd: int, R: int = 2,
             device: str = "cpu") -> dict[int, SlabData]:
    """Halo exchange over torch.distributed point-to-point messages.

    Every rank posts, in this order: send its last R slabs to the right
    neighbour, send its first R slabs to the left neighbour, receive from the
    left (its last R slabs), receive from the right (its first R slabs) --
    first the per-cell counts (fixed size), then the positions.  With two
    ranks both neighbours are the same peer and the per-pair message order
    keeps the two directions apart.  Returns the received halo slabs."""
    if world == 1:
        return {}
    import torch
    import torch.distributed as dist
    lo, hi, left, right, lh, rh = halo_plan(rank, world, cpd, R)
    to_right = list(range(hi - R, hi))
    to_left = list(range(lo, lo + R))
    c_r, x_r = _pack(owned, to_right)
    c_l, x_l = _pack(owned, to_left)
    n = R * cpd * cpd
    t = lambda a: torch.from_numpy(a).to(device)
    recv_cl = torch.empty(n, dtype=torch.int64, device=device)
    recv_cr = torch.empty(n, dtype=torch.int64, device=device)
    ops = [dist.P2POp(dist.isend, t(c_r), right), dist.P2POp(dist.isend, t(c_l), left),
           dist.P2POp(dist.irecv, recv_cl, left), dist.P2POp(dist.irecv, recv_cr, right)]
    for q in dist.batch_isend_irecv(ops):
        q.wait()
    nl, nr = int(recv_cl.sum()), int(recv_cr.sum())
    recv_xl = torch.empty((3, nl), dtype=torch.float32, device=device)
    recv_xr = torch.empty((3, nr), dtype=torch.float32, device=device)
    ops = [dist.P2POp(dist.isend, t(x_r), right), dist.P2POp(dist.isend, t(x_l), left),
           dist.P2POp(dist.irecv, recv_xl, left), dist.P2POp(dist.irecv, recv_xr, right)]
    for q in dist.batch_isend_irecv(ops):
        q.wait()
    out = _unpack(lh, recv_cl.cpu().numpy(), recv_xl.cpu().numpy(), cpd)
    out.update(_unpack(rh, recv_cr.cpu().numpy(), recv_xr.cpu().numpy(), cpd))
    return out
