"""Seeded synthetic periodic boxes in the abacus cell layout.

The reference publishes no benchmark inputs for the near-field path, so these
generators stand in for them.  A box is a periodic unit cube centred on the
origin (first cell spans -0.5 .. -0.5 + 1/cpd, singlestep/DataModel/grid.cpp:
92-96) cut into cpd^3 cells (cpd odd, grid.cpp:50).  Positions are float32
relative to their cell centre, produced the way grid.cpp:174-178
(LocalPosition2Cell) does it: bin in double, subtract the double cell centre,
round to float32.  Particles are sorted by linear cell id
((cx*cpd)+cy)*cpd+cz, which is the reference's PosXYZ order within a slab
(x-slab major, then y, then z; singlestep/DataModel/cellparticles.cpp:218-226).

Two families:

* uniform_box: n uniform random particles.
* clustered_box: a fraction in uniform background, the rest in seeded NFW-like
  clumps (concentration c, truncated at r_t cell widths), clump masses drawn
  log-uniform over [m_lo, m_hi] of the total and rescaled so that the clumps
  hold exactly the requested fraction.
"""
from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass
class Box:
    cpd: int
    x: np.ndarray  # float32[N], cell-relative
    y: np.ndarray
    z: np.ndarray
    cell_start: np.ndarray  # int64[cpd^3 + 1]
    name: str = ""

    @property
    def n(self) -> int:
        return int(self.x.shape[0])

    @property
    def counts(self) -> np.ndarray:
        return np.diff(self.cell_start)

    def slab_range(self, slab: int) -> tuple[int, int]:
        c2 = self.cpd * self.cpd
        return int(self.cell_start[slab * c2]), int(self.cell_start[(slab + 1) * c2])

    def global_positions(self) -> np.ndarray:
        """Box coordinates in double (cell centre + local offset)."""
        cpd = self.cpd
        cid = np.repeat(np.arange(cpd ** 3, dtype=np.int64), self.counts)
        cz = cid % cpd
        cy = (cid // cpd) % cpd
        cx = cid // (cpd * cpd)
        half = (cpd - 1) // 2
        h = 1.0 / cpd
        out = np.empty((self.n, 3), dtype=np.float64)
        out[:, 0] = (cx - half) * h + self.x
        out[:, 1] = (cy - half) * h + self.y
        out[:, 2] = (cz - half) * h + self.z
        return out


def _finish(gpos: np.ndarray, cpd: int, name: str) -> Box:
    """Wrap, bin to cells, convert to cell-relative float32 and sort."""
    gpos = gpos - np.floor(gpos + 0.5)  # wrap into [-0.5, 0.5)
    c = np.floor((gpos + 0.5) * cpd).astype(np.int64)
    np.clip(c, 0, cpd - 1, out=c)
    half = (cpd - 1) // 2
    h = 1.0 / cpd
    local = gpos - (c - half) * h
    lf = local.astype(np.float32)
    hh = np.float32(0.5 * h)
    hi = np.nextafter(hh, np.float32(0.0))
    np.clip(lf, -hh, hi, out=lf)
    cid = (c[:, 0] * cpd + c[:, 1]) * cpd + c[:, 2]
    order = np.argsort(cid, kind="stable")
    counts = np.bincount(cid, minlength=cpd ** 3)
    cell_start = np.zeros(cpd ** 3 + 1, dtype=np.int64)
    np.cumsum(counts, out=cell_start[1:])
    return Box(cpd=cpd,
               x=np.ascontiguousarray(lf[order, 0]),
               y=np.ascontiguousarray(lf[order, 1]),
               z=np.ascontiguousarray(lf[order, 2]),
               cell_start=cell_start, name=name)


def uniform_box(n: int, cpd: int, seed: int = 0) -> Box:
    rng = np.random.default_rng(seed)
    gpos = rng.random((n, 3)) - 0.5
    return _finish(gpos, cpd, f"uniform n={n} cpd={cpd} seed={seed}")


def _nfw_radii(rng, n: int, conc: float, r_trunc: float) -> np.ndarray:
    """Radii with NFW enclosed mass m(x) = ln(1+x) - x/(1+x), x = r/r_s,
    r_s = r_trunc/conc, truncated at x = conc (inverse CDF on a table)."""
    xs = np.concatenate([[0.0], np.geomspace(1e-6, conc, 4096)])
    m = np.log1p(xs) - xs / (1.0 + xs)
    u = rng.random(n) * m[-1]
    x = np.interp(u, m, xs)
    return x * (r_trunc / conc)


def clustered_box(n: int, cpd: int, seed: int = 0, n_clumps: int = 2000,
                  clump_fraction: float = 0.6, m_lo: float = 1e-5, m_hi: float = 1e-3,
                  conc: float = 10.0, r_trunc_cells: float = 0.6) -> Box:
    rng = np.random.default_rng(seed)
    n_clumped = int(round(clump_fraction * n))
    raw = np.exp(rng.uniform(np.log(m_lo), np.log(m_hi), n_clumps)) * n
    m = raw * (n_clumped / raw.sum())
    mi = np.floor(m).astype(np.int64)
    short = n_clumped - int(mi.sum())
    if short > 0:  # hand the rounding remainder to the largest fractional parts
        mi[np.argsort(m - mi)[::-1][:short]] += 1
    centres = rng.random((n_clumps, 3)) - 0.5
    r = _nfw_radii(rng, n_clumped, conc, r_trunc_cells / cpd)
    v = rng.normal(size=(n_clumped, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    gpos = np.empty((n, 3), dtype=np.float64)
    gpos[:n_clumped] = np.repeat(centres, mi, axis=0) + v * r[:, None]
    gpos[n_clumped:] = rng.random((n - n_clumped, 3)) - 0.5
    return _finish(gpos, cpd, f"clustered n={n} cpd={cpd} seed={seed}")


# The workloads, by what they are.
def config_uniform_64(seed: int = 1) -> Box:
    """64^3 uniform particles, cpd 17 (~53 per cell)."""
    return uniform_box(64 ** 3, 17, seed)


def config_clustered_256(seed: int = 2) -> Box:
    """256^3 particles, cpd 65, 40% uniform + 60% in 2000 NFW clumps."""
    return clustered_box(256 ** 3, 65, seed)


def config_clustered_512(seed: int = 3) -> Box:
    """512^3 particles, cpd 125, same clustered mixture."""
    return clustered_box(512 ** 3, 125, seed)


def plummer_eps(n_side: int) -> float:
    """Plummer softening length: 1/40 of the mean interparticle spacing."""
    return (1.0 / n_side) / 40.0


# Ratio of the single-spline internal length to the Plummer-equivalent
# length (singlestep/singlestep.cpp:113-125).
SINGLE_SPLINE_FACTOR = 2.15517


def kernel_eps(softening: int, length_plummer: float) -> float:
    """The reference's float kernel parameter for a softening id
    (singlestep/Timestep/directdriver.cpp:109-117): Plummer eps^2, single
    spline 1/eps_int^2, cubic spline 1/eps_int, cubic Plummer eps_int^3."""
    if softening == 0:
        return float(np.float32(length_plummer * length_plummer))
    if softening == 1:
        e = length_plummer * SINGLE_SPLINE_FACTOR
        return float(np.float32(1.0 / (e * e)))
    if softening == 2:
        e = length_plummer * 1.10064
        return float(np.float32(1.0 / e))
    e = length_plummer
    return float(np.float32(e * e * e))


def clustered_box_device(n: int, cpd: int, seed: int = 0, device="cuda", n_clumps: int = 2000,
                         clump_fraction: float = 0.6, m_lo: float = 1e-5, m_hi: float = 1e-3,
                         conc: float = 10.0, r_trunc_cells: float = 0.6, chunk: int = 1 << 26):
    """The clustered mixture of clustered_box, generated on a GPU with torch
    for boxes too large for host memory (10^9 particles): the same recipe
    (clump masses, NFW radii, uniform background, binning in double, float32
    cell-relative positions sorted by cell), a different random stream.
    Returns (x, y, z) float32 device tensors in cell order and the host
    cell_start (int64[cpd^3 + 1])."""
    import torch
    dev = torch.device(device)
    rng = np.random.default_rng(seed)
    n_clumped = int(round(clump_fraction * n))
    raw = np.exp(rng.uniform(np.log(m_lo), np.log(m_hi), n_clumps)) * n
    m = raw * (n_clumped / raw.sum())
    mi = np.floor(m).astype(np.int64)
    short = n_clumped - int(mi.sum())
    if short > 0:
        mi[np.argsort(m - mi)[::-1][:short]] += 1
    centres = torch.from_numpy(rng.random((n_clumps, 3)) - 0.5).to(dev)
    ends = torch.from_numpy(np.cumsum(mi)).to(dev)
    xs = np.concatenate([[0.0], np.geomspace(1e-6, conc, 4096)])
    mtab = np.log1p(xs) - xs / (1.0 + xs)
    xs_t, m_t = torch.from_numpy(xs).to(dev), torch.from_numpy(mtab).to(dev)
    r_s = (r_trunc_cells / cpd) / conc
    g = torch.Generator(device=dev)
    g.manual_seed(int(seed) * 7919 + 17)
    half = (cpd - 1) // 2
    h = 1.0 / cpd
    hh = np.float32(0.5 * h)
    hi_f = float(np.nextafter(hh, np.float32(0.0)))
    cid = torch.empty(n, dtype=torch.int64, device=dev)
    lf = torch.empty((3, n), dtype=torch.float32, device=dev)
    for p0 in range(0, n, chunk):
        p1 = min(n, p0 + chunk)
        idx = torch.arange(p0, p1, device=dev)
        gpos = torch.rand((p1 - p0, 3), generator=g, device=dev, dtype=torch.float64) - 0.5
        cl = idx < n_clumped
        if bool(cl.any()):
            ic = idx[cl]
            which = torch.searchsorted(ends, ic, right=True)
            u = torch.rand(ic.numel(), generator=g, device=dev, dtype=torch.float64) * m_t[-1]
            k = torch.clamp(torch.searchsorted(m_t, u), 1, m_t.numel() - 1)
            t = (u - m_t[k - 1]) / (m_t[k] - m_t[k - 1])
            r = (xs_t[k - 1] + t * (xs_t[k] - xs_t[k - 1])) * r_s
            v = torch.randn((ic.numel(), 3), generator=g, device=dev, dtype=torch.float64)
            v /= torch.linalg.norm(v, dim=1, keepdim=True)
            gpos[cl] = centres[which] + v * r[:, None]
        gpos -= torch.floor(gpos + 0.5)
        c = torch.clamp(torch.floor((gpos + 0.5) * cpd).to(torch.int64), 0, cpd - 1)
        local = (gpos - (c - half).to(torch.float64) * h).to(torch.float32)
        local.clamp_(-float(hh), hi_f)
        cid[p0:p1] = (c[:, 0] * cpd + c[:, 1]) * cpd + c[:, 2]
        lf[:, p0:p1] = local.T
        del gpos, c, local
    counts = torch.bincount(cid, minlength=cpd ** 3).cpu().numpy()
    _, order = torch.sort(cid, stable=True)
    del cid
    out = []
    for k in range(3):
        out.append(lf[k][order].contiguous())
    del lf, order
    cell_start = np.zeros(cpd ** 3 + 1, dtype=np.int64)
    np.cumsum(counts, out=cell_start[1:])
    return out[0], out[1], out[2], cell_start
