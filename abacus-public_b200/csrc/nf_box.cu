// nf_box.cu -- batched near-field form: positions resident in HBM, one
// persistent launch per slab range, deterministic co-add.
//
// Work decomposition (the reference's pencil-on-pencil scheme,
// singlestep/Direct/SetInteractionCollection.hh:4-35 and
// PencilOnPencil.cc:390-416, re-blocked for device-resident data):
//   a sink pencil is the z-run of 2R+1 cells (x, y, zc-R .. zc+R); it meets
//   the (2R+1)^2 source cells (x+dx, y+dy, zc).  Each sink cell lies in 2R+1
//   pencils, so every (sink cell, source cell) pair of the 5x5x5
//   neighbourhood is visited exactly once.  Coordinates are taken in the
//   pencil-centre frame: the sink's z is shifted by (a-R)h, the source's x
//   and y by (dx h, dy h) when staged (the reference shifts x on the host,
//   PencilPlan.cc:226-239, and y on the device, PencilKernel.cu:140).
//
// One warp runs one tile: up to 32*S sinks of one pencil (S sinks per lane,
// kept in registers) against the pencil's source stream -- the 25 source
// cells concatenated, staged 64 at a time into the warp's shared-memory slot
// from float4 HBM records (register prefetch of the next chunk overlaps the
// current chunk's math), each source read by every lane with broadcast
// loads.  A lane evaluates its sinks two at a time with sm_100's paired FP32
// instructions (f32x2).  Every 128 sources the FP32 partial is folded into
// a compensated (hi, lo) pair.  A tile writes that pair per sink and
// component into the sink's pencil slot; the co-add kernel sums the 2R+1
// slots in a fixed order, in compensated FP32.
//
// Resident boxes are stored with the particles of each cell in Morton order
// of their cell-relative position (the co-add writes results back in the
// caller's order): consecutive sinks of a tile then cover a compact region,
// and for the single spline only the sources within eps of the tile's sink
// bounding box need the near branch (decided per 32 sources by a warp vote).
//
// Scheduling: the host builds a work list per slab range, ordered longest
// first (LPT).  Tiles whose cost exceeds a share of the launch are split
// over the W warps of a CTA along the source stream ("heavy groups", taken
// by whole CTAs first); the CTA sums its warps' partials in warp order.  The
// rest are taken one warp at a time from an atomic counter.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

#include <cub/device/device_radix_sort.cuh>

#include "nf_internal.h"
#include "nf_pair.cuh"

namespace nf {

constexpr unsigned FULL = 0xffffffffu;
constexpr int MAXW = 5;     // 2R+1 with R <= 2
constexpr int MAXSRC = 25;  // (2R+1)^2
constexpr int TILE_MAX = 128;
constexpr int WARPS_PER_CTA = 8;

struct KParams {
    const float4 *__restrict__ pos;
    const int64_t *__restrict__ cs;
    int cpd, R;
    const Item *heavy;
    int n_heavy_groups;
    const Item *light;
    int n_light;
    int *counters;    // [0] heavy groups, [1] light items
    Partial *part;    // [(2R+1) * nc][n_range] compensated (hi, lo) pairs
    int64_t p0, n_range;
    int nc;           // 3, or 4 with the density channel
    int plain;        // NF_ACC_PLAIN
    PairConst pc;
    float zshift[MAXW];   // (a-R) h, sink cell a of the pencil
    float xyshift[MAXW];  // n h, n = -R .. R
    signed char odx[MAXSRC], ody[MAXSRC];  // source cell order: outer ring first
    int n_outer;                           // cells with max(|dx|,|dy|) == 2
    // single spline: a source can be closer than eps to one of a tile's
    // sinks only if it lies within near_w (eps plus a rounding allowance) of
    // the tile's sink bounding box
    float near_w;
};

constexpr int CHUNK = 64;  // sources staged per chunk (two per lane)

// Staged sources are stored negated and duplicated: (-x, -x, -y, -y) and
// (-z, -z).  A lane then forms sink - source for two of its sinks with one
// paired add, and every lane reads a source with two broadcast loads.
struct WarpSmem {
    float4 bxy[CHUNK];
    float2 bz[CHUNK];
    int64_t cstart[MAXSRC];
    int32_t cpre[MAXSRC + 1];
    float csx[MAXSRC], csy[MAXSRC];
    float4 tbb;  // the tile's sink x and y range widened by near_w (single spline)
    int64_t sstart[MAXW];
    int32_t spre[MAXW + 1];
};

__device__ __forceinline__ int wrapc(int i, int cpd) {
    return i < 0 ? i + cpd : (i >= cpd ? i - cpd : i);
}

__device__ __forceinline__ int warp_incl_scan(int v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(FULL, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Source and sink tables of one pencil, built by the warp's lanes.
__device__ void setup_tables(const KParams &kp, const Item &it, WarpSmem &ws, int lane) {
    const int cpd = kp.cpd, R = kp.R, W = 2 * R + 1, nsrc = W * W;
    int pc = it.pencil;
    int cz = pc % cpd, cy = (pc / cpd) % cpd, cx = pc / (cpd * cpd);
    int cnt = 0;
    if (lane < nsrc) {
        int dx = kp.odx[lane], dy = kp.ody[lane];
        int64_t c = ((int64_t)wrapc(cx + dx, cpd) * cpd + wrapc(cy + dy, cpd)) * cpd + cz;
        int64_t st = kp.cs[c];
        cnt = (int)(kp.cs[c + 1] - st);
        ws.cstart[lane] = st;
        ws.csx[lane] = kp.xyshift[dx + R];
        ws.csy[lane] = kp.xyshift[dy + R];
    }
    int incl = warp_incl_scan(cnt, lane);
    if (lane < nsrc) ws.cpre[lane + 1] = incl;
    if (lane == 0) ws.cpre[0] = 0;
    int scnt = 0;
    if (lane < W) {
        int64_t c = ((int64_t)cx * cpd + cy) * cpd + wrapc(cz + lane - R, cpd);
        int64_t st = kp.cs[c];
        scnt = (int)(kp.cs[c + 1] - st);
        ws.sstart[lane] = st;
    }
    int sincl = warp_incl_scan(scnt, lane);
    if (lane < W) ws.spre[lane + 1] = sincl;
    if (lane == 0) ws.spre[0] = 0;
    __syncwarp();
}

// Source record for stream index i (null record far away past the end), in
// the pencil frame.  FLAG: w = 1 if the source may lie within eps of a sink
// of the tile (single spline), else 0: it must lie inside the tile's sink
// bounding box widened by eps (x, y from ws.tbb; z in [zlo, zhi]; source
// cells share the pencil's z cell, so z needs no shift).
template <bool FLAG>
__device__ __forceinline__ float4 load_src(const KParams &kp, const WarpSmem &ws, int i,
                                           int src_end, int &k, float zlo, float zhi) {
    if (i >= src_end) return make_float4(1e18f, 1e18f, 1e18f, 0.f);
    while (i >= ws.cpre[k + 1]) k++;
    int64_t p = ws.cstart[k] + (i - ws.cpre[k]);
    float4 t = __ldg(&kp.pos[p]);
    t.x += ws.csx[k];
    t.y += ws.csy[k];
    if (FLAG) {
        const float4 bb = ws.tbb;
        t.w = (t.x >= bb.x && t.x <= bb.y && t.y >= bb.z && t.y <= bb.w && t.z >= zlo &&
               t.z <= zhi)
                  ? 1.f
                  : 0.f;
    }
    return t;
}

// One staged chunk (m_pad sources, a multiple of UNR) against the lane's
// sinks, accumulated straight into the running partials.  Separations are
// taken sink - source, so a += g * d.  NEAR selects the both-branch single
// spline evaluation.  Scalar form: one sink per lane.
template <int SOFT, bool DENS, bool NEAR, int UNR>
__device__ __forceinline__ void chunk_scalar(const float4 *bxy, const float2 *bz, int m_pad,
                                             float sx, float sy, float sz, float &px, float &py,
                                             float &pz, float &pw, const PairConst &pc) {
#pragma unroll 1
    for (int j = 0; j < m_pad; j += UNR) {
#pragma unroll
        for (int u = 0; u < UNR; u++) {
            float4 t = bxy[j + u];
            float tz = bz[j + u].x;
            float dx = sx + t.x, dy = sy + t.z, dz = sz + tz;
            float g;
            if (NEAR) {
                g = spline_g_both(dx, dy, dz, pc);
            } else {
                float r2;
                g = pair_g_fast<SOFT>(dx, dy, dz, pc, r2);
            }
            px = fmaf(g, dx, px);
            py = fmaf(g, dy, py);
            pz = fmaf(g, dz, pz);
            if (DENS) pw += dens_term(dx, dy, dz, pc.b2);
        }
    }
}

// Paired form: SP pairs of sinks per lane, two sinks per FP32 instruction.
template <int SOFT, bool DENS, int SP, bool NEAR, int UNR>
__device__ __forceinline__ void chunk_paired(const float4 *bxy, const float2 *bz, int m_pad,
                                             const float2 (&sx)[SP], const float2 (&sy)[SP],
                                             const float2 (&sz)[SP], float2 (&px)[SP],
                                             float2 (&py)[SP], float2 (&pz)[SP],
                                             float2 (&pw)[SP], const PairConst &pc) {
#pragma unroll 1
    for (int j = 0; j < m_pad; j += UNR) {
#pragma unroll
        for (int u = 0; u < UNR; u++) {
            float4 t = bxy[j + u];
            float2 tz = bz[j + u];
            float2 tx = make_float2(t.x, t.y), ty = make_float2(t.z, t.w);
#pragma unroll
            for (int q = 0; q < SP; q++) {
                float2 dx = add2(sx[q], tx), dy = add2(sy[q], ty), dz = add2(sz[q], tz);
                float2 g;
                if (SOFT == SOFT_PLUMMER || SOFT == SOFT_SINGLE_SPLINE) {
                    float2 r2 = r2_x2(dx, dy, dz, SOFT == SOFT_PLUMMER ? pc.eps : 1e-25f);
                    g = NEAR ? spline_g_both_x2(r2, pc) : inv_r3_x2(r2);
                } else {  // the cubic kernels: component-wise scalar evaluation
                    float r2;
                    g.x = pair_g_fast<SOFT>(dx.x, dy.x, dz.x, pc, r2);
                    g.y = pair_g_fast<SOFT>(dx.y, dy.y, dz.y, pc, r2);
                }
                px[q] = fma2(g, dx, px[q]);
                py[q] = fma2(g, dy, py[q]);
                pz[q] = fma2(g, dz, pz[q]);
                if (DENS) {
                    pw[q].x += dens_term(dx.x, dy.x, dz.x, pc.b2);
                    pw[q].y += dens_term(dx.y, dy.y, dz.y, pc.b2);
                }
            }
        }
    }
}

// Combine area for CTA-split tiles: [warp][component][sink] partials.
struct CombSmem {
    Partial v[WARPS_PER_CTA][4][TILE_MAX];
};

// (s, e) += the partial (hi, lo), compensated FP32: s the running sum, e
// the running correction (the value is s + e).
__device__ __forceinline__ void add_partial(float &s, float &e, Partial p) {
    float t, err;
    two_sum(s, p.x, t, err);
    s = t;
    e = e + (err + p.y);
}

// Particle index and pencil slot of sink i of the tile's pencil.
__device__ __forceinline__ int64_t sink_particle(const WarpSmem &ws, int i, int &a) {
    a = 0;
    while (i >= ws.spre[a + 1]) a++;
    return ws.sstart[a] + (i - ws.spre[a]);
}

// Fold a partial p into the running compensated sum (h, l) and clear it
// (plain: one FP32 running sum).  Kahan's compensated summation with the
// correction kept as the low part to add (the sum is h + l):
//   y = p + l;  t = h + y;  l = y - (t - h);  h = t
// four paired instructions per component and sink pair.  Scalar and paired
// (two sinks) forms; a - b is formed as fma(b, -1, a), which rounds exactly
// like a subtraction.
__device__ __forceinline__ void fold1(float &h, float &l, float &p, bool plain) {
    if (plain) {
        h += p;
    } else {
        float y = p + l;
        float t = h + y;
        l = y - (t - h);
        h = t;
    }
    p = 0.f;
}

__device__ __forceinline__ void fold2(float2 &h, float2 &l, float2 &p, bool plain) {
    if (plain) {
        h = add2(h, p);
    } else {
        const float2 m1 = dup2(-1.0f);
        float2 y = add2(p, l);
        float2 t = add2(h, y);
        l = fma2(fma2(h, m1, t), m1, y);  // y - (t - h)
        h = t;
    }
    p = make_float2(0.f, 0.f);
}

// FP32 partials are folded into the compensated (h, l) sums every FOLD_CHUNKS chunks.
constexpr int FOLD_CHUNKS = 2;

template <int SOFT, bool DENS, int S, int UNR>
__device__ void run_tile(const KParams &kp, WarpSmem &ws, const Item &it, int lane,
                         CombSmem *comb, int wslot) {
    const int NC = DENS ? 4 : 3;
    constexpr int SP = S >= 2 ? S / 2 : 1;  // sink pairs of the paired form
    float sx[S], sy[S], sz[S];
#pragma unroll
    for (int s = 0; s < S; s++) {
        int j = s * 32 + lane;
        sx[s] = sy[s] = sz[s] = -1e18f;  // idle lane: far from every source
        if (j < it.nsink) {
            int a;
            int64_t p = sink_particle(ws, it.sink_begin + j, a);
            float4 q = __ldg(&kp.pos[p]);
            sx[s] = q.x;
            sy[s] = q.y;
            sz[s] = q.z + kp.zshift[a];
        }
    }
    // scalar form (S == 1): partial p*1 and running (h*1, l*1); paired form:
    // sinks 2q, 2q+1 in the two halves of qx/qy/qz, px.., hx.., lx..
    float px1 = 0.f, py1 = 0.f, pz1 = 0.f, pw1 = 0.f;
    float hx1 = 0.f, hy1 = 0.f, hz1 = 0.f, lx1 = 0.f, ly1 = 0.f, lz1 = 0.f;
    float2 qx[SP], qy[SP], qz[SP], px[SP], py[SP], pz[SP], pw[SP];
    float2 hx[SP], hy[SP], hz[SP], lx[SP], ly[SP], lz[SP];
#pragma unroll
    for (int q = 0; q < SP; q++) {
        if (S >= 2) {
            qx[q] = make_float2(sx[2 * q], sx[2 * q + 1]);
            qy[q] = make_float2(sy[2 * q], sy[2 * q + 1]);
            qz[q] = make_float2(sz[2 * q], sz[2 * q + 1]);
        }
        px[q] = py[q] = pz[q] = pw[q] = make_float2(0.f, 0.f);
        hx[q] = hy[q] = hz[q] = lx[q] = ly[q] = lz[q] = make_float2(0.f, 0.f);
    }
    constexpr bool FLAG = SOFT == SOFT_SINGLE_SPLINE;
    const bool plain = kp.plain;
    // the tile's sink bounding box (pencil frame), widened by eps: sources
    // outside it cannot be near any of the tile's sinks
    float zlo = 3.0e38f, zhi = -3.0e38f;
    if (FLAG) {
        float xlo = 3.0e38f, xhi = -3.0e38f, ylo = 3.0e38f, yhi = -3.0e38f;
#pragma unroll
        for (int s = 0; s < S; s++)
            if (s * 32 + lane < it.nsink) {
                xlo = fminf(xlo, sx[s]);
                xhi = fmaxf(xhi, sx[s]);
                ylo = fminf(ylo, sy[s]);
                yhi = fmaxf(yhi, sy[s]);
                zlo = fminf(zlo, sz[s]);
                zhi = fmaxf(zhi, sz[s]);
            }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            xlo = fminf(xlo, __shfl_xor_sync(FULL, xlo, off));
            xhi = fmaxf(xhi, __shfl_xor_sync(FULL, xhi, off));
            ylo = fminf(ylo, __shfl_xor_sync(FULL, ylo, off));
            yhi = fmaxf(yhi, __shfl_xor_sync(FULL, yhi, off));
            zlo = fminf(zlo, __shfl_xor_sync(FULL, zlo, off));
            zhi = fmaxf(zhi, __shfl_xor_sync(FULL, zhi, off));
        }
        const float w = kp.near_w;
        __syncwarp();
        if (lane == 0) ws.tbb = make_float4(xlo - w, xhi + w, ylo - w, yhi + w);
        __syncwarp();
        zlo -= w;
        zhi += w;
    }
    int k0 = 0, k1 = 0;
    int base = it.src_begin;
    // two sources per lane per chunk: stream indices base+lane, base+32+lane
    float4 pre0 = load_src<FLAG>(kp, ws, base + lane, it.src_end, k0, zlo, zhi);
    float4 pre1 = load_src<FLAG>(kp, ws, base + 32 + lane, it.src_end, k1, zlo, zhi);
    for (int chunk = 1; base < it.src_end; base += CHUNK, chunk++) {
        // the chunk takes the both-branch path only if one of its sources
        // may lie within eps of one of the tile's sinks
        const bool near = FLAG && __any_sync(FULL, pre0.w + pre1.w != 0.f);
        __syncwarp();
        ws.bxy[lane] = make_float4(-pre0.x, -pre0.x, -pre0.y, -pre0.y);
        ws.bz[lane] = make_float2(-pre0.z, -pre0.z);
        ws.bxy[lane + 32] = make_float4(-pre1.x, -pre1.x, -pre1.y, -pre1.y);
        ws.bz[lane + 32] = make_float2(-pre1.z, -pre1.z);
        __syncwarp();
        const bool more = base + CHUNK < it.src_end;
        if (more) {
            pre0 = load_src<FLAG>(kp, ws, base + CHUNK + lane, it.src_end, k0, zlo, zhi);
            pre1 = load_src<FLAG>(kp, ws, base + CHUNK + 32 + lane, it.src_end, k1, zlo, zhi);
        }
        const int m = min(CHUNK, it.src_end - base);
        const int mpad = (m + UNR - 1) / UNR * UNR;  // padding reads null records
        if constexpr (S == 1) {
            if (FLAG && near)
                chunk_scalar<SOFT, DENS, true, UNR>(ws.bxy, ws.bz, mpad, sx[0], sy[0], sz[0], px1,
                                                    py1, pz1, pw1, kp.pc);
            else
                chunk_scalar<SOFT, DENS, false, UNR>(ws.bxy, ws.bz, mpad, sx[0], sy[0], sz[0], px1,
                                                     py1, pz1, pw1, kp.pc);
        } else {
            if (FLAG && near)
                chunk_paired<SOFT, DENS, SP, true, UNR>(ws.bxy, ws.bz, mpad, qx, qy, qz, px, py, pz,
                                                        pw, kp.pc);
            else
                chunk_paired<SOFT, DENS, SP, false, UNR>(ws.bxy, ws.bz, mpad, qx, qy, qz, px, py, pz,
                                                         pw, kp.pc);
        }
        if (chunk % FOLD_CHUNKS == 0 || !more) {
            if constexpr (S == 1) {
                fold1(hx1, lx1, px1, plain);
                fold1(hy1, ly1, py1, plain);
                fold1(hz1, lz1, pz1, plain);
            } else {
#pragma unroll
                for (int q = 0; q < SP; q++) {
                    fold2(hx[q], lx[q], px[q], plain);
                    fold2(hy[q], ly[q], py[q], plain);
                    fold2(hz[q], lz[q], pz[q], plain);
                }
            }
        }
    }
#pragma unroll
    for (int s = 0; s < S; s++) {
        int j = s * 32 + lane;
        if (j >= it.nsink) continue;
        // the sink's running sums, kept as (hi, lo) pairs
        Partial vx, vy, vz, vw = make_float2(0.f, 0.f);
        if constexpr (S == 1) {
            vx = make_float2(hx1, lx1);
            vy = make_float2(hy1, ly1);
            vz = make_float2(hz1, lz1);
            if (DENS) vw = make_float2(pw1, 0.f);
        } else {
            const int q = s >> 1;
            const bool odd = s & 1;
            vx = odd ? make_float2(hx[q].y, lx[q].y) : make_float2(hx[q].x, lx[q].x);
            vy = odd ? make_float2(hy[q].y, ly[q].y) : make_float2(hy[q].x, ly[q].x);
            vz = odd ? make_float2(hz[q].y, lz[q].y) : make_float2(hz[q].x, lz[q].x);
            if (DENS) vw = make_float2(odd ? pw[q].y : pw[q].x, 0.f);
        }
        if (comb) {  // split tiles hold at most TILE_MAX sinks (host-built)
            if (j >= TILE_MAX) continue;
            comb->v[wslot][0][j] = vx;
            comb->v[wslot][1][j] = vy;
            comb->v[wslot][2][j] = vz;
            if (DENS) comb->v[wslot][3][j] = vw;
        } else {
            int a;
            int64_t idx = sink_particle(ws, it.sink_begin + j, a) - kp.p0;
            Partial *bp = kp.part + (int64_t)a * NC * kp.n_range + idx;
            bp[0] = vx;
            bp[kp.n_range] = vy;
            bp[2 * kp.n_range] = vz;
            if (DENS) bp[3 * kp.n_range] = vw;
        }
    }
}

template <int SOFT, bool DENS, int SMAX, int UNR>
__device__ __forceinline__ void dispatch_tile(const KParams &kp, WarpSmem &ws, const Item &it,
                                              int lane, CombSmem *comb, int wslot) {
    setup_tables(kp, it, ws, lane);
    if (it.S == 1)
        run_tile<SOFT, DENS, 1, UNR>(kp, ws, it, lane, comb, wslot);
    else if (SMAX == 2 || it.S == 2)
        run_tile<SOFT, DENS, 2, UNR>(kp, ws, it, lane, comb, wslot);
    else if (SMAX == 4 || it.S == 4)
        run_tile<SOFT, DENS, 4, UNR>(kp, ws, it, lane, comb, wslot);
    else
        run_tile<SOFT, DENS, (SMAX >= 8 ? 8 : 4), UNR>(kp, ws, it, lane, comb, wslot);
}

// The persistent pencil kernel.  Shape knobs (chosen by the autotuner):
//   SMAX  largest tile 32*SMAX sinks (S = sinks per lane in {1, 2, SMAX})
//   UNR   sources per unrolled step
//   MINB  CTAs per SM the register allocation must leave room for
template <int SOFT, bool DENS, int SMAX, int UNR, int MINB>
__global__ void __launch_bounds__(WARPS_PER_CTA * 32, MINB) pencil_kernel(KParams kp) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    WarpSmem *wsm = reinterpret_cast<WarpSmem *>(smem_raw);
    CombSmem *comb = reinterpret_cast<CombSmem *>(smem_raw + sizeof(WarpSmem) * WARPS_PER_CTA);
    __shared__ int s_group;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int NC = DENS ? 4 : 3;
    // Phase 1: heavy tiles, split over the CTA's warps along the source stream.
    for (;;) {
        if (threadIdx.x == 0) s_group = atomicAdd(&kp.counters[0], 1);
        __syncthreads();
        int g = s_group;
        __syncthreads();
        if (g >= kp.n_heavy_groups) break;
        Item it = kp.heavy[(int64_t)g * WARPS_PER_CTA + warp];
        dispatch_tile<SOFT, DENS, SMAX, UNR>(kp, wsm[warp], it, lane, comb, warp);
        __syncthreads();
        // warp 0's tables describe the (common) sink tile
        const WarpSmem &w0 = wsm[0];
        for (int j = threadIdx.x; j < it.nsink; j += blockDim.x) {
            int a;
            int64_t idx = sink_particle(w0, it.sink_begin + j, a) - kp.p0;
            Partial *bp = kp.part + (int64_t)a * NC * kp.n_range + idx;
#pragma unroll
            for (int c = 0; c < NC; c++) {
                float cs = 0.f, ce = 0.f;  // the warps' partials, summed in warp order
#pragma unroll
                for (int w = 0; w < WARPS_PER_CTA; w++) add_partial(cs, ce, comb->v[w][c][j]);
                bp[(int64_t)c * kp.n_range] = make_float2(cs, ce);
            }
        }
        __syncthreads();
    }
    // Phase 2: one tile per warp.
    for (;;) {
        int i = 0;
        if (lane == 0) i = atomicAdd(&kp.counters[1], 1);
        i = __shfl_sync(FULL, i, 0);
        if (i >= kp.n_light) break;
        Item it = kp.light[i];
        dispatch_tile<SOFT, DENS, SMAX, UNR>(kp, wsm[warp], it, lane, nullptr, 0);
    }
}

// Sum the 2R+1 pencil partials of every particle in a fixed order, apply the
// output scale (single spline: eps^3) and write accstruct records.
// perm (optional): the caller's particle index of each packed slot; the
// record of slot p0 + p goes to perm[p0 + p] - p0 (a permutation of the
// range, since the in-cell ordering never moves a particle out of its cell).
// The 2R+1 partials of particle p of the range, summed in compensated FP32
// in pencil-slot order; x, y, z times the output scale (one rounding: the
// correction is scaled and added inside the FMA), w unscaled.
__device__ __forceinline__ void coadd_sink(const Partial *__restrict__ part, int64_t n, int W,
                                           int nc, int64_t p, float scale, float r[4]) {
    float s[4] = {0.f, 0.f, 0.f, 0.f}, e[4] = {0.f, 0.f, 0.f, 0.f};
    for (int a = 0; a < W; a++)
#pragma unroll
        for (int c = 0; c < 4; c++)
            if (c < nc) add_partial(s[c], e[c], part[((int64_t)a * nc + c) * n + p]);
#pragma unroll
    for (int c = 0; c < 3; c++) r[c] = fmaf(s[c], scale, e[c] * scale);
    r[3] = nc == 4 ? s[3] + e[3] : 0.f;
}

__global__ void coadd_kernel(const Partial *__restrict__ part, int64_t n, int W, int nc,
                             float scale, int out_kind, void *out,
                             const uint32_t *__restrict__ perm, int64_t p0) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride) {
        float r[4];
        coadd_sink(part, n, W, nc, p, scale, r);
        const float x = r[0], y = r[1], z = r[2];
        const int64_t o_i = perm ? (int64_t)perm[p0 + p] - p0 : p;
        if (out_kind == NF_OUT_FLOAT4) {
            reinterpret_cast<float4 *>(out)[o_i] = make_float4(x, y, z, r[3]);
        } else {
            float *o = reinterpret_cast<float *>(out) + 3 * o_i;
            o[0] = x;
            o[1] = y;
            o[2] = z;
        }
    }
}

__global__ void pack_positions(const float *__restrict__ x, const float *__restrict__ y,
                               const float *__restrict__ z, int64_t n, float4 *out) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride)
        out[p] = make_float4(x[p], y[p], z[p], 0.f);
}

// In-cell ordering of a resident box.  Particles keep their cell but are
// ordered inside it along a Morton curve of their cell-relative position, so
// that a tile of consecutive sinks covers a compact region: the tile's
// bounding box then keeps most sources out of the single spline's
// near-branch evaluation.  Key = cell id (high bits) : 30-bit Morton code.
__device__ __forceinline__ uint32_t spread_bits10(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__device__ __forceinline__ uint32_t cell_coord10(float u, int cpd) {
    float t = fmaf(u, (float)cpd, 0.5f) * 1024.0f;  // cell-relative -> [0, 1024)
    return (uint32_t)fminf(fmaxf(t, 0.0f), 1023.0f);
}

// Component c of particle p is at x/y/z[p * comp_stride] (1: three
// arrays; 3: one array of (x, y, z) records).
__global__ void order_keys(const float *__restrict__ x, const float *__restrict__ y,
                           const float *__restrict__ z, int comp_stride,
                           const int64_t *__restrict__ cs, int64_t ncell, int cpd, int64_t p_begin,
                           int64_t p_end, uint64_t *key, uint32_t *val) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = p_begin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < p_end;
         p += stride) {
        // cell of particle p: the last c with cs[c] <= p
        int64_t lo = 0, hi = ncell;  // cs[lo] <= p < cs[hi]
        while (hi - lo > 1) {
            int64_t mid = (lo + hi) >> 1;
            if (cs[mid] <= p) lo = mid;
            else hi = mid;
        }
        const int64_t q = p * comp_stride;
        uint32_t m = spread_bits10(cell_coord10(x[q], cpd)) << 2 |
                     spread_bits10(cell_coord10(y[q], cpd)) << 1 |
                     spread_bits10(cell_coord10(z[q], cpd));
        key[p] = (uint64_t)lo << 30 | m;
        val[p] = (uint32_t)p;
    }
}

__global__ void pack_ordered(const float *__restrict__ x, const float *__restrict__ y,
                             const float *__restrict__ z, int comp_stride,
                             const uint32_t *__restrict__ perm, int64_t p_begin, int64_t p_end,
                             float4 *out) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = p_begin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < p_end;
         p += stride) {
        int64_t q = (int64_t)perm[p] * comp_stride;
        out[p] = make_float4(x[q], y[q], z[q], 0.f);
    }
}

// The step after the near field, fused with the co-add: the reference's
// RescaleAndCoAddAcceleration (singlestep/Timestep/kick.cpp:72-107)
//   a = (nacc * near_scale + facc) * rescale,  w = nacc.w - b2
// and KickCell (kick.cpp:30-56)
//   v += a kick1; cell stats of v and a; v += a kick2.
// One warp per cell of the range; each particle's near acceleration is
// co-added from its pencil partials exactly as coadd_kernel does (nacc is
// the float record nf_box_forces would return), then the float operations
// above run unfused, in the reference's order.  Cell stats: mean square
// velocity (after the first half kick), max |v| and max |a| component.
struct KickConst {
    float near_scale, rescale, kick1, kick2, b2;
};

__global__ void kick_kernel(const Partial *__restrict__ part, int64_t n, int W, int nc,
                            float scale, const int64_t *__restrict__ cs, int64_t c0,
                            int64_t ncells, int64_t p0, const uint32_t *__restrict__ perm,
                            KickConst k, const float *__restrict__ far, float *vel, void *acc_out,
                            int out_kind, float *stats) {
    const int lane = threadIdx.x & 31;
    const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t c = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < ncells;
         c += nwarps) {
        const int64_t s0 = cs[c0 + c], s1 = cs[c0 + c + 1];
        float sv2 = 0.f, mv = 0.f, ma = 0.f;
        for (int64_t slot = s0 + lane; slot < s1; slot += 32) {
            const int64_t i = slot - p0;
            float r[4];
            coadd_sink(part, n, W, nc, i, scale, r);
            const float nx = r[0], ny = r[1], nz = r[2], nw = r[3];
            const int64_t o = perm ? (int64_t)perm[slot] - p0 : i;
            const float fx = far ? far[3 * o] : 0.f, fy = far ? far[3 * o + 1] : 0.f,
                        fz = far ? far[3 * o + 2] : 0.f;
            const float ax = __fmul_rn(__fadd_rn(__fmul_rn(nx, k.near_scale), fx), k.rescale);
            const float ay = __fmul_rn(__fadd_rn(__fmul_rn(ny, k.near_scale), fy), k.rescale);
            const float az = __fmul_rn(__fadd_rn(__fmul_rn(nz, k.near_scale), fz), k.rescale);
            const float aw = __fsub_rn(nw, k.b2);
            float vx = vel[3 * o], vy = vel[3 * o + 1], vz = vel[3 * o + 2];
            vx = __fadd_rn(vx, __fmul_rn(ax, k.kick1));
            vy = __fadd_rn(vy, __fmul_rn(ay, k.kick1));
            vz = __fadd_rn(vz, __fmul_rn(az, k.kick1));
            sv2 = __fadd_rn(sv2, __fadd_rn(__fadd_rn(__fmul_rn(vx, vx), __fmul_rn(vy, vy)),
                                           __fmul_rn(vz, vz)));
            mv = fmaxf(mv, fmaxf(fabsf(vx), fmaxf(fabsf(vy), fabsf(vz))));
            ma = fmaxf(ma, fmaxf(fabsf(ax), fmaxf(fabsf(ay), fabsf(az))));
            vel[3 * o] = __fadd_rn(vx, __fmul_rn(ax, k.kick2));
            vel[3 * o + 1] = __fadd_rn(vy, __fmul_rn(ay, k.kick2));
            vel[3 * o + 2] = __fadd_rn(vz, __fmul_rn(az, k.kick2));
            if (acc_out) {
                if (out_kind == NF_OUT_FLOAT4) {
                    reinterpret_cast<float4 *>(acc_out)[o] = make_float4(ax, ay, az, aw);
                } else {
                    float *r = reinterpret_cast<float *>(acc_out) + 3 * o;
                    r[0] = ax;
                    r[1] = ay;
                    r[2] = az;
                }
            }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            sv2 += __shfl_xor_sync(FULL, sv2, off);
            mv = fmaxf(mv, __shfl_xor_sync(FULL, mv, off));
            ma = fmaxf(ma, __shfl_xor_sync(FULL, ma, off));
        }
        if (lane == 0 && stats) {
            const int64_t cnt = s1 - s0;
            stats[3 * c] = cnt > 0 ? sv2 / (float)cnt : 0.f;
            stats[3 * c + 1] = mv;
            stats[3 * c + 2] = ma;
        }
    }
}

// ------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------

typedef void (*KernelFn)(KParams);

// Kernel shapes the autotuner chooses among (tunable for the Plummer and
// single-spline kernels without the density channel; the other kernels run
// shape 0).
struct Variant {
    int smax, unr, minb;
    const char *name;
};
static const Variant VARIANTS[] = {
    {4, 8, 2, "sinks/lane<=4 unroll 8, 2 CTAs/SM"},
    {4, 16, 2, "sinks/lane<=4 unroll 16, 2 CTAs/SM"},
    {8, 4, 1, "sinks/lane<=8 unroll 4, 1 CTA/SM"},
    {2, 4, 3, "sinks/lane<=2 unroll 4, 3 CTAs/SM"},
    {2, 2, 4, "sinks/lane<=2 unroll 2, 4 CTAs/SM"},
};
static constexpr int NVARIANTS = sizeof(VARIANTS) / sizeof(VARIANTS[0]);

template <int SOFT, bool DENS>
static KernelFn variant_kernel(int v) {
    switch (v) {
    case 1: return pencil_kernel<SOFT, DENS, 4, 16, 2>;
    case 2: return pencil_kernel<SOFT, DENS, 8, 4, 1>;
    case 3: return pencil_kernel<SOFT, DENS, 2, 4, 3>;
    case 4: return pencil_kernel<SOFT, DENS, 2, 2, 4>;
    default: return pencil_kernel<SOFT, DENS, 4, 8, 2>;
    }
}

static bool tunable(int soft, bool dens) {
    return !dens && (soft == SOFT_PLUMMER || soft == SOFT_SINGLE_SPLINE);
}

static KernelFn pick_kernel(int soft, bool dens, int v) {
    if (!tunable(soft, dens)) v = 0;
    switch (soft) {
    case SOFT_PLUMMER:
        return dens ? pencil_kernel<SOFT_PLUMMER, true, 4, 8, 2> : variant_kernel<SOFT_PLUMMER, false>(v);
    case SOFT_SINGLE_SPLINE:
        return dens ? pencil_kernel<SOFT_SINGLE_SPLINE, true, 4, 8, 2>
                    : variant_kernel<SOFT_SINGLE_SPLINE, false>(v);
    case SOFT_CUBIC_SPLINE:
        return dens ? pencil_kernel<SOFT_CUBIC_SPLINE, true, 4, 8, 2>
                    : pencil_kernel<SOFT_CUBIC_SPLINE, false, 4, 8, 2>;
    default:
        return dens ? pencil_kernel<SOFT_CUBIC_PLUMMER, true, 4, 8, 2>
                    : pencil_kernel<SOFT_CUBIC_PLUMMER, false, 4, 8, 2>;
    }
}

static size_t kernel_smem() { return sizeof(WarpSmem) * WARPS_PER_CTA + sizeof(CombSmem); }

static inline int wrap_h(int i, int cpd) {
    while (i < 0) i += cpd;
    while (i >= cpd) i -= cpd;
    return i;
}

// Source cell order: outer ring (max(|dx|,|dy|) == R >= 2) first, so that the
// chunks that can hold pairs closer than one cell width come last.
static void source_order(int R, signed char *odx, signed char *ody, int *n_outer) {
    int n = 0;
    for (int pass = 0; pass < 2; pass++)
        for (int dx = -R; dx <= R; dx++)
            for (int dy = -R; dy <= R; dy++) {
                bool outer = std::max(std::abs(dx), std::abs(dy)) >= 2;
                if ((pass == 0) == outer) {
                    odx[n] = (signed char)dx;
                    ody[n] = (signed char)dy;
                    n++;
                }
            }
    int no = 0;
    for (int dx = -R; dx <= R; dx++)
        for (int dy = -R; dy <= R; dy++)
            if (std::max(std::abs(dx), std::abs(dy)) >= 2) no++;
    *n_outer = no;
}

struct HostTile {
    Item it;
    double cost;
};

static nf_status build_plan(nf_ctx *ctx, nf_box *box, int lo, int hi, int variant, Plan &pl) {
    const int cpd = box->cpd, R = ctx->cfg.near_field_radius, W = 2 * R + 1;
    const auto &cs = box->cell_start;
    auto count = [&](int x, int y, int z) -> int64_t {
        int64_t c = ((int64_t)wrap_h(x, cpd) * cpd + wrap_h(y, cpd)) * cpd + wrap_h(z, cpd);
        return cs[c + 1] - cs[c];
    };
    pl.lo = lo;
    pl.hi = hi;
    pl.variant = variant;
    const int smax = VARIANTS[variant].smax;
    const int unr = VARIANTS[variant].unr;
    pl.p0 = cs[(int64_t)lo * cpd * cpd];
    pl.n_range = cs[(int64_t)hi * cpd * cpd] - pl.p0;
    std::vector<HostTile> tiles;
    tiles.reserve((size_t)(hi - lo) * cpd * cpd + 1024);
    uint64_t pairs = 0, padded = 0;
    double total = 0;
    int forced_S = ctx->cfg.sinks_per_lane;
    for (int x = lo; x < hi; x++)
        for (int y = 0; y < cpd; y++)
            for (int zc = 0; zc < cpd; zc++) {
                int64_t np_ = 0;
                for (int a = -R; a <= R; a++) np_ += count(x, y, zc + a);
                if (np_ == 0) continue;
                int64_t M = 0;
                for (int dx = -R; dx <= R; dx++)
                    for (int dy = -R; dy <= R; dy++) M += count(x + dx, y + dy, zc);
                if (np_ > INT32_MAX / 2 || M > INT32_MAX / 2) {
                    set_error("pencil too large for 32-bit stream indices");
                    return NF_EINVAL;
                }
                int pencil = (int)(((int64_t)x * cpd + y) * cpd + zc);
                int64_t done = 0;
                while (done < np_) {
                    int64_t rem = np_ - done;
                    int S;
                    if (forced_S)
                        S = std::min(forced_S, smax);
                    else  // smallest tile that holds the rest; a rest of 65-96 sinks
                          // takes 64 + 32 slots instead of 128
                        S = rem <= 32 ? 1
                            : (rem <= 96 || smax == 2) ? 2
                            : (rem <= 128 || smax == 4) ? 4 : 8;
                    int take = (int)std::min<int64_t>(rem, 32 * S);
                    HostTile t;
                    t.it = Item{pencil, (int)done, take, S, 0, (int)M, 0, 0};
                    int64_t Mpad = (M / CHUNK) * CHUNK + ((M % CHUNK) + unr - 1) / unr * unr;
                    t.cost = (double)(32 * S) * (double)Mpad + 2000.0 * S;
                    pairs += (uint64_t)take * (uint64_t)M;
                    padded += (uint64_t)(32 * S) * (uint64_t)Mpad;
                    total += t.cost;
                    tiles.push_back(t);
                    done += take;
                }
            }
    pl.pairs = pairs;
    pl.padded_pairs = padded;
    // occupancy-derived persistent grid
    KernelFn fn = pick_kernel(ctx->cfg.softening, ctx->cfg.b2 > 0.f, variant);
    int per_sm = 0;
    NF_CUDA(cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kernel_smem()));
    NF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)fn,
                                                          WARPS_PER_CTA * 32, kernel_smem()));
    if (per_sm < 1) per_sm = 1;
    pl.grid = ctx->sms * per_sm;
    pl.warps = pl.grid * WARPS_PER_CTA;
    // heavy threshold: a tile costing more than half the mean per-warp share
    double thr = total / (2.0 * pl.warps);
    std::vector<HostTile> heavy, light;
    for (auto &t : tiles) {
        if (t.cost > thr && t.it.src_end >= 64 * WARPS_PER_CTA) {
            // split tiles are summed through shared memory sized for
            // TILE_MAX sinks: halve larger tiles first
            if (t.it.nsink > TILE_MAX) {
                HostTile a = t, b = t;
                a.it.S = b.it.S = 4;
                a.it.nsink = TILE_MAX;
                b.it.sink_begin += TILE_MAX;
                b.it.nsink = t.it.nsink - TILE_MAX;
                if (b.it.nsink <= 64) b.it.S = b.it.nsink <= 32 ? 1 : 2;
                a.cost = b.cost = t.cost / 2;
                heavy.push_back(a);
                heavy.push_back(b);
            } else {
                heavy.push_back(t);
            }
        } else {
            light.push_back(t);
        }
    }
    auto by_cost = [](const HostTile &a, const HostTile &b) {
        if (a.cost != b.cost) return a.cost > b.cost;
        if (a.it.pencil != b.it.pencil) return a.it.pencil < b.it.pencil;
        return a.it.sink_begin < b.it.sink_begin;
    };
    std::sort(heavy.begin(), heavy.end(), by_cost);
    std::sort(light.begin(), light.end(), by_cost);
    std::vector<Item> hv;
    hv.reserve(heavy.size() * WARPS_PER_CTA);
    for (auto &t : heavy) {
        int M = t.it.src_end;
        int per = ((M + WARPS_PER_CTA - 1) / WARPS_PER_CTA + CHUNK - 1) / CHUNK * CHUNK;
        for (int w = 0; w < WARPS_PER_CTA; w++) {
            Item it = t.it;
            it.src_begin = std::min(M, w * per);
            it.src_end = std::min(M, (w + 1) * per);
            hv.push_back(it);
        }
    }
    std::vector<Item> lv;
    lv.reserve(light.size());
    for (auto &t : light) lv.push_back(t.it);
    pl.n_heavy_groups = (int)heavy.size();
    pl.n_light = (int)lv.size();
    NF_CUDA(cudaMalloc(&pl.d_counters, 2 * sizeof(int)));
    if (!hv.empty()) {
        NF_CUDA(cudaMalloc(&pl.d_heavy, hv.size() * sizeof(Item)));
        NF_CUDA(cudaMemcpy(pl.d_heavy, hv.data(), hv.size() * sizeof(Item), cudaMemcpyHostToDevice));
    }
    if (!lv.empty()) {
        NF_CUDA(cudaMalloc(&pl.d_light, lv.size() * sizeof(Item)));
        NF_CUDA(cudaMemcpy(pl.d_light, lv.data(), lv.size() * sizeof(Item), cudaMemcpyHostToDevice));
    }
    int rec = ctx->cfg.out_kind == NF_OUT_FLOAT4 ? 16 : 12;
    pl.out_bytes = (size_t)pl.n_range * rec;
    NF_CUDA(cudaMalloc(&pl.d_out, pl.out_bytes ? pl.out_bytes : 16));
    (void)W;
    return NF_OK;
}

static void free_plan(Plan &pl) {
    if (pl.graph) cudaGraphExecDestroy(pl.graph);
    cudaFree(pl.d_heavy);
    cudaFree(pl.d_light);
    cudaFree(pl.d_counters);
    cudaFree(pl.d_out);
    pl = Plan{};
}

static KParams params_from(nf_ctx *ctx, const EngineLaunch &L) {
    KParams kp;
    memset(&kp, 0, sizeof(kp));
    const nf_config &cfg = ctx->cfg;
    const int R = cfg.near_field_radius;
    kp.pos = L.pos;
    kp.cs = L.cs;
    kp.cpd = L.cpd;
    kp.R = R;
    kp.heavy = L.heavy;
    kp.n_heavy_groups = L.n_heavy_groups;
    kp.light = L.light;
    kp.n_light = L.n_light;
    kp.counters = L.counters;
    kp.part = L.part;
    kp.p0 = L.p0;
    kp.n_range = L.n_range;
    kp.nc = cfg.b2 > 0.f ? 4 : 3;
    kp.plain = cfg.accumulation == NF_ACC_PLAIN;
    const float eps = L.eps > 0.f ? L.eps : cfg.eps;
    kp.pc.eps = eps;
    kp.pc.b2 = cfg.b2;
    if (cfg.softening == SOFT_SINGLE_SPLINE) {
        double ie2 = (double)eps;  // eps_int^-2
        kp.pc.near_thr = (float)(1.0 / ie2);
        kp.pc.inv_eps3 = (float)pow(ie2, 1.5);
        kp.pc.c1 = (float)(-15.0 * ie2 * ie2);
        kp.pc.c2 = (float)(6.0 * pow(ie2, 2.5));
        kp.pc.c3 = (float)(10.0 * pow(ie2, 1.5));
    }
    {
        // margin of the near test: eps (+1% and a rounding allowance)
        double h = 1.0 / (double)L.cpd;
        double e = cfg.softening == SOFT_SINGLE_SPLINE ? 1.0 / sqrt((double)eps) : 0.0;
        kp.near_w = (float)(e * 1.01 + 1e-6 * h);
    }
    double h = 1.0 / (double)L.cpd;
    for (int a = 0; a < 2 * R + 1; a++) {
        kp.zshift[a] = (float)((a - R) * h);
        kp.xyshift[a] = (float)((a - R) * h);
    }
    source_order(R, kp.odx, kp.ody, &kp.n_outer);
    return kp;
}

static KParams make_params(nf_ctx *ctx, nf_box *box, const Plan &pl) {
    EngineLaunch L;
    L.pos = box->d_pos;
    L.cs = box->d_cs;
    L.cpd = box->cpd;
    L.heavy = pl.d_heavy;
    L.n_heavy_groups = pl.n_heavy_groups;
    L.light = pl.d_light;
    L.n_light = pl.n_light;
    L.counters = pl.d_counters;
    L.part = box->d_part;
    L.p0 = pl.p0;
    L.n_range = pl.n_range;
    L.variant = pl.variant;
    L.eps = box->eps;
    return params_from(ctx, L);
}

// Output scale of the co-add, formed in double on the host and rounded once
// to float (single spline: eps_int^3, the raw kernel's units; otherwise 1).
// eps: the softening parameter in use (0: the context's).
static float output_scale(const nf_config &cfg, float eps = 0.f) {
    if (eps <= 0.f) eps = cfg.eps;
    if (cfg.softening == SOFT_SINGLE_SPLINE) return (float)pow((double)eps, -1.5);  // eps_int^3
    return 1.0f;
}

int engine_variant_smax(int variant) { return VARIANTS[variant].smax; }
// The plain drop-in runs the reference's block shape: 64-sink tiles.
int engine_plain_variant() { return 3; }

int engine_grid(nf_ctx *ctx, int variant) {
    KernelFn fn = pick_kernel(ctx->cfg.softening, ctx->cfg.b2 > 0.f, variant);
    int per_sm = 0;
    if (cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kernel_smem()) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)fn,
                                                      WARPS_PER_CTA * 32, kernel_smem()) !=
            cudaSuccess) {
        cudaGetLastError();
        per_sm = 1;
    }
    return ctx->sms * std::max(per_sm, 1);
}

nf_status engine_launch(nf_ctx *ctx, const EngineLaunch &L, double, cudaStream_t st) {
    if (L.n_heavy_groups + L.n_light == 0) return NF_OK;
    KParams kp = params_from(ctx, L);
    KernelFn fn = pick_kernel(ctx->cfg.softening, ctx->cfg.b2 > 0.f, L.variant);
    NF_CUDA(cudaMemsetAsync(L.counters, 0, 2 * sizeof(int), st));
    int grid = L.grid > 0 ? L.grid : engine_grid(ctx, L.variant);
    void *args[] = {&kp};
    NF_CUDA(cudaLaunchKernel((const void *)fn, dim3(grid), dim3(WARPS_PER_CTA * 32), args,
                             kernel_smem(), st));
    return NF_OK;
}

nf_status engine_coadd(nf_ctx *ctx, const Partial *part, int64_t n, void *out, cudaStream_t st,
                       float eps, const uint32_t *perm, int64_t p0) {
    if (n <= 0) return NF_OK;
    const nf_config &cfg = ctx->cfg;
    coadd_kernel<<<ctx->sms * 8, 256, 0, st>>>(part, n, 2 * cfg.near_field_radius + 1,
                                              cfg.b2 > 0.f ? 4 : 3, output_scale(cfg, eps),
                                              cfg.out_kind, out, perm, p0);
    NF_CUDA(cudaGetLastError());
    return NF_OK;
}

nf_status engine_pack(nf_ctx *ctx, const float *x, const float *y, const float *z, int64_t n,
                      float4 *out, cudaStream_t st) {
    if (n <= 0) return NF_OK;
    pack_positions<<<ctx->sms * 8, 256, 0, st>>>(x, y, z, n, out);
    NF_CUDA(cudaGetLastError());
    return NF_OK;
}

// The pencil kernel of a plan into the box's partials, between events 0 and 1.
static nf_status enqueue_pencil(nf_ctx *ctx, nf_box *box, Plan &pl, cudaStream_t st,
                                unsigned evflags) {
    const nf_config &cfg = ctx->cfg;
    KParams kp = make_params(ctx, box, pl);
    KernelFn fn = pick_kernel(cfg.softening, cfg.b2 > 0.f, pl.variant);
    NF_CUDA(cudaMemsetAsync(pl.d_counters, 0, 2 * sizeof(int), st));
    NF_CUDA(cudaEventRecordWithFlags(ctx->ev[0], st, evflags));
    if (pl.n_heavy_groups + pl.n_light > 0) {
        void *args[] = {&kp};
        NF_CUDA(cudaLaunchKernel((const void *)fn, dim3(pl.grid), dim3(WARPS_PER_CTA * 32), args,
                                 kernel_smem(), st));
    }
    NF_CUDA(cudaEventRecordWithFlags(ctx->ev[1], st, evflags));
    return NF_OK;
}

static nf_status enqueue_forces(nf_ctx *ctx, nf_box *box, Plan &pl, cudaStream_t st) {
    const nf_config &cfg = ctx->cfg;
    nf_status est = enqueue_pencil(ctx, box, pl, st, cudaEventRecordExternal);
    if (est != NF_OK) return est;
    const int nc = cfg.b2 > 0.f ? 4 : 3;
    if (pl.n_range > 0) {
        int W = 2 * cfg.near_field_radius + 1;
        int blocks = ctx->sms * 8;
        coadd_kernel<<<blocks, 256, 0, st>>>(box->d_part, pl.n_range, W, nc, output_scale(cfg, box->eps),
                                            cfg.out_kind, pl.d_out, box->d_perm, pl.p0);
        NF_CUDA(cudaGetLastError());
    }
    NF_CUDA(cudaEventRecordWithFlags(ctx->ev[2], st, cudaEventRecordExternal));
    return NF_OK;
}

// The plan's CUDA graph (pencil kernel + co-add), captured on first use.
static nf_status ensure_graph(nf_ctx *ctx, nf_box *box, Plan &pl) {
    if (pl.graph) return NF_OK;
    cudaStream_t s = ctx->stream;
    cudaGraph_t g = nullptr;
    NF_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    nf_status est = enqueue_forces(ctx, box, pl, s);
    cudaError_t ce = cudaStreamEndCapture(s, &g);
    if (est != NF_OK) {
        if (g) cudaGraphDestroy(g);
        return est;
    }
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
    ce = cudaGraphInstantiate(&pl.graph, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) {
        pl.graph = nullptr;
        return cuda_fail(ce, "cudaGraphInstantiate");
    }
    return NF_OK;
}

}  // namespace nf

using namespace nf;

size_t nf_box::device_bytes() const {
    size_t b = (size_t)np * sizeof(float4) + cell_start.size() * sizeof(int64_t) + part_bytes +
               (d_stage ? 3 * (size_t)np * sizeof(float) : 0) + sort_bytes +
               (d_perm ? (size_t)np * sizeof(uint32_t) : 0);
    for (auto &kv : plans) {
        b += kv.second->out_bytes + (size_t)kv.second->n_light * sizeof(Item) +
             (size_t)kv.second->n_heavy_groups * WARPS_PER_CTA * sizeof(Item);
    }
    return b;
}

extern "C" nf_status nf_box_create(nf_ctx *ctx, int cpd, int64_t np, const int64_t *cell_start,
                                   const float *x, const float *y, const float *z,
                                   nf_box **out) {
    if (!ctx || !out || !cell_start || (np > 0 && (!x || !y || !z))) {
        set_error("nf_box_create: null argument");
        return NF_EINVAL;
    }
    if (cpd < 2 * ctx->cfg.near_field_radius + 1 || (cpd & 1) == 0 || np < 0) {
        set_error("nf_box_create: cpd must be odd and >= 2R+1");
        return NF_EINVAL;
    }
    // work items name a pencil by its centre cell's linear id in 32 bits
    if (np >= ((int64_t)1 << 31) || (int64_t)cpd * cpd * cpd >= ((int64_t)1 << 31)) {
        set_error("nf_box_create: at most 2^31 - 1 particles and cpd^3 < 2^31 cells "
                  "(cpd <= 1290) per box");
        return NF_EINVAL;
    }
    int64_t ncell = (int64_t)cpd * cpd * cpd;
    if (cell_start[0] != 0 || cell_start[ncell] != np) {
        set_error("nf_box_create: cell_start must run from 0 to np");
        return NF_EINVAL;
    }
    for (int64_t c = 0; c < ncell; c++)
        if (cell_start[c + 1] < cell_start[c]) {
            set_error("nf_box_create: cell_start not monotone");
            return NF_EINVAL;
        }
    NF_CUDA(cudaSetDevice(ctx->device));
    std::unique_ptr<nf_box> box(new nf_box);
    box->cpd = cpd;
    box->np = np;
    box->cell_start.assign(cell_start, cell_start + ncell + 1);
    if (cudaMalloc(&box->d_pos, (size_t)std::max<int64_t>(np, 1) * sizeof(float4)) != cudaSuccess ||
        cudaMalloc(&box->d_cs, (size_t)(ncell + 1) * sizeof(int64_t)) != cudaSuccess) {
        cudaFree(box->d_pos);
        cudaFree(box->d_cs);
        cudaGetLastError();
        set_error("nf_box_create: device allocation failed");
        return NF_ENOMEM;
    }
    NF_CUDA(cudaMemcpy(box->d_cs, cell_start, (size_t)(ncell + 1) * sizeof(int64_t),
                       cudaMemcpyHostToDevice));
    *out = box.release();
    nf_status st = np > 0 ? nf_box_update(ctx, *out, x, y, z) : NF_OK;
    if (st != NF_OK) {
        nf_box_destroy(ctx, *out);
        *out = nullptr;
    }
    return st;
}

namespace nf {
// Upload positions into a box: SoA (x, y, z arrays; aos == nullptr) or AoS
// (aos = n records of three floats), host or device memory; then order the
// particles inside their cells and pack them (ctx->mu held by the caller).
static nf_status box_upload(nf_ctx *ctx, nf_box *box, const float *x, const float *y,
                            const float *z, const float *aos);
}  // namespace nf

extern "C" nf_status nf_box_update(nf_ctx *ctx, nf_box *box, const float *x, const float *y,
                                   const float *z) {
    if (!ctx || !box || !x || !y || !z) {
        set_error("nf_box_update: null argument");
        return NF_EINVAL;
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    return box_upload(ctx, box, x, y, z, nullptr);
}

extern "C" nf_status nf_box_update_aos(nf_ctx *ctx, nf_box *box, const float *xyz) {
    if (!ctx || !box || (!xyz && box->np > 0)) {
        set_error("nf_box_update_aos: null argument");
        return NF_EINVAL;
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    return box_upload(ctx, box, nullptr, nullptr, nullptr, xyz);
}

namespace nf {
// Staging buffer, ordering scratch and permutation of a box (allocated once).
struct OrderScratch {
    uint64_t *k_in, *k_out;
    uint32_t *v_in;
    void *temp;
    size_t temp_bytes;
    int key_bits;
};

static nf_status upload_scratch(nf_ctx *ctx, nf_box *box, OrderScratch &o) {
    const int64_t n = box->np;
    const size_t bytes = (size_t)n * sizeof(float);
    if (!box->d_stage && n > 0) {
        if (cudaMalloc(&box->d_stage, 3 * bytes) != cudaSuccess) {
            cudaGetLastError();
            box->d_stage = nullptr;
            set_error("nf_box_update: device allocation failed");
            return NF_ENOMEM;
        }
    }
    const int64_t ncell = (int64_t)box->cpd * box->cpd * box->cpd;
    o.key_bits = 30;
    while (o.key_bits < 64 && ((uint64_t)1 << (o.key_bits - 30)) < (uint64_t)ncell) o.key_bits++;
    o.temp_bytes = 0;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(
        nullptr, o.temp_bytes, (const uint64_t *)nullptr, (uint64_t *)nullptr,
        (const uint32_t *)nullptr, (uint32_t *)nullptr, (int)n, 0, o.key_bits, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "box upload (ordering size query)");
    const size_t kb = ((size_t)n * 8 + 255) & ~(size_t)255, vb = ((size_t)n * 4 + 255) & ~(size_t)255;
    const size_t need = 2 * kb + vb + o.temp_bytes;
    if (box->sort_bytes < need) {
        cudaFree(box->d_sort);
        box->d_sort = nullptr;
        box->sort_bytes = 0;
        if (cudaMalloc(&box->d_sort, need) != cudaSuccess) {
            cudaGetLastError();
            box->d_sort = nullptr;
            set_error("nf_box_update: device allocation failed (ordering scratch)");
            return NF_ENOMEM;
        }
        box->sort_bytes = need;
    }
    if (!box->d_perm && cudaMalloc(&box->d_perm, vb) != cudaSuccess) {
        cudaGetLastError();
        box->d_perm = nullptr;
        set_error("nf_box_update: device allocation failed (permutation)");
        return NF_ENOMEM;
    }
    unsigned char *sb = (unsigned char *)box->d_sort;
    o.k_in = (uint64_t *)sb;
    o.k_out = (uint64_t *)(sb + kb);
    o.v_in = (uint32_t *)(sb + 2 * kb);
    o.temp = sb + 2 * kb + vb;
    return NF_OK;
}

// Order the staged particles [p0, p1) inside their cells and pack them into
// the box (the range must hold whole cells).  Components at x/y/z with
// stride cstride.
static cudaError_t order_range(nf_ctx *ctx, nf_box *box, const OrderScratch &o, const float *x,
                               const float *y, const float *z, int cstride, int64_t p0,
                               int64_t p1, cudaStream_t st) {
    if (p1 <= p0) return cudaSuccess;
    const int64_t ncell = (int64_t)box->cpd * box->cpd * box->cpd;
    order_keys<<<ctx->sms * 8, 256, 0, st>>>(x, y, z, cstride, box->d_cs, ncell, box->cpd, p0, p1,
                                             o.k_in, o.v_in);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    size_t tb = o.temp_bytes;
    e = cub::DeviceRadixSort::SortPairs(o.temp, tb, o.k_in + p0, o.k_out + p0, o.v_in + p0,
                                        box->d_perm + p0, (int)(p1 - p0), 0, o.key_bits, st);
    if (e != cudaSuccess) return e;
    pack_ordered<<<ctx->sms * 8, 256, 0, st>>>(x, y, z, cstride, box->d_perm, p0, p1, box->d_pos);
    return cudaGetLastError();
}
}  // namespace nf

static nf_status nf::box_upload(nf_ctx *ctx, nf_box *box, const float *x, const float *y,
                                const float *z, const float *aos) {
    NF_CUDA(cudaSetDevice(ctx->device));
    OrderScratch o;
    nf_status ost = upload_scratch(ctx, box, o);
    if (ost != NF_OK) return ost;
    const int64_t n = box->np;
    const size_t bytes = (size_t)n * sizeof(float);
    float *tmp = box->d_stage;
    cudaStream_t st = ctx->stream;
    // staged components: SoA at tmp, tmp + n, tmp + 2n (stride 1) or the
    // AoS records as given at tmp, tmp + 1, tmp + 2 (stride 3)
    const float *sx = tmp, *sy = aos ? tmp + 1 : tmp + n, *sz = aos ? tmp + 2 : tmp + 2 * n;
    cudaError_t e;
    if (aos) {
        e = cudaMemcpyAsync(tmp, aos, 3 * bytes, cudaMemcpyDefault, st);
    } else {
        e = cudaMemcpyAsync(tmp, x, bytes, cudaMemcpyDefault, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(tmp + n, y, bytes, cudaMemcpyDefault, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(tmp + 2 * n, z, bytes, cudaMemcpyDefault, st);
    }
    if (e == cudaSuccess) e = order_range(ctx, box, o, sx, sy, sz, aos ? 3 : 1, 0, n, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "nf_box_update");
    return NF_OK;
}

extern "C" void nf_box_destroy(nf_ctx *ctx, nf_box *box) {
    if (!box) return;
    if (ctx) cudaSetDevice(ctx->device);
    for (auto &kv : box->plans) free_plan(*kv.second);
    cudaFree(box->d_pos);
    cudaFree(box->d_cs);
    cudaFree(box->d_part);
    cudaFree(box->d_stage);
    cudaFree(box->d_perm);
    cudaFree(box->d_sort);
    if (box->s_in) cudaStreamDestroy(box->s_in);
    if (box->s_out) cudaStreamDestroy(box->s_out);
    for (cudaEvent_t e : box->step_ev) cudaEventDestroy(e);
    delete box;
}

extern "C" nf_status nf_box_set_eps(nf_ctx *ctx, nf_box *box, float eps) {
    if (!ctx || !box || !(eps >= 0.f) || !std::isfinite(eps)) {
        set_error("nf_box_set_eps: bad argument (eps must be finite and >= 0)");
        return NF_EINVAL;
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    NF_CUDA(cudaSetDevice(ctx->device));
    if (eps == box->eps) return NF_OK;
    // cached plans hold graphs with the old constants: wait for every launch
    // that may use them, then drop them (the kernel-shape choice is kept)
    NF_CUDA(cudaDeviceSynchronize());
    for (auto &kv : box->plans) free_plan(*kv.second);
    box->plans.clear();
    box->eps = eps;
    return NF_OK;
}

extern "C" size_t nf_box_device_bytes(const nf_box *box) { return box ? box->device_bytes() : 0; }

extern "C" nf_status nf_box_pair_count(nf_ctx *ctx, const nf_box *box, int lo, int hi,
                                       uint64_t *pairs) {
    if (!ctx || !box || !pairs || lo < 0 || hi > box->cpd || lo >= hi) {
        set_error("nf_box_pair_count: bad argument");
        return NF_EINVAL;
    }
    const int cpd = box->cpd, R = ctx->cfg.near_field_radius;
    const auto &cs = box->cell_start;
    auto count = [&](int x, int y, int z) -> uint64_t {
        int64_t c = ((int64_t)wrap_h(x, cpd) * cpd + wrap_h(y, cpd)) * cpd + wrap_h(z, cpd);
        return (uint64_t)(cs[c + 1] - cs[c]);
    };
    uint64_t tot = 0;
    for (int x = lo; x < hi; x++)
        for (int y = 0; y < cpd; y++)
            for (int z = 0; z < cpd; z++) {
                uint64_t ns = count(x, y, z);
                if (!ns) continue;
                uint64_t src = 0;
                for (int dx = -R; dx <= R; dx++)
                    for (int dy = -R; dy <= R; dy++)
                        for (int dz = -R; dz <= R; dz++) src += count(x + dx, y + dy, z + dz);
                tot += ns * src;
            }
    *pairs = tot;
    return NF_OK;
}

// Partial scratch: (2R+1) slots x nc components x n_range (hi, lo) pairs, shared by
// the box's plans (grown on demand; cached graphs that refer to the old
// buffer are dropped).
static nf_status ensure_scratch(nf_ctx *ctx, nf_box *box, int64_t n_range) {
    int nc = ctx->cfg.b2 > 0.f ? 4 : 3;
    size_t need = (size_t)(2 * ctx->cfg.near_field_radius + 1) * nc * (size_t)n_range * sizeof(Partial);
    if (need <= box->part_bytes) return NF_OK;
    cudaFree(box->d_part);
    box->d_part = nullptr;
    box->part_bytes = 0;
    for (auto &kv : box->plans)
        if (kv.second->graph) {
            cudaGraphExecDestroy(kv.second->graph);
            kv.second->graph = nullptr;
        }
    if (cudaMalloc(&box->d_part, need) != cudaSuccess) {
        cudaGetLastError();
        set_error("nf_box_forces: cannot allocate partial scratch");
        return NF_ENOMEM;
    }
    box->part_bytes = need;
    return NF_OK;
}

static nf_status new_plan(nf_ctx *ctx, nf_box *box, int lo, int hi, int variant,
                          std::unique_ptr<Plan> &out) {
    std::unique_ptr<Plan> pl(new Plan);
    nf_status st = build_plan(ctx, box, lo, hi, variant, *pl);
    if (st == NF_OK) st = ensure_scratch(ctx, box, pl->n_range);
    if (st != NF_OK) {
        free_plan(*pl);
        return st;
    }
    out = std::move(pl);
    return NF_OK;
}

// Device time of one launch of a plan's pencil kernel (no co-add).
static nf_status time_pencil(nf_ctx *ctx, nf_box *box, Plan &pl, float *ms) {
    nf_status st = enqueue_pencil(ctx, box, pl, ctx->stream, cudaEventRecordDefault);
    if (st != NF_OK) return st;
    NF_CUDA(cudaEventSynchronize(ctx->ev[1]));
    NF_CUDA(cudaEventElapsedTime(ms, ctx->ev[0], ctx->ev[1]));
    return NF_OK;
}

// The autotuner: run every candidate kernel shape on the requested slab
// range and keep the fastest for the box.  A candidate whose first launch
// is short (< 50 ms, where loading the kernel and a cold L2 weigh) is timed
// again and the second launch counts; a long first launch counts as it is.
static nf_status autotune(nf_ctx *ctx, nf_box *box, int lo, int hi) {
    const bool tun = tunable(ctx->cfg.softening, ctx->cfg.b2 > 0.f);
    const int nv = tun ? NVARIANTS : 1;
    int best = 0;
    float best_ms = 3.0e38f;
    for (int v = 0; v < nv; v++) {
        std::unique_ptr<Plan> pl;
        nf_status st = new_plan(ctx, box, lo, hi, v, pl);
        if (st != NF_OK) return st;
        float ms = 0;
        st = time_pencil(ctx, box, *pl, &ms);
        if (st == NF_OK && ms < 50.f) st = time_pencil(ctx, box, *pl, &ms);
        free_plan(*pl);
        if (st != NF_OK) return st;
        box->tune_ms[v] = ms;
        if (ms < best_ms) {
            best_ms = ms;
            best = v;
        }
    }
    box->variant = best;
    return NF_OK;
}

static nf_status get_plan(nf_ctx *ctx, nf_box *box, int lo, int hi, Plan **out) {
    auto key = std::make_pair(lo, hi);
    auto it = box->plans.find(key);
    if (it != box->plans.end()) {
        *out = it->second.get();
        return NF_OK;
    }
    int v = ctx->cfg.kernel_variant;
    if (v < 0) {
        if (box->variant < 0) {
            nf_status st = autotune(ctx, box, lo, hi);
            if (st != NF_OK) return st;
        }
        v = box->variant;
    }
    std::unique_ptr<Plan> pl;
    nf_status st = new_plan(ctx, box, lo, hi, v, pl);
    if (st != NF_OK) return st;
    *out = pl.get();
    box->plans[key] = std::move(pl);
    return NF_OK;
}

// The cached plan of a slab range (built, and the box tuned, on first use),
// for launches that bring their own partials, counters and output (serving).
nf_status nf::box_plan(nf_ctx *ctx, nf_box *box, int lo, int hi, const Plan **out) {
    std::lock_guard<std::mutex> lk(ctx->mu);
    NF_CUDA(cudaSetDevice(ctx->device));
    Plan *pl = nullptr;
    nf_status st = get_plan(ctx, box, lo, hi, &pl);
    *out = pl;
    return st;
}

extern "C" int nf_kernel_variant_count(void) { return NVARIANTS; }

extern "C" const char *nf_kernel_variant_name(int v) {
    return (v >= 0 && v < NVARIANTS) ? VARIANTS[v].name : "";
}

extern "C" nf_status nf_box_tuning(const nf_box *box, int *variant, float *ms, int n) {
    if (!box || !variant) {
        set_error("nf_box_tuning: null argument");
        return NF_EINVAL;
    }
    *variant = box->variant;
    for (int i = 0; ms && i < n && i < NVARIANTS; i++) ms[i] = box->tune_ms[i];
    return NF_OK;
}

extern "C" nf_status nf_box_forces(nf_ctx *ctx, nf_box *box, int lo, int hi, void *out,
                                   int out_on_device) {
    if (!ctx || !box || !out || lo < 0 || hi > box->cpd || lo >= hi) {
        set_error("nf_box_forces: bad argument");
        return NF_EINVAL;
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    NF_CUDA(cudaSetDevice(ctx->device));
    Plan *pl = nullptr;
    nf_status st = get_plan(ctx, box, lo, hi, &pl);
    if (st == NF_OK) st = ensure_graph(ctx, box, *pl);
    if (st != NF_OK) return st;
    cudaStream_t s = ctx->stream;
    cudaEventRecord(ctx->ev[3], s);
    NF_CUDA(cudaGraphLaunch(pl->graph, s));
    NF_CUDA(cudaMemcpyAsync(out, pl->d_out, pl->out_bytes,
                            out_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
    NF_CUDA(cudaStreamSynchronize(s));
    float k_ms = 0, c_ms = 0, t_ms = 0;
    cudaEventElapsedTime(&k_ms, ctx->ev[0], ctx->ev[1]);
    cudaEventElapsedTime(&c_ms, ctx->ev[1], ctx->ev[2]);
    cudaEventElapsedTime(&t_ms, ctx->ev[3], ctx->ev[2]);
    ctx->last.kernel_ms = k_ms;
    ctx->last.coadd_ms = c_ms;
    ctx->last.total_ms = t_ms;
    ctx->last.pairs = pl->pairs;
    ctx->last.padded_pairs = pl->padded_pairs;
    ctx->last.launches = (pl->n_heavy_groups + pl->n_light > 0 ? 1 : 0) + (pl->n_range > 0 ? 1 : 0);
    ctx->last.items = pl->n_heavy_groups * WARPS_PER_CTA + pl->n_light;
    ctx->last.variant = pl->variant;
    return NF_OK;
}

extern "C" nf_status nf_box_kick(nf_ctx *ctx, nf_box *box, int lo, int hi,
                                 const nf_kick_params *kick, const float *far_acc, float *vel,
                                 void *acc_out, float *cell_stats) {
    if (!ctx || !box || !kick || !vel || lo < 0 || hi > box->cpd || lo >= hi) {
        set_error("nf_box_kick: bad argument");
        return NF_EINVAL;
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    NF_CUDA(cudaSetDevice(ctx->device));
    // the kernel dereferences these directly: they must be device-accessible
    for (const void *q : {(const void *)far_acc, (const void *)vel, (const void *)acc_out,
                          (const void *)cell_stats}) {
        if (!q) continue;
        cudaPointerAttributes pa;
        if (cudaPointerGetAttributes(&pa, q) != cudaSuccess || !pa.devicePointer) {
            cudaGetLastError();
            set_error("nf_box_kick: far_acc, vel, acc_out and cell_stats must be device memory");
            return NF_EINVAL;
        }
    }
    Plan *pl = nullptr;
    nf_status st = get_plan(ctx, box, lo, hi, &pl);
    if (st != NF_OK) return st;
    cudaStream_t s = ctx->stream;
    const nf_config &cfg = ctx->cfg;
    cudaEventRecord(ctx->ev[3], s);
    st = enqueue_pencil(ctx, box, *pl, s, cudaEventRecordDefault);
    if (st != NF_OK) return st;
    const int64_t c2 = (int64_t)box->cpd * box->cpd;
    KickConst k{kick->near_scale, kick->rescale, kick->kick1, kick->kick2, kick->b2};
    if (pl->n_range > 0 || cell_stats) {
        kick_kernel<<<ctx->sms * 8, 256, 0, s>>>(
            box->d_part, pl->n_range, 2 * cfg.near_field_radius + 1, cfg.b2 > 0.f ? 4 : 3,
            output_scale(cfg, box->eps), box->d_cs, (int64_t)lo * c2, (int64_t)(hi - lo) * c2,
            pl->p0, box->d_perm, k, far_acc, vel, acc_out, cfg.out_kind, cell_stats);
        NF_CUDA(cudaGetLastError());
    }
    NF_CUDA(cudaEventRecord(ctx->ev[2], s));
    NF_CUDA(cudaStreamSynchronize(s));
    float k_ms = 0, c_ms = 0, t_ms = 0;
    cudaEventElapsedTime(&k_ms, ctx->ev[0], ctx->ev[1]);
    cudaEventElapsedTime(&c_ms, ctx->ev[1], ctx->ev[2]);
    cudaEventElapsedTime(&t_ms, ctx->ev[3], ctx->ev[2]);
    ctx->last.kernel_ms = k_ms;
    ctx->last.coadd_ms = c_ms;
    ctx->last.total_ms = t_ms;
    ctx->last.pairs = pl->pairs;
    ctx->last.padded_pairs = pl->padded_pairs;
    ctx->last.launches = (pl->n_heavy_groups + pl->n_light > 0 ? 1 : 0) + 1;
    ctx->last.items = pl->n_heavy_groups * WARPS_PER_CTA + pl->n_light;
    ctx->last.variant = pl->variant;
    return NF_OK;
}

extern "C" nf_status nf_box_step(nf_ctx *ctx, nf_box *box, const float *x, const float *y,
                                 const float *z, void *out, int n_chunks) {
    if (!ctx || !box || !out || (box->np > 0 && (!x || !y || !z))) {
        set_error("nf_box_step: null argument");
        return NF_EINVAL;
    }
    const int cpd = box->cpd, R = ctx->cfg.near_field_radius;
    int K = n_chunks > 0 ? n_chunks : 8;
    K = std::max(1, std::min(K, cpd / std::max(R, 1)));
    if (n_chunks > 0 && K != n_chunks) {
        set_error("nf_box_step: every chunk needs at least R slabs");
        return NF_EINVAL;
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    NF_CUDA(cudaSetDevice(ctx->device));
    // chunk bounds (slabs) and the plans of the chunk ranges
    std::vector<int> b(K + 1);
    for (int k = 0; k <= K; k++) b[k] = (int)((int64_t)cpd * k / K);
    std::vector<Plan *> pls(K);
    for (int k = 0; k < K; k++) {  // all plans first: a new plan may regrow the partials
        nf_status st = get_plan(ctx, box, b[k], b[k + 1], &pls[k]);
        if (st != NF_OK) return st;
    }
    for (int k = 0; k < K; k++) {
        nf_status st = ensure_graph(ctx, box, *pls[k]);
        if (st != NF_OK) return st;
    }
    OrderScratch o;
    nf_status ost = upload_scratch(ctx, box, o);
    if (ost != NF_OK) return ost;
    if (!box->s_in) NF_CUDA(cudaStreamCreateWithFlags(&box->s_in, cudaStreamNonBlocking));
    if (!box->s_out) NF_CUDA(cudaStreamCreateWithFlags(&box->s_out, cudaStreamNonBlocking));
    while ((int)box->step_ev.size() < 2 * K + 2) {
        cudaEvent_t e;
        NF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        box->step_ev.push_back(e);
    }
    cudaEvent_t *ev_in = box->step_ev.data(), *ev_out = ev_in + K, ev_go = ev_in[2 * K],
                ev_done = ev_in[2 * K + 1];
    cudaStream_t sc = ctx->stream, si = box->s_in, so = box->s_out;
    const int64_t c2 = (int64_t)cpd * cpd, n = box->np;
    auto P = [&](int slab) { return box->cell_start[(int64_t)slab * c2]; };
    const size_t rec = ctx->cfg.out_kind == NF_OUT_FLOAT4 ? 16 : 12;
    float *tmp = box->d_stage;
    // copies in on s_in, ordering and sweeps on the context stream, copies
    // out on s_out; the context stream waits for both at the end
    NF_CUDA(cudaEventRecord(ev_go, sc));
    NF_CUDA(cudaStreamWaitEvent(si, ev_go, 0));
    NF_CUDA(cudaStreamWaitEvent(so, ev_go, 0));
    for (int k = 0; k < K; k++) {
        const int64_t p0 = P(b[k]), m = P(b[k + 1]) - p0;
        if (m > 0) {
            const size_t by = (size_t)m * sizeof(float);
            NF_CUDA(cudaMemcpyAsync(tmp + p0, x + p0, by, cudaMemcpyDefault, si));
            NF_CUDA(cudaMemcpyAsync(tmp + n + p0, y + p0, by, cudaMemcpyDefault, si));
            NF_CUDA(cudaMemcpyAsync(tmp + 2 * n + p0, z + p0, by, cudaMemcpyDefault, si));
        }
        NF_CUDA(cudaEventRecord(ev_in[k], si));
    }
    auto sweep = [&](int k) -> nf_status {
        // range k: its halo chunks are ordered already (stream order on sc)
        NF_CUDA(cudaGraphLaunch(pls[k]->graph, sc));
        NF_CUDA(cudaEventRecord(ev_out[k], sc));
        NF_CUDA(cudaStreamWaitEvent(so, ev_out[k], 0));
        if (pls[k]->out_bytes)
            NF_CUDA(cudaMemcpyAsync((char *)out + (size_t)(P(b[k]) - P(0)) * rec, pls[k]->d_out,
                                    pls[k]->out_bytes, cudaMemcpyDefault, so));
        return NF_OK;
    };
    for (int k = 0; k < K; k++) {
        NF_CUDA(cudaStreamWaitEvent(sc, ev_in[k], 0));
        cudaError_t e = order_range(ctx, box, o, tmp, tmp + n, tmp + 2 * n, 1, P(b[k]),
                                    P(b[k + 1]), sc);
        if (e != cudaSuccess) return cuda_fail(e, "nf_box_step (ordering)");
        if (k >= 2) {  // range k-1 has both halos: chunks k-2 and k
            nf_status st = sweep(k - 1);
            if (st != NF_OK) return st;
        }
    }
    // the ranges next to the periodic wrap need the last chunk
    if (K >= 2) {
        nf_status st = sweep(K - 1);
        if (st != NF_OK) return st;
    }
    nf_status st = sweep(0);
    if (st != NF_OK) return st;
    NF_CUDA(cudaEventRecord(ev_done, so));
    NF_CUDA(cudaStreamWaitEvent(sc, ev_done, 0));
    NF_CUDA(cudaStreamSynchronize(sc));
    uint64_t pairs = 0, padded = 0;
    for (Plan *pl : pls) {
        pairs += pl->pairs;
        padded += pl->padded_pairs;
    }
    ctx->last.pairs = pairs;
    ctx->last.padded_pairs = padded;
    ctx->last.launches = 2 * K;
    return NF_OK;
}

// ------------------------------------------------------------------------
// Allocation-free entry point (nf_forces_noalloc)
//
// For callers that cannot allocate device memory: code running where
// cudaMalloc is off limits (inside another framework's memory pool, a
// caching allocator that owns the device, or a context whose allocations
// are frozen after start-up).  The caller passes device inputs and outputs;
// the only scratch is the file-scope array below, which every GPU that loads
// this library holds until the process exits.
// ------------------------------------------------------------------------
namespace nf {

constexpr int64_t NOALLOC_MAX_SINKS = 196608;             // particles per call
constexpr size_t NOALLOC_SCRATCH_BYTES = (size_t)32 << 20;  // 32 MiB
constexpr size_t NOALLOC_COUNTER_BYTES = 256;
static_assert(NOALLOC_COUNTER_BYTES + (size_t)MAXW * 4 * sizeof(Partial) * NOALLOC_MAX_SINKS <=
                  NOALLOC_SCRATCH_BYTES,
              "scratch holds (2R+1) x 4 pencil partials per sink");
// [0, 256): work counters; then (2R+1) x nc x n pencil partials.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

// Warps take whole pencils from a counter and run their tiles in order.
template <int SOFT, bool DENS>
__global__ void __launch_bounds__(WARPS_PER_CTA * 32, 2)
    noalloc_pencil_kernel(KParams kp, int pencil0, int n_pencils) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    WarpSmem &ws = reinterpret_cast<WarpSmem *>(smem_raw)[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int W = 2 * kp.R + 1;
    for (;;) {
        int q = 0;
        if (lane == 0) q = atomicAdd(&kp.counters[1], 1);
        q = __shfl_sync(FULL, q, 0);
        if (q >= n_pencils) break;
        Item it{pencil0 + q, 0, 0, 4, 0, 0, 0, 0};
        setup_tables(kp, it, ws, lane);
        const int np_ = ws.spre[W];
        it.src_end = ws.cpre[W * W];
        for (int b = 0; b < np_; b += TILE_MAX) {
            it.sink_begin = b;
            it.nsink = min(TILE_MAX, np_ - b);
            if (it.nsink <= 32)
                run_tile<SOFT, DENS, 1, 8>(kp, ws, it, lane, nullptr, 0);
            else if (it.nsink <= 64)
                run_tile<SOFT, DENS, 2, 8>(kp, ws, it, lane, nullptr, 0);
            else
                run_tile<SOFT, DENS, 4, 8>(kp, ws, it, lane, nullptr, 0);
        }
    }
}

typedef void (*NoallocFn)(KParams, int, int);

static NoallocFn noalloc_kernel(int soft, bool dens) {
    switch (soft) {
    case SOFT_PLUMMER: return dens ? noalloc_pencil_kernel<SOFT_PLUMMER, true> : noalloc_pencil_kernel<SOFT_PLUMMER, false>;
    case SOFT_SINGLE_SPLINE:
        return dens ? noalloc_pencil_kernel<SOFT_SINGLE_SPLINE, true> : noalloc_pencil_kernel<SOFT_SINGLE_SPLINE, false>;
    case SOFT_CUBIC_SPLINE:
        return dens ? noalloc_pencil_kernel<SOFT_CUBIC_SPLINE, true> : noalloc_pencil_kernel<SOFT_CUBIC_SPLINE, false>;
    default:
        return dens ? noalloc_pencil_kernel<SOFT_CUBIC_PLUMMER, true> : noalloc_pencil_kernel<SOFT_CUBIC_PLUMMER, false>;
    }
}

static std::mutex g_noalloc_mu;
static void *g_noalloc_base[128];  // device address of the scratch, per device ordinal

}  // namespace nf

extern "C" nf_status nf_forces_noalloc(const nf_config *cfg, int cpd, const void *pos,
                                       const int64_t *cell_start, int slab_lo, int slab_hi,
                                       void *out, void *stream) {
    if (!cfg || !pos || !cell_start || !out) {
        set_error("nf_forces_noalloc: null argument");
        return NF_EINVAL;
    }
    const int R = cfg->near_field_radius;
    if (R < 1 || R > 2 || cpd < 2 * R + 1 || (cpd & 1) == 0 || slab_lo < 0 || slab_hi > cpd ||
        slab_lo >= slab_hi || cfg->softening < 0 || cfg->softening > 3 ||
        !std::isfinite(cfg->eps) || cfg->eps <= 0.f || !(cfg->b2 >= 0.f) ||
        (cfg->out_kind != NF_OUT_FLOAT3 && cfg->out_kind != NF_OUT_FLOAT4) ||
        (cfg->out_kind == NF_OUT_FLOAT3 && cfg->b2 > 0.f)) {
        set_error("nf_forces_noalloc: bad configuration or slab range");
        return NF_EINVAL;
    }
    if ((int64_t)cpd * cpd * cpd >= ((int64_t)1 << 31)) {
        // pencil ids (linear cell ids) are 32-bit in the work loop
        set_error("nf_forces_noalloc: cpd^3 must be below 2^31 (cpd <= 1290)");
        return NF_EINVAL;
    }
    cudaStream_t st = (cudaStream_t)stream;
    int dev = 0;
    NF_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 128) {
        set_error("nf_forces_noalloc: device ordinal beyond 127");
        return NF_EINVAL;
    }
    void *base = nullptr;
    {
        // once per device, with that device current: the array's device address
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_base[dev]) {
            void *p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess) return cuda_fail(e, "nf_forces_noalloc: cudaGetSymbolAddress");
            g_noalloc_base[dev] = p;
        }
        base = g_noalloc_base[dev];
    }
    const int64_t c2 = (int64_t)cpd * cpd;
    int64_t bounds[2] = {0, 0};
    NF_CUDA(cudaMemcpyAsync(&bounds[0], cell_start + slab_lo * c2, sizeof(int64_t),
                            cudaMemcpyDeviceToHost, st));
    NF_CUDA(cudaMemcpyAsync(&bounds[1], cell_start + slab_hi * c2, sizeof(int64_t),
                            cudaMemcpyDeviceToHost, st));
    NF_CUDA(cudaStreamSynchronize(st));
    const int64_t n = bounds[1] - bounds[0];
    if (n < 0 || n > NOALLOC_MAX_SINKS) {
        set_error("nf_forces_noalloc: at most 196608 particles in the requested slabs "
                  "(32 MiB static scratch)");
        return NF_EINVAL;
    }
    if (n == 0) return NF_OK;
    nf_ctx tmp;  // parameters only; no stream, event or memory of its own
    tmp.cfg = *cfg;
    tmp.device = dev;
    NF_CUDA(cudaDeviceGetAttribute(&tmp.sms, cudaDevAttrMultiProcessorCount, dev));
    NF_CUDA(cudaMemsetAsync(base, 0, NOALLOC_COUNTER_BYTES, st));
    EngineLaunch L;
    L.pos = (const float4 *)pos;
    L.cs = cell_start;
    L.cpd = cpd;
    L.counters = (int *)base;
    L.part = (Partial *)((char *)base + NOALLOC_COUNTER_BYTES);
    L.p0 = bounds[0];
    L.n_range = n;
    KParams kp = params_from(&tmp, L);
    NoallocFn fn = noalloc_kernel(cfg->softening, cfg->b2 > 0.f);
    const size_t smem = sizeof(WarpSmem) * WARPS_PER_CTA;
    int per_sm = 1;
    NF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)fn,
                                                          WARPS_PER_CTA * 32, smem));
    int pencil0 = (int)(slab_lo * c2), npen = (int)((slab_hi - slab_lo) * c2);
    void *args[] = {&kp, &pencil0, &npen};
    NF_CUDA(cudaLaunchKernel((const void *)fn, dim3(tmp.sms * std::max(per_sm, 1)),
                             dim3(WARPS_PER_CTA * 32), args, smem, st));
    coadd_kernel<<<tmp.sms * 8, 256, 0, st>>>(L.part, n, 2 * R + 1, kp.nc, output_scale(*cfg),
                                              cfg->out_kind, out, nullptr, 0);
    NF_CUDA(cudaGetLastError());
    return NF_OK;
}
