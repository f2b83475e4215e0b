// nf_sic.cu -- plain drop-in: GPU control and SetInteractionCollection execution.
//
// Replaces singlestep/Direct/GPUControl.cu (GPUSetup, GPUReset, the queue
// watchers) and PencilTask.cu (GPUPencilTask).  The contract kept from the
// reference: one SIC covers every sink z-pencil of rows [j_low, j_high) of
// one x-slab and the 2R+1 source slabs around it; after it completes, the
// caller's AccSlab rows [j_low, j_high) hold the near-field accelerations and
// the SIC's completion flag is set.  SICs are queued to worker threads, one
// per (GPU x buffers-per-device) buffer, each with its own stream.
//
// How a SIC runs here (B200-first, not the reference's pencil gather):
//   1. the SIC's source rows of the 2R+1 slabs (each particle once, rather
//      than the reference's five copies per pencil, PencilPlan.cc:22-90,
//      214-255) are packed into pinned staging and copied to the device;
//   2. a pack kernel builds float4 records, forming a "mini box" of 2R+1
//      slabs with the SIC's cell offsets;
//   3. one launch of the pencil engine (the reference's block shape: tiles of
//      64 sinks, in SIC order, no splitting, no graph) writes per-pencil
//      compensated FP32 partials, and the co-add kernel sums the 2R+1 pencils of each
//      sink on the device (PencilPlan.cc:140-207 co-adds on the host);
//   4. the rows' accelerations are copied back and stored into AccSlab.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>

#include "nf_internal.h"

namespace nf {

static_assert(ENGINE_WARPS_PER_CTA == 8, "engine CTA shape");

constexpr int NFBLOCK = 64;    // NFBlockSize (configure.ac:160-162)
constexpr int SPLIT_MIN_SOURCES = 64;  // sources per warp of a split tile (one staged chunk)
constexpr int REF_WIDTH = 5;   // WIDTH = 2*NFRADIUS+1, NFRADIUS = 2 (GPUControl.cu:109-113)

struct SicTask {
    nf_sic_desc d;  // shallow copy: the arrays stay owned by the caller
    int jlow = 0, jhigh = 0;
    volatile int *completion = nullptr;
};

struct SicBuffer {
    int index = 0, device = 0;
    bool pinned = true;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;  // around the pencil kernel of a SIC
    std::mutex mu;
    float *d_raw = nullptr;
    float4 *d_pos = nullptr;
    int64_t *d_cs = nullptr;
    Item *d_items = nullptr;
    Partial *d_part = nullptr;
    void *d_out = nullptr;
    int *d_counters = nullptr;
    float *h_raw = nullptr;
    void *h_out = nullptr;
    int64_t *h_cs = nullptr;
    Item *h_items = nullptr;
    size_t cap_particles = 0, cap_sinks = 0, cap_items = 0, cap_cells = 0;
};

static void host_free(void *p, bool pinned) {
    if (!p) return;
    if (pinned)
        cudaFreeHost(p);
    else
        free(p);
}

static cudaError_t host_alloc(void **p, size_t bytes, bool pinned, bool wc) {
    if (pinned) return cudaHostAlloc(p, bytes, wc ? cudaHostAllocWriteCombined : cudaHostAllocDefault);
    *p = aligned_alloc(4096, (bytes + 4095) / 4096 * 4096);
    return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}

static void release(SicBuffer &b) {
    cudaSetDevice(b.device);
    cudaFree(b.d_raw);
    cudaFree(b.d_pos);
    cudaFree(b.d_cs);
    cudaFree(b.d_items);
    cudaFree(b.d_part);
    cudaFree(b.d_out);
    cudaFree(b.d_counters);
    host_free(b.h_raw, b.pinned);
    host_free(b.h_out, b.pinned);
    host_free(b.h_cs, b.pinned);
    host_free(b.h_items, b.pinned);
    if (b.stream) cudaStreamDestroy(b.stream);
    if (b.ev0) cudaEventDestroy(b.ev0);
    if (b.ev1) cudaEventDestroy(b.ev1);
    b.ev0 = b.ev1 = nullptr;
    b.d_raw = nullptr;
    b.d_pos = nullptr;
    b.d_cs = nullptr;
    b.d_items = nullptr;
    b.d_part = nullptr;
    b.d_out = nullptr;
    b.d_counters = nullptr;
    b.h_raw = nullptr;
    b.h_out = nullptr;
    b.h_cs = nullptr;
    b.h_items = nullptr;
    b.stream = nullptr;
    b.cap_particles = b.cap_sinks = b.cap_items = b.cap_cells = 0;
}

// Grow a buffer's arrays to hold a task (1.25x headroom; never shrinks).
static nf_status grow(nf_ctx *ctx, SicBuffer &b, size_t particles, size_t sinks, size_t items,
                      size_t cells) {
    const int W = 2 * ctx->cfg.near_field_radius + 1;
    const int nc = ctx->cfg.b2 > 0.f ? 4 : 3;
    const size_t rec = ctx->cfg.out_kind == NF_OUT_FLOAT4 ? 16 : 12;
    auto up = [](size_t n) { return n + n / 4 + 1024; };
    if (particles > b.cap_particles) {
        size_t c = up(particles);
        cudaFree(b.d_raw);
        cudaFree(b.d_pos);
        host_free(b.h_raw, b.pinned);
        b.d_raw = nullptr;
        b.d_pos = nullptr;
        b.h_raw = nullptr;
        b.cap_particles = 0;
        NF_CUDA(cudaMalloc(&b.d_raw, 3 * c * sizeof(float)));
        NF_CUDA(cudaMalloc(&b.d_pos, c * sizeof(float4)));
        NF_CUDA(host_alloc((void **)&b.h_raw, 3 * c * sizeof(float), b.pinned, true));
        b.cap_particles = c;
    }
    if (sinks > b.cap_sinks) {
        size_t c = up(sinks);
        cudaFree(b.d_part);
        cudaFree(b.d_out);
        host_free(b.h_out, b.pinned);
        b.d_part = nullptr;
        b.d_out = nullptr;
        b.h_out = nullptr;
        b.cap_sinks = 0;
        NF_CUDA(cudaMalloc(&b.d_part, (size_t)W * nc * c * sizeof(Partial)));
        NF_CUDA(cudaMalloc(&b.d_out, c * rec));
        NF_CUDA(host_alloc(&b.h_out, c * rec, b.pinned, false));
        b.cap_sinks = c;
    }
    if (items > b.cap_items) {
        size_t c = up(items);
        cudaFree(b.d_items);
        host_free(b.h_items, b.pinned);
        b.d_items = nullptr;
        b.h_items = nullptr;
        b.cap_items = 0;
        NF_CUDA(cudaMalloc(&b.d_items, c * sizeof(Item)));
        NF_CUDA(host_alloc((void **)&b.h_items, c * sizeof(Item), b.pinned, true));
        b.cap_items = c;
    }
    if (cells > b.cap_cells) {
        size_t c = cells;
        cudaFree(b.d_cs);
        host_free(b.h_cs, b.pinned);
        b.d_cs = nullptr;
        b.h_cs = nullptr;
        b.cap_cells = 0;
        NF_CUDA(cudaMalloc(&b.d_cs, c * sizeof(int64_t)));
        NF_CUDA(host_alloc((void **)&b.h_cs, c * sizeof(int64_t), b.pinned, true));
        b.cap_cells = c;
    }
    if (!b.d_counters) NF_CUDA(cudaMalloc(&b.d_counters, 2 * sizeof(int)));
    return NF_OK;
}

static inline int wrapi(int i, int n) {
    i %= n;
    return i < 0 ? i + n : i;
}

// Validate the descriptor against the SIC geometry (the reference asserts
// the same sizes, PencilOnPencil.cc:221-236, 380-401).
static nf_status check_desc(nf_ctx *ctx, const nf_sic_desc &d, int jlow, int jhigh) {
    const int R = d.nfradius, W = 2 * R + 1;
    if (R != ctx->cfg.near_field_radius) {
        set_error("nf_sic_execute: nfradius differs from the context's near_field_radius");
        return NF_EINVAL;
    }
    const bool two_d = d.node_z_size > 0;
    if (d.cpd < W || (d.cpd & 1) == 0 || jlow < 0 || jhigh > d.cpd || jlow >= jhigh ||
        (!two_d && d.nk != d.cpd) ||
        (two_d && (d.nk != d.node_z_size + 2 * R || d.node_z_size + 2 * R > d.cpd ||
                   d.node_z_start < 0 || d.node_z_start >= d.cpd))) {
        set_error("nf_sic_execute: bad geometry (odd cpd >= 2R+1, 0 <= jlow < jhigh <= cpd, Nk == "
                  "cpd; 2D: Nk == node_z_size + 2R, node_z_size + 2R <= cpd)");
        return NF_EINVAL;
    }
    const int jw = jhigh - jlow;
    if (d.nsinksets != jw * d.nk || d.nsourcesets != d.nk * (jw + 2 * R) ||
        d.interaction_count != W * d.nsinksets) {
        set_error("nf_sic_execute: set counts do not match j_width, Nk and nfradius");
        return NF_EINVAL;
    }
    if (!d.sink_plan || !d.source_plan || !d.sink_pos_slab || !d.source_pos_slab ||
        !d.source_nslab || !d.sink_acc_slab || !d.sink_set_count || !d.source_set_count) {
        set_error("nf_sic_execute: null array in the descriptor");
        return NF_EINVAL;
    }
    if (d.interaction_list) {
        for (int j = 0; j < jw; j++)
            for (int k = 0; k < d.nk; k++)
                for (int y = 0; y < W; y++)
                    if (d.interaction_list[(j * d.nk + k) * W + y] != (j + y) * d.nk + k) {
                        set_error("nf_sic_execute: interaction list is not the pencil pattern");
                        return NF_EINVAL;
                    }
    }
    return NF_OK;
}

static uint64_t items_pairs(const std::vector<Item> &items) {
    uint64_t p = 0;
    for (const Item &it : items) p += (uint64_t)it.nsink * (uint64_t)(it.src_end - it.src_begin);
    return p;
}

static void sic_account(nf_ctx *ctx, float kernel_ms, uint64_t pairs);

static nf_status run_task(nf_ctx *ctx, SicBuffer &b, const SicTask &t) {
    const nf_sic_desc &d = t.d;
    nf_status st = check_desc(ctx, d, t.jlow, t.jhigh);
    if (st != NF_OK) return st;
    NF_CUDA(cudaSetDevice(b.device));
    const int R = d.nfradius, W = 2 * R + 1, cpd = d.cpd, nk = d.nk;
    const int jw = t.jhigh - t.jlow, nrows = jw + 2 * R;
    const int64_t ncell = (int64_t)W * cpd * cpd;
    // Pencil k of a row is centred on z = (k + R) mod cpd (index_to_zcen,
    // PencilOnPencil.cc:37-43, one z-domain per node); 2D: on node_z_start +
    // k + R, brought back by node_z_size + 2R past the upper ghost edge, so
    // the centres cover the primary cells and R ghost cells on each side.
    const bool two_d = d.node_z_size > 0;
    const int zs = d.node_z_start, zn = d.node_z_size;
    auto zcen = [&](int k) {
        if (!two_d) return (k + R) % cpd;
        int kk = k + zs + R;
        if (kk >= zs + zn + R) kk -= zn + 2 * R;
        return wrapi(kk, cpd);
    };
    auto primary = [&](int z) { return !two_d || wrapi(z - zs, cpd) < zn; };
    // cell counts of the mini box: slot s = source slab x-R+s, rows of the SIC
    std::vector<int64_t> cnt(ncell, 0), rowstart(W * cpd, -1), cellstart(two_d ? ncell : 0, -1);
    std::vector<char> row_used(cpd, 0);
    for (int r = 0; r < nrows; r++) {
        int y = wrapi(t.jlow - R + r, cpd);
        row_used[y] = 1;
        for (int k = 0; k < nk; k++) {
            int z = zcen(k);
            const nf_cell_plan *pl = d.source_plan + ((int64_t)r * nk + k) * W;
            for (int s = 0; s < W; s++) {
                if (pl[s].n < 0) {
                    set_error("nf_sic_execute: negative cell count");
                    return NF_EINVAL;
                }
                cnt[((int64_t)s * cpd + y) * cpd + z] = pl[s].n;
                if (two_d) cellstart[((int64_t)s * cpd + y) * cpd + z] = pl[s].start;
                else if (z == 0) rowstart[s * cpd + y] = pl[s].start;
            }
        }
    }
    // dense mirror offsets (linear cell order)
    size_t nitems = 0;
    NF_CUDA(cudaSetDevice(b.device));
    std::vector<int64_t> cs(ncell + 1, 0);
    for (int64_t c = 0; c < ncell; c++) cs[c + 1] = cs[c] + cnt[c];
    const int64_t n_mini = cs[ncell];
    const int64_t p0 = cs[((int64_t)R * cpd + t.jlow) * cpd];
    const int64_t p1 = cs[((int64_t)R * cpd + t.jhigh) * cpd];
    const int64_t n_sinks = p1 - p0;
    // work items: every sink pencil in tiles of 64 sinks (the reference block)
    std::vector<Item> items;
    items.reserve((size_t)d.nsinksets * 2);
    auto count = [&](int s, int y, int z) {
        return cnt[((int64_t)s * cpd + wrapi(y, cpd)) * cpd + wrapi(z, cpd)];
    };
    for (int j = 0; j < jw; j++)
        for (int k = 0; k < nk; k++) {
            int y = t.jlow + j, zc = zcen(k);
            // 2D: the primary cells of a pencil are contiguous in its sink
            // stream, after g_lo ghost sinks; only they are swept (the
            // reference truncates sink pencils the same way,
            // PencilPlan.cc:110-116)
            int64_t np_ = 0, g_lo = 0;
            bool seen_primary = false;
            for (int a = -R; a <= R; a++) {
                if (primary(zc + a)) {
                    np_ += count(R, y, zc + a);
                    seen_primary = true;
                } else if (!seen_primary) {
                    g_lo += count(R, y, zc + a);
                }
            }
            if (np_ != d.sink_set_count[j * nk + k]) {
                set_error("nf_sic_execute: SinkSetCount disagrees with the source plans");
                return NF_EINVAL;
            }
            if (np_ == 0) continue;
            int64_t M = 0;
            for (int dx = -R; dx <= R; dx++)
                for (int dy = -R; dy <= R; dy++) M += count(R + dx, y + dy, zc);
            int pencil = (int)(((int64_t)R * cpd + y) * cpd + zc);
            for (int64_t b0 = 0; b0 < np_; b0 += NFBLOCK) {
                int take = (int)std::min<int64_t>(NFBLOCK, np_ - b0);
                items.push_back(
                    Item{pencil, (int)(g_lo + b0), take, take <= 32 ? 1 : 2, 0, (int)M, 0, 0});
            }
        }
    // longest tiles first (the order of execution does not change any
    // result: every tile writes its own partials)
    std::stable_sort(items.begin(), items.end(), [](const Item &a, const Item &b) {
        return (int64_t)a.nsink * a.src_end > (int64_t)b.nsink * b.src_end;
    });
    // A SIC with fewer tiles than the launch has warps (small boxes, thin
    // y-splits) would leave most of the GPU idle: then every tile with at
    // least 64 sources per warp is split over the 8 warps of a CTA along its
    // source stream (summed in warp order in shared memory), the engine's
    // CTA-split path.  Launch order: split tiles, then the others.
    std::vector<Item> launch_items;
    int n_split = 0;
    {
        const int warps = engine_grid(ctx, engine_plain_variant()) * ENGINE_WARPS_PER_CTA;
        std::vector<Item> keep;
        if ((int64_t)items.size() < warps) {
            for (const Item &t : items) {
                const int M = t.src_end;
                if (M < SPLIT_MIN_SOURCES * ENGINE_WARPS_PER_CTA) {
                    keep.push_back(t);
                    continue;
                }
                const int per = ((M + ENGINE_WARPS_PER_CTA - 1) / ENGINE_WARPS_PER_CTA +
                                 SPLIT_MIN_SOURCES - 1) / SPLIT_MIN_SOURCES * SPLIT_MIN_SOURCES;
                for (int w = 0; w < ENGINE_WARPS_PER_CTA; w++) {
                    Item it = t;
                    it.src_begin = std::min(M, w * per);
                    it.src_end = std::min(M, (w + 1) * per);
                    launch_items.push_back(it);
                }
                n_split++;
            }
        } else {
            keep = items;
        }
        launch_items.insert(launch_items.end(), keep.begin(), keep.end());
    }
    nitems = launch_items.size();
    st = grow(ctx, b, (size_t)n_mini, (size_t)n_sinks, nitems, (size_t)ncell + 1);
    if (st != NF_OK) return st;
    // stage the source rows (each particle once) into pinned memory
    float *hx = b.h_raw, *hy = b.h_raw + b.cap_particles, *hz = b.h_raw + 2 * b.cap_particles;
    for (int s = 0; s < W; s++) {
        const float *slab = d.source_pos_slab[s];
        const uint64_t ns = d.source_nslab[s];
        // 2D: cell by cell (ghost cells included), cells that follow each
        // other in both the slab and the mini box copied as one run
        int64_t run_src = 0, run_dst = 0, run_n = 0;
        auto flush = [&]() {
            if (run_n == 0) return;
            memcpy(hx + run_dst, slab + run_src, run_n * sizeof(float));
            memcpy(hy + run_dst, slab + ns + run_src, run_n * sizeof(float));
            memcpy(hz + run_dst, slab + 2 * ns + run_src, run_n * sizeof(float));
            run_n = 0;
        };
        for (int y = 0; y < cpd && two_d; y++) {
            if (!row_used[y]) continue;
            for (int z = 0; z < cpd; z++) {
                const int64_t c = ((int64_t)s * cpd + y) * cpd + z;
                const int64_t n = cnt[c], src = cellstart[c], dst = cs[c];
                if (n == 0) continue;
                if (src < 0 || (uint64_t)(src + n) > ns) {
                    set_error("nf_sic_execute: source cell outside its slab");
                    return NF_EINVAL;
                }
                if (run_n > 0 && src == run_src + run_n && dst == run_dst + run_n) {
                    run_n += n;
                } else {
                    flush();
                    run_src = src;
                    run_dst = dst;
                    run_n = n;
                }
            }
        }
        flush();
        for (int y = 0; y < cpd && !two_d; y++) {
            if (!row_used[y]) continue;
            int64_t dst = cs[((int64_t)s * cpd + y) * cpd];
            int64_t n = cs[((int64_t)s * cpd + y + 1) * cpd] - dst;
            if (n == 0) continue;
            int64_t src = rowstart[s * cpd + y];
            if (src < 0 || (uint64_t)(src + n) > ns) {
                set_error("nf_sic_execute: source row outside its slab");
                return NF_EINVAL;
            }
            memcpy(hx + dst, slab + src, n * sizeof(float));
            memcpy(hy + dst, slab + ns + src, n * sizeof(float));
            memcpy(hz + dst, slab + 2 * ns + src, n * sizeof(float));
        }
    }
    memcpy(b.h_cs, cs.data(), cs.size() * sizeof(int64_t));
    if (nitems) memcpy(b.h_items, launch_items.data(), nitems * sizeof(Item));
    cudaStream_t sm = b.stream;
    size_t pb = (size_t)n_mini * sizeof(float);
    NF_CUDA(cudaMemcpyAsync(b.d_raw, hx, pb, cudaMemcpyHostToDevice, sm));
    NF_CUDA(cudaMemcpyAsync(b.d_raw + b.cap_particles, hy, pb, cudaMemcpyHostToDevice, sm));
    NF_CUDA(cudaMemcpyAsync(b.d_raw + 2 * b.cap_particles, hz, pb, cudaMemcpyHostToDevice, sm));
    NF_CUDA(cudaMemcpyAsync(b.d_cs, b.h_cs, cs.size() * sizeof(int64_t), cudaMemcpyHostToDevice, sm));
    if (nitems)
        NF_CUDA(cudaMemcpyAsync(b.d_items, b.h_items, nitems * sizeof(Item), cudaMemcpyHostToDevice, sm));
    st = engine_pack(ctx, b.d_raw, b.d_raw + b.cap_particles, b.d_raw + 2 * b.cap_particles, n_mini,
                     b.d_pos, sm);
    if (st != NF_OK) return st;
    EngineLaunch L;
    L.pos = b.d_pos;
    L.cs = b.d_cs;
    L.cpd = cpd;
    L.heavy = b.d_items;
    L.n_heavy_groups = n_split;
    L.light = b.d_items + (size_t)n_split * ENGINE_WARPS_PER_CTA;
    L.n_light = (int)nitems - n_split * ENGINE_WARPS_PER_CTA;
    L.counters = b.d_counters;
    L.part = b.d_part;
    L.p0 = p0;
    L.n_range = n_sinks;
    L.variant = engine_plain_variant();
    NF_CUDA(cudaEventRecord(b.ev0, sm));
    st = engine_launch(ctx, L, 1.0 / cpd, sm);
    if (st != NF_OK) return st;
    NF_CUDA(cudaEventRecord(b.ev1, sm));
    st = engine_coadd(ctx, b.d_part, n_sinks, b.d_out, sm);
    if (st != NF_OK) return st;
    const size_t rec = ctx->cfg.out_kind == NF_OUT_FLOAT4 ? 16 : 12;
    NF_CUDA(cudaMemcpyAsync(b.h_out, b.d_out, (size_t)n_sinks * rec, cudaMemcpyDeviceToHost, sm));
    NF_CUDA(cudaStreamSynchronize(sm));
    float kms = 0.f;
    NF_CUDA(cudaEventElapsedTime(&kms, b.ev0, b.ev1));
    sic_account(ctx, kms, items_pairs(items));
    if (two_d) {
        // primary cells only, each at its AccSlab start (the centre cell of
        // the pencil centred on it); cells adjacent in both go as one run
        size_t run_acc = 0, run_out = 0, run_bytes = 0;
        auto flush = [&]() {
            if (run_bytes)
                memcpy((char *)d.sink_acc_slab + run_acc, (char *)b.h_out + run_out, run_bytes);
            run_bytes = 0;
        };
        for (int j = 0; j < jw; j++)
            for (int k = 0; k < nk; k++) {
                const int y = t.jlow + j, zc = zcen(k);
                if (!primary(zc)) continue;
                const nf_cell_plan &ce = d.sink_plan[((int64_t)j * nk + k) * W + R];
                const int64_t c = ((int64_t)R * cpd + y) * cpd + zc;
                if (ce.n != cnt[c]) {
                    set_error("nf_sic_execute: sink plan and source plan disagree on a cell");
                    return NF_EINVAL;
                }
                if (ce.n == 0) continue;
                const size_t acc = (size_t)ce.start * rec, out = (size_t)(cs[c] - p0) * rec;
                const size_t bytes = (size_t)ce.n * rec;
                if (run_bytes && acc == run_acc + run_bytes && out == run_out + run_bytes) {
                    run_bytes += bytes;
                } else {
                    flush();
                    run_acc = acc;
                    run_out = out;
                    run_bytes = bytes;
                }
            }
        flush();
    } else if (n_sinks > 0) {
        // AccSlab rows [jlow, jhigh) are contiguous from the first sink cell of row jlow
        // the centre cell of the row-jlow pencil centred on z = 0 is cell (jlow, 0)
        int k0 = (cpd - R) % cpd;
        int64_t acc0 = d.sink_plan[(int64_t)k0 * W + R].start;
        memcpy((char *)d.sink_acc_slab + acc0 * rec, b.h_out, (size_t)n_sinks * rec);
    }
    if (d.bytes_to_device)
        *d.bytes_to_device += 3 * pb + cs.size() * sizeof(int64_t) + nitems * sizeof(Item);
    if (d.bytes_from_device) *d.bytes_from_device += (size_t)n_sinks * rec;
    return NF_OK;
}

}  // namespace nf

using namespace nf;

struct nf_ctx::Sic {
    std::vector<std::unique_ptr<SicBuffer>> buffers;
    std::deque<SicTask> queue;
    std::mutex mu;
    std::condition_variable cv, idle;
    bool stop = false;
    int active = 0;
    std::vector<std::thread> workers;
    nf_gpu_limits limits{};
    int cpd = 0;
    std::string error;  // first failure seen by a worker
    // pencil-kernel time of completed SICs (CUDA events around each launch)
    double kernel_ms = 0.0;
    uint64_t sics = 0, pairs = 0;
};

void nf::sic_account(nf_ctx *ctx, float kernel_ms, uint64_t pairs) {
    std::lock_guard<std::mutex> lk(ctx->sic->mu);
    ctx->sic->kernel_ms += kernel_ms;
    ctx->sic->sics++;
    ctx->sic->pairs += pairs;
}

static void finish(nf_ctx *ctx, const SicTask &t, nf_status st) {
    if (st != NF_OK) {
        std::lock_guard<std::mutex> lk(ctx->sic->mu);
        if (ctx->sic->error.empty()) ctx->sic->error = nf_last_error();
    }
    __atomic_store_n((int *)t.completion, st == NF_OK ? 1 : -1, __ATOMIC_RELEASE);
}

static void worker_main(nf_ctx *ctx, SicBuffer *b) {
    cudaSetDevice(b->device);
    auto *S = ctx->sic;
    for (;;) {
        SicTask t;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cv.wait(lk, [&] { return S->stop || !S->queue.empty(); });
            if (S->queue.empty()) break;  // stop requested and drained
            t = S->queue.front();
            S->queue.pop_front();
            S->active++;
        }
        nf_status st;
        {
            std::lock_guard<std::mutex> bl(b->mu);
            st = run_task(ctx, *b, t);
        }
        finish(ctx, t, st);
        {
            std::lock_guard<std::mutex> lk(S->mu);
            S->active--;
        }
        S->idle.notify_all();
    }
}

void nf_sic_shutdown(nf_ctx *ctx) {
    if (!ctx || !ctx->sic) return;
    auto *S = ctx->sic;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
    }
    S->cv.notify_all();
    for (auto &th : S->workers)
        if (th.joinable()) th.join();
    for (auto &b : S->buffers) release(*b);
    delete S;
    ctx->sic = nullptr;
    cudaSetDevice(ctx->device);
}

// MaxSinkBlocks and friends from a buffer budget, GPUControl.cu:374-408:
// per sink block 64*accstruct bytes of default memory plus 64*3*FLOAT +
// (4+FLOAT)*WIDTH + 4 bytes of write-combined memory, plus WIDTH source
// blocks of 64*3*FLOAT + 8 bytes.
nf_status nf::sic_limits(int out_kind, int cpd, uint64_t max_buffer_bytes, nf_gpu_limits *lim) {
    const float acc_bytes = out_kind == NF_OUT_FLOAT4 ? 16.f : 12.f;
    float src_wc = sizeof(float) * 3 * NFBLOCK + 8.0f;
    float sink_wc = sizeof(float) * 3 * NFBLOCK + (4.0f + sizeof(float)) * REF_WIDTH + 4.0f;
    float sink_def = acc_bytes * NFBLOCK;
    float total = sink_def + sink_wc + REF_WIDTH * src_wc;
    double blocks = ((double)max_buffer_bytes - 1e5) / total;
    if (!(blocks >= 1.0) || blocks > (double)INT32_MAX / REF_WIDTH) {
        set_error("nf_gpu_setup: buffer budget out of range");
        return NF_EINVAL;
    }
    lim->max_sink_blocks = (int)blocks;
    lim->max_source_blocks = REF_WIDTH * lim->max_sink_blocks;
    lim->max_sink_size = (size_t)NFBLOCK * lim->max_sink_blocks;
    lim->max_source_size = (size_t)NFBLOCK * lim->max_source_blocks;
    lim->max_nsink = lim->max_sink_blocks;
    lim->max_nsource = lim->max_nsink;
    if (lim->max_nsink <= 2 * cpd || lim->max_nsource <= (2 + REF_WIDTH) * cpd) {
        set_error("nf_gpu_setup: MaxNSink too small for this cpd (GPUControl.cu:407-408)");
        return NF_EINVAL;
    }
    return NF_OK;
}

extern "C" nf_status nf_gpu_setup(nf_ctx *ctx, int cpd, uint64_t max_buffer_bytes, int ngpu,
                                  int buffers_per_device, int use_pinned, nf_gpu_limits *limits) {
    if (!ctx || !limits || ngpu < 1 || buffers_per_device < 1 || cpd < 1) {
        set_error("nf_gpu_setup: bad argument");
        return NF_EINVAL;
    }
    if (ctx->sic) {  // GPUSetup runs once (GPUControl.cu:364)
        *limits = ctx->sic->limits;
        return NF_OK;
    }
    int ndev = 0;
    nf_status st = nf_get_ngpu(&ndev);
    if (st != NF_OK) return st;
    if (ngpu > ndev) {
        set_error("nf_gpu_setup: more GPUs requested than present");
        return NF_EINVAL;
    }
    nf_gpu_limits lim{};
    st = sic_limits(ctx->cfg.out_kind, cpd, max_buffer_bytes, &lim);
    if (st != NF_OK) return st;
    auto *S = new nf_ctx::Sic;
    S->limits = lim;
    S->cpd = cpd;
    // UsePinnedGPUMemory < 0: pin when the problem is large (GPUControl.cu:431-432)
    bool pinned = use_pinned < 0 ? lim.max_sink_blocks >= 10000 : use_pinned != 0;
    ctx->sic = S;
    for (int g = 0; g < ngpu * buffers_per_device; g++) {
        auto b = std::make_unique<SicBuffer>();
        b->index = g;
        b->device = ngpu == 1 ? ctx->device : g % ngpu;
        b->pinned = pinned;
        cudaError_t e = cudaSetDevice(b->device);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreate(&b->ev0);
        if (e == cudaSuccess) e = cudaEventCreate(&b->ev1);
        if (e != cudaSuccess) {
            nf_status s2 = cuda_fail(e, "nf_gpu_setup");
            S->buffers.push_back(std::move(b));
            nf_sic_shutdown(ctx);
            return s2;
        }
        S->buffers.push_back(std::move(b));
    }
    for (auto &b : S->buffers) S->workers.emplace_back(worker_main, ctx, b.get());
    cudaSetDevice(ctx->device);
    *limits = lim;
    return NF_OK;
}

extern "C" nf_status nf_gpu_reset(nf_ctx *ctx) {
    if (!ctx) {
        set_error("nf_gpu_reset: null context");
        return NF_EINVAL;
    }
    nf_sic_shutdown(ctx);
    return NF_OK;
}

extern "C" nf_status nf_sic_execute(nf_ctx *ctx, const nf_sic_desc *sic, int jlow, int jhigh,
                                    int blocking, volatile int *completion) {
    if (!ctx || !sic || !completion) {
        set_error("nf_sic_execute: null argument");
        return NF_EINVAL;
    }
    if (!ctx->sic) {
        set_error("nf_sic_execute: nf_gpu_setup has not run");
        return NF_EINVAL;
    }
    nf_status st = check_desc(ctx, *sic, jlow, jhigh);
    if (st != NF_OK) return st;
    SicTask t;
    t.d = *sic;
    t.jlow = jlow;
    t.jhigh = jhigh;
    t.completion = completion;
    *completion = 0;
    if (blocking) {  // GPUExecute(blocking=1) runs on the caller's thread, buffer 0
        SicBuffer &b = *ctx->sic->buffers[0];
        {
            std::lock_guard<std::mutex> bl(b.mu);
            st = run_task(ctx, b, t);
        }
        finish(ctx, t, st);
        cudaSetDevice(ctx->device);
        return st;
    }
    {
        std::lock_guard<std::mutex> lk(ctx->sic->mu);
        ctx->sic->queue.push_back(t);
    }
    ctx->sic->cv.notify_one();
    return NF_OK;
}

extern "C" nf_status nf_sic_drain(nf_ctx *ctx, uint64_t timeout_ns) {
    if (!ctx) {
        set_error("nf_sic_drain: null context");
        return NF_EINVAL;
    }
    if (!ctx->sic) return NF_OK;
    auto *S = ctx->sic;
    std::unique_lock<std::mutex> lk(S->mu);
    bool ok = S->idle.wait_for(lk, std::chrono::nanoseconds(timeout_ns),
                               [&] { return S->queue.empty() && S->active == 0; });
    if (!ok) {
        set_error("nf_sic_drain: SICs still in flight at the timeout");
        return NF_ETIMEDOUT;
    }
    if (!S->error.empty()) {
        set_error(S->error);
        S->error.clear();
        return NF_EDEVICE;
    }
    return NF_OK;
}

extern "C" nf_status nf_sic_timing(nf_ctx *ctx, double *kernel_ms, uint64_t *sics,
                                   uint64_t *pairs, int reset) {
    if (!ctx) {
        set_error("nf_sic_timing: null context");
        return NF_EINVAL;
    }
    double ms = 0.0;
    uint64_t n = 0, p = 0;
    if (ctx->sic) {
        std::lock_guard<std::mutex> lk(ctx->sic->mu);
        ms = ctx->sic->kernel_ms;
        n = ctx->sic->sics;
        p = ctx->sic->pairs;
        if (reset) {
            ctx->sic->kernel_ms = 0.0;
            ctx->sic->sics = ctx->sic->pairs = 0;
        }
    }
    if (kernel_ms) *kernel_ms = ms;
    if (sics) *sics = n;
    if (pairs) *pairs = p;
    return NF_OK;
}
