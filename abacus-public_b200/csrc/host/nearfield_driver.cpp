// nearfield_driver.cpp -- host side of the plain drop-in.
//
// NearFieldDriver (singlestep/Timestep/directdriver.cpp:22-532) and
// SetInteractionCollection (singlestep/Direct/SetInteractionCollection.hh:
// 171-283, planner PencilOnPencil.cc:180-418, pencil plans PencilPlan.cc:
// 95-138, 260-279) with the reference's method surface, written over the
// library's C ABI.  The reference reads the simulation state through global
// singletons (CP cell info, SB slab buffers, SS slab sizes, P parameters);
// here the caller registers one view per slab (nf_slab_view) and the driver
// reads those.  Differences by design: no CPU fallback (ForceCPU and
// CheckGPUCPU live in the test oracle, not in the product), SIC arrays owned
// by the SIC instead of a slab arena.  The MPI 2D z-split is the
// node_z_start / node_z_size pair of nf_driver_params (the reference's
// globals of the same names).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "nf_capi.h"
#include "nf_internal.h"

namespace nfd {

constexpr int NFBlockSize = 64;  // configure.ac:160-162
constexpr int NFRADIUS = 2;      // configure.ac:155-157 (sizes the buffers)
constexpr int MAXSPLITS = 1024;  // directdriver.cpp:276, 297

using clock_t_ = std::chrono::steady_clock;

// Accumulating wall-clock timer (include/STimer.h).
struct STimer {
    double elapsed = 0;
    clock_t_::time_point t0;
    bool on = false;
    void Start() {
        t0 = clock_t_::now();
        on = true;
    }
    void Stop() {
        if (on) elapsed += std::chrono::duration<double>(clock_t_::now() - t0).count();
        on = false;
    }
};

// The caller's slabs (replaces CP / SB / SS lookups).
struct SlabEnv {
    int cpd = 0, R = 2;
    int zs = 0, zn = 0;  // 2D z-split node (zn = 0: one z-domain)
    std::vector<nf_slab_view> slabs;
    std::vector<char> present;
    int wrap(int i) const {
        i %= cpd;
        return i < 0 ? i + cpd : i;
    }
    const nf_cellinfo &cell(int x, int y, int z) const {
        return slabs[wrap(x)].cellinfo[(size_t)wrap(y) * cpd + wrap(z)];
    }
    // NumParticlesInSkewer (PencilOnPencil.cc:90-109): particles of row j
    // (2D: of the node's z range, ghost cells included for sources).
    uint64_t skewer(int slab, int j, bool ghost) const {
        if (zn > 0) {
            uint64_t n = 0;
            const int pad = ghost ? R : 0;
            for (int z = zs - pad; z < zs + zn + pad; z++) n += (uint64_t)cell(slab, j, z).count;
            return n;
        }
        const nf_slab_view &v = slabs[wrap(slab)];
        const nf_cellinfo &c0 = v.cellinfo[(size_t)j * cpd];
        uint64_t start = ghost ? c0.startindex_with_ghost : c0.startindex;
        uint64_t end;
        if (j < cpd - 1) {
            const nf_cellinfo &c1 = v.cellinfo[(size_t)(j + 1) * cpd];
            end = ghost ? c1.startindex_with_ghost : c1.startindex;
        } else {
            end = v.nslab;
        }
        return end - start;
    }
};

class SetInteractionCollection {
  public:
    STimer DeviceThreadTimer;
    uint64_t bytes_to_device = 0, bytes_from_device = 0;

    std::vector<int32_t> SinkSetStart, SinkSetCount;
    std::vector<uint32_t> SinkSetIdMax;
    std::vector<nf_cell_plan> SinkPlan;  // [NSinkSets][nfwidth]
    std::vector<int32_t> SinkWrapcell;
    std::vector<int32_t> SourceSetStart, SourceSetCount;
    std::vector<nf_cell_plan> SourcePlan;  // [NSourceSets][nfwidth]
    std::vector<int32_t> SinkBlockParentPencil;
    std::vector<int32_t> SinkSourceInteractionList;
    std::vector<float> SinkSourceYOffset;

    float b2 = 0;
    volatile int CompletionFlag = 0;
    int SlabId = 0, k_low = 0, k_high = 0, Nk = 0, j_low = 0, j_high = 0, j_width = 0;
    int cpd = 0, nfradius = 0, nfwidth = 0;
    int InteractionCount = 0, NSinkBlocks = 0, NSourceBlocks = 0, NSinkSets = 0,
        NSourceSets = 0;
    uint64_t DirectTotal = 0, SinkTotal = 0, SourceTotal = 0, PaddedDirectTotal = 0,
             PaddedSinkTotal = 0, PaddedSourceTotal = 0;
    nf_status status = NF_OK;  // planning outcome (the reference asserts instead)

    // The constructor is the planner.
    SetInteractionCollection(const SlabEnv &env, const nf_gpu_limits &lim, int slab, int jlow,
                             int jhigh, float _b2, int NearFieldRadius);

    // GPUExecute (GPUControl.cu:235-261): hand the SIC to the library.
    nf_status GPUExecute(nf_ctx *ctx, const SlabEnv &env, int blocking);
    int CheckCompletion() const { return __atomic_load_n((int *)&CompletionFlag, __ATOMIC_ACQUIRE); }
    void SetCompleted() { __atomic_store_n((int *)&CompletionFlag, 1, __ATOMIC_RELEASE); }

    int NumPaddedBlocks(int n) const { return (n + NFBlockSize - 1) / NFBlockSize; }
    int PaddedSinkCount(int i) const { return NFBlockSize * NumPaddedBlocks(SinkSetCount[i]); }
    // index_to_zcen (PencilOnPencil.cc:37-43): the first pencil is the
    // first whose cells all lie in the primary range; 2D pencils also centre
    // on the R ghost cells each side (no z wrap).
    int index_to_zcen(int k) const {
        int kk = k + k_low + nfradius;
        const int pad = twoD ? nfradius : 0;
        if (kk >= k_high + pad) kk -= (k_high - k_low) + 2 * pad;
        return kk;
    }
    bool twoD = false;

  private:
    nf_sic_desc desc_{};
    std::vector<const float *> src_slabs_;
    std::vector<uint64_t> src_nslab_;
    nf_status fail(const char *msg) {
        nf::set_error(msg);
        status = NF_EINVAL;
        return status;
    }
};

SetInteractionCollection::SetInteractionCollection(const SlabEnv &env, const nf_gpu_limits &lim,
                                                   int slab, int jlow, int jhigh, float _b2,
                                                   int NearFieldRadius) {
    b2 = _b2;
    j_low = jlow;
    j_high = jhigh;
    cpd = env.cpd;
    SlabId = slab;
    nfradius = NearFieldRadius;
    nfwidth = 2 * NearFieldRadius + 1;
    j_width = j_high - j_low;
    // k_low, k_high: the node's primary sink cells (PencilOnPencil.cc:200-204)
    twoD = env.zn > 0;
    k_low = twoD ? env.zs : 0;
    k_high = twoD ? env.zs + env.zn : cpd;
    Nk = twoD ? k_high - k_low + nfwidth - 1 : k_high - k_low;
    const int W = nfwidth;
    if ((uint64_t)j_width * Nk >= INT32_MAX) {
        fail("NSinkSets would overflow int32");
        return;
    }
    NSinkSets = j_width * Nk;
    NSourceSets = Nk * (j_width + nfwidth - 1);
    if (NSinkSets > lim.max_nsink || NSourceSets > lim.max_nsource ||
        NSourceSets > cpd * (cpd + nfwidth)) {
        fail("SIC larger than the GPU buffer limits (MaxNSink / MaxNSource)");
        return;
    }
    SinkSetStart.assign(NSinkSets, 0);
    SinkSetCount.assign(NSinkSets, 0);
    SinkSetIdMax.assign(NSinkSets, 0);
    SinkPlan.assign((size_t)NSinkSets * W, nf_cell_plan{0, 0});
    SinkWrapcell.assign(NSinkSets, 0);
    SourceSetStart.assign(NSourceSets, 0);
    SourceSetCount.assign(NSourceSets, 0);
    SourcePlan.assign((size_t)NSourceSets * W, nf_cell_plan{0, 0});

    // Sink pencils: cells (slab, y, zc-R .. zc+R); wrapcell = the cell where
    // z wraps or leaves the primary range; 2D pencils are truncated to the
    // primary cells (SinkPencilPlan::load, PencilPlan.cc:95-138).
    std::vector<uint64_t> skewer_blocks(j_width + nfwidth, 0);
    for (int j = 0; j < j_width; j++)
        for (int k = 0; k < Nk; k++) {
            int zmid = index_to_zcen(k);
            int si = j * Nk + k;
            int total = 0, wrapcell = 0;
            for (int c = 0; c < W; c++) {
                int zc = zmid + c - nfradius;
                if (twoD && env.wrap(zc - k_low) >= k_high - k_low) {
                    SinkPlan[(size_t)si * W + c] = nf_cell_plan{0, 0};  // no-op cell
                } else {
                    const nf_cellinfo &ci = env.cell(slab, j + j_low, zc);
                    SinkPlan[(size_t)si * W + c] = nf_cell_plan{(uint32_t)ci.startindex, ci.count};
                    total += ci.count;
                }
                if (env.wrap(zc - k_high) == 0 || env.wrap(zc) == k_low) wrapcell = c;
            }
            SinkWrapcell[si] = wrapcell;
            SinkSetCount[si] = total;
            SinkTotal += total;
            skewer_blocks[j] += NumPaddedBlocks(total);
        }
    // Padded block enumeration per y skewer (PencilOnPencil.cc:271-311).
    std::vector<uint64_t> start(j_width + nfwidth + 1, 0);
    for (int j = 0; j < j_width; j++) start[j + 1] = start[j] + skewer_blocks[j];
    if (start[j_width] * NFBlockSize >= INT32_MAX) {
        fail("padded sinks overflow int32");
        return;
    }
    NSinkBlocks = (int)start[j_width];
    if (NSinkBlocks > lim.max_sink_blocks) {
        fail("NSinkBlocks larger than MaxSinkBlocks");
        return;
    }
    SinkBlockParentPencil.assign(NSinkBlocks, 0);
    for (int j = 0; j < j_width; j++) {
        int block = (int)start[j];
        int padded = NFBlockSize * block;
        for (int k = 0; k < Nk; k++) {
            int si = j * Nk + k;
            SinkSetStart[si] = padded;
            SinkSetIdMax[si] = (uint32_t)(padded + SinkSetCount[si]);
            int nb = NumPaddedBlocks(SinkSetCount[si]);
            padded += nb * NFBlockSize;
            for (int b = block; b < block + nb; b++) SinkBlockParentPencil[b] = si;
            block += nb;
        }
    }
    PaddedSinkTotal = (uint64_t)NFBlockSize * NSinkBlocks;
    if (PaddedSinkTotal > lim.max_sink_size) {
        fail("NPaddedSinks larger than MaxSinkSize");
        return;
    }

    // Source pencils: rows j_low-R .. j_high+R-1, cells (slab-R .. slab+R, y, zc)
    // (SourcePencilPlan::load, PencilPlan.cc:260-279; ghost start indices).
    std::fill(skewer_blocks.begin(), skewer_blocks.end(), 0);
    for (int j = 0; j < j_width + nfwidth - 1; j++)
        for (int k = 0; k < Nk; k++) {
            int zmid = index_to_zcen(k);
            int si = j * Nk + k;
            int total = 0;
            for (int c = 0; c < W; c++) {
                const nf_cellinfo &ci = env.cell(slab + c - W / 2, j + j_low - nfradius, zmid);
                SourcePlan[(size_t)si * W + c] =
                    nf_cell_plan{(uint32_t)ci.startindex_with_ghost, ci.count};
                total += ci.count;
            }
            SourceSetCount[si] = total;
            SourceTotal += total;
            skewer_blocks[j] += NumPaddedBlocks(total);
        }
    start[0] = 0;
    for (int j = 0; j < j_width + nfwidth - 1; j++) start[j + 1] = start[j] + skewer_blocks[j];
    if (start[j_width + nfwidth - 1] * NFBlockSize >= INT32_MAX) {
        fail("padded sources overflow int32");
        return;
    }
    NSourceBlocks = (int)start[j_width + nfwidth - 1];
    for (int j = 0; j < j_width + nfwidth - 1; j++) {
        int padded = NFBlockSize * (int)start[j];
        for (int k = 0; k < Nk; k++) {
            int si = j * Nk + k;
            SourceSetStart[si] = padded;
            padded += NumPaddedBlocks(SourceSetCount[si]) * NFBlockSize;
        }
    }
    PaddedSourceTotal = (uint64_t)NFBlockSize * NSourceBlocks;
    if (PaddedSourceTotal > lim.max_source_size) {
        fail("NPaddedSources larger than MaxSourceSize");
        return;
    }

    // Interactions: sink pencil (j, k) meets source pencils (j + y, k),
    // y = 0 .. 2R, shifted in y by (y - R) cells (PencilOnPencil.cc:380-416).
    InteractionCount = nfwidth * j_width * Nk;
    SinkSourceInteractionList.assign(InteractionCount, 0);
    SinkSourceYOffset.assign(InteractionCount, 0.f);
    const float cellsize = (float)(1.0 / cpd);
    for (int j = 0; j < j_width; j++)
        for (int k = 0; k < Nk; k++) {
            int si = j * Nk + k;
            int l = nfwidth * si;
            for (int y = 0; y < nfwidth; y++) {
                int src = (j + y) * Nk + k;
                SinkSourceInteractionList[l + y] = src;
                SinkSourceYOffset[l + y] = (float)(y - nfradius) * cellsize;
                DirectTotal += (uint64_t)SinkSetCount[si] * (uint64_t)SourceSetCount[src];
                PaddedDirectTotal += (uint64_t)PaddedSinkCount(si) * (uint64_t)SourceSetCount[src];
            }
        }
}

nf_status SetInteractionCollection::GPUExecute(nf_ctx *ctx, const SlabEnv &env, int blocking) {
    if (status != NF_OK) return status;
    const int W = nfwidth;
    src_slabs_.resize(W);
    src_nslab_.resize(W);
    for (int c = 0; c < W; c++) {
        const nf_slab_view &v = env.slabs[env.wrap(SlabId + c - nfradius)];
        src_slabs_[c] = v.posxyz;
        src_nslab_[c] = v.nslab;
    }
    const nf_slab_view &sv = env.slabs[env.wrap(SlabId)];
    nf_sic_desc &d = desc_;
    memset(&d, 0, sizeof(d));
    d.cpd = cpd;
    d.nfradius = nfradius;
    d.nk = Nk;
    d.nsinksets = NSinkSets;
    d.nsourcesets = NSourceSets;
    d.nsinkblocks = NSinkBlocks;
    d.nsourceblocks = NSourceBlocks;
    d.interaction_count = InteractionCount;
    d.sink_set_start = SinkSetStart.data();
    d.sink_set_count = SinkSetCount.data();
    d.sink_set_id_max = SinkSetIdMax.data();
    d.sink_plan = SinkPlan.data();
    d.sink_wrapcell = SinkWrapcell.data();
    d.sink_block_parent = SinkBlockParentPencil.data();
    d.source_set_start = SourceSetStart.data();
    d.source_set_count = SourceSetCount.data();
    d.source_plan = SourcePlan.data();
    d.interaction_list = SinkSourceInteractionList.data();
    d.y_offset = SinkSourceYOffset.data();
    d.sink_pos_slab = sv.posxyz;
    d.sink_nslab = sv.nslab;
    d.source_pos_slab = src_slabs_.data();
    d.source_nslab = src_nslab_.data();
    d.sink_acc_slab = sv.acc;
    d.b2 = b2;
    d.bytes_to_device = &bytes_to_device;
    d.bytes_from_device = &bytes_from_device;
    d.node_z_start = twoD ? k_low : 0;
    d.node_z_size = twoD ? k_high - k_low : 0;
    DeviceThreadTimer.Start();
    return nf_sic_execute(ctx, &d, j_low, j_high, blocking, &CompletionFlag);
}

struct SlabWork {
    std::vector<std::unique_ptr<SetInteractionCollection>> sics;
    int complete = 0;
};

class NearFieldDriver {
  public:
    NearFieldDriver(const nf_driver_params &p, nf_status *st);
    ~NearFieldDriver();

    nf_status ExecuteSlab(int slabID, int blocking);
    int SlabDone(int slabID);
    nf_status Finalize(int slabID);
    void AggregateStats();

    double SofteningLength = 0, SofteningLengthInternal = 0;
    float eps = 0;
    int NGPU = 0, DirectBPD = 1, NBuffers = 1;
    std::string GPUName;
    uint64_t TotalDirectInteractions_GPU = 0, TotalPaddedDirectInteractions_GPU = 0;
    double total_GB_to = 0, total_GB_from = 0, total_sinks = 0, total_sources = 0,
           total_padded_sinks = 0, total_padded_sources = 0, mean_splits_per_slab = 0;
    int MaxNSplits = 0;
    double GPUThroughputTime = 0;
    STimer CalcSplitDirects, SICConstruction, SICExecute, FinalizeTimer;

    SlabEnv env;
    nf_ctx *ctx = nullptr;
    nf_gpu_limits lim{};
    nf_driver_params params{};

  private:
    nf_status ExecuteSlabGPU(int slabID, int blocking);
    std::vector<SlabWork> work_;
    std::vector<int> SlabNSplit;
    int RADIUS = 2, WIDTH = 5, MinSplits = 1;
    // aggregated in Finalize
    uint64_t DirectInteractions_GPU = 0, PaddedDirectInteractions_GPU = 0;
    double GB_to_device = 0, GB_from_device = 0;
    uint64_t DeviceSinks = 0, DeviceSources = 0, PaddedDeviceSinks = 0, PaddedDeviceSources = 0;
    // wall time with at least one SIC in flight (GPUThroughputTimer)
    int inflight_slabs_ = 0;
    clock_t_::time_point busy_since_;
};

NearFieldDriver::NearFieldDriver(const nf_driver_params &p, nf_status *st) : params(p) {
    *st = NF_OK;
    RADIUS = p.near_field_radius;
    WIDTH = 2 * RADIUS + 1;
    SofteningLength = p.softening_length;
    // singlestep.cpp:113-125 internal lengths, directdriver.cpp:109-117 eps
    double f = p.softening == NF_SOFT_SINGLE_SPLINE ? 2.15517
               : p.softening == NF_SOFT_CUBIC_SPLINE ? 1.10064 : 1.0;
    SofteningLengthInternal = SofteningLength * f;
    double e = SofteningLengthInternal;
    switch (p.softening) {
    case NF_SOFT_CUBIC_SPLINE: eps = (float)(1. / e); break;
    case NF_SOFT_CUBIC_PLUMMER: eps = (float)(e * e * e); break;
    case NF_SOFT_SINGLE_SPLINE: eps = (float)(1. / (e * e)); break;
    default: eps = (float)(e * e); break;
    }
    if (!std::isfinite(eps) || eps <= 0.f) {
        nf::set_error("Infinite eps!  Softening length too small for this precision?");
        *st = NF_EINVAL;
        return;
    }
    if (RADIUS < 1 || RADIUS > NFRADIUS || p.cpd < WIDTH || (p.cpd & 1) == 0) {
        nf::set_error("nf_driver_create: need odd cpd >= 2R+1 and 1 <= R <= 2");
        *st = NF_EINVAL;
        return;
    }
    if (p.node_z_size < 0 || (p.node_z_size > 0 && (p.node_z_start < 0 || p.node_z_start >= p.cpd ||
                                                      p.node_z_size + 2 * RADIUS > p.cpd))) {
        nf::set_error("nf_driver_create: 2D node needs 0 <= node_z_start < cpd and "
                      "node_z_size + 2R <= cpd");
        *st = NF_EINVAL;
        return;
    }
    env.cpd = p.cpd;
    env.R = RADIUS;
    env.zs = p.node_z_size > 0 ? p.node_z_start : 0;
    env.zn = p.node_z_size;
    env.slabs.assign(p.cpd, nf_slab_view{nullptr, 0, nullptr, nullptr});
    env.present.assign(p.cpd, 0);
    work_.resize(p.cpd);
    SlabNSplit.assign(p.cpd, 0);
    DirectBPD = std::max(1, p.direct_bpd);
    const size_t accstruct = p.out_kind == NF_OUT_FLOAT4 ? 16 : 12;
    double mem = p.mem_per_gpu_buffer_gb * 1e9;
    if (p.device < 0) {  // planner only, no GPU
        NGPU = 1;
        NBuffers = DirectBPD;
        if (mem <= 0) mem = 1e9;
        GPUName = "none";
    } else {
        nf_status s = nf_get_ngpu(&NGPU);
        if (s != NF_OK) {
            *st = s;
            return;
        }
        NGPU = 1;  // one device per driver; run one driver per GPU
        NBuffers = NGPU * DirectBPD;
        size_t gpumem = 0;
        char name[256];
        s = nf_get_device_info(&gpumem, name, sizeof(name));
        if (s != NF_OK) {
            *st = s;
            return;
        }
        GPUName = name;
        if (mem <= 0) {  // directdriver.cpp:157-168
            double m = (double)gpumem / DirectBPD;
            m = std::min(m, 1. * p.np * accstruct * 3 * (2 * NFRADIUS + 1) / NBuffers * 1.3 * 2 + 4e6);
            if (p.max_ram_mb > 0) m = std::min(m, 0.05 / NBuffers * p.max_ram_mb * 1e6);
            mem = m;
        }
    }
    MinSplits = NBuffers;
    MaxNSplits = MinSplits;
    if (p.device < 0) {
        *st = nf::sic_limits(p.out_kind, p.cpd, (uint64_t)mem, &lim);
        return;
    }
    nf_config cfg;
    nf_config_default(&cfg);
    cfg.device = p.device;
    cfg.near_field_radius = RADIUS;
    cfg.softening = p.softening;
    cfg.eps = eps;
    cfg.b2 = p.density_kernel_rad2;
    cfg.accumulation = p.accumulation;
    cfg.out_kind = p.out_kind;
    *st = nf_init(&cfg, &ctx);
    if (*st != NF_OK) return;
    *st = nf_gpu_setup(ctx, p.cpd, (uint64_t)mem, NGPU, DirectBPD, p.use_pinned_gpu_memory, &lim);
}

NearFieldDriver::~NearFieldDriver() {
    if (ctx) {
        nf_sic_drain(ctx, 60ull * 1000000000ull);
        nf_gpu_reset(ctx);
        nf_shutdown(ctx);
    }
}

nf_status NearFieldDriver::ExecuteSlab(int slabID, int blocking) {
    // ForceCPU has no counterpart: the CPU direct is the test oracle only.
    return ExecuteSlabGPU(env.wrap(slabID), blocking);
}

nf_status NearFieldDriver::ExecuteSlabGPU(int slab, int blocking) {
    if (!ctx) {
        nf::set_error("ExecuteSlab: the driver was created without a GPU");
        return NF_EINVAL;
    }
    for (int c = -RADIUS; c <= RADIUS; c++)
        if (!env.present[env.wrap(slab + c)]) {
            nf::set_error("ExecuteSlab: slabs slab-R .. slab+R are not all registered");
            return NF_EINVAL;
        }
    if (!work_[slab].sics.empty()) {
        nf::set_error("ExecuteSlab: slab already in flight (Finalize it first)");
        return NF_EINVAL;
    }
    const int cpd = env.cpd;
    CalcSplitDirects.Start();
    // Worst-case blocks per y skewer (ComputeSinkBlocks / ComputeSourceBlocks,
    // PencilOnPencil.cc:113-126).
    std::vector<int> SinkBlocks(cpd), SourceBlocks(cpd);
    int64_t totSinkBlocks = 0;
    for (int j = 0; j < cpd; j++) {
        SinkBlocks[j] = (int)((2 * RADIUS + 1) * (env.skewer(slab, j, false) / NFBlockSize) + cpd);
        uint64_t np = 0;
        for (int c = -RADIUS; c <= RADIUS; c++) np += env.skewer(slab + c, j, true);
        SourceBlocks[j] = (int)(np / NFBlockSize + cpd);
        totSinkBlocks += SinkBlocks[j];
    }
    // Greedy y-splits, at least one per buffer (directdriver.cpp:266-307).
    int useMaxSink = (int)(totSinkBlocks / NBuffers);
    useMaxSink = (int)(useMaxSink * (1 + 1.1 * NBuffers / cpd));
    useMaxSink = std::min(useMaxSink, lim.max_sink_blocks);
    int useMaxSource = lim.max_source_blocks;
    std::vector<int> SplitPoint;
    int64_t thisSink = 0, thisSource = 0;
    int NSplit = 0;
    for (int j = 0; j < cpd; j++) {
        thisSink += SinkBlocks[j];
        thisSource += SourceBlocks[env.wrap(j + RADIUS)];
        if (j == 0 || thisSink > useMaxSink || thisSource > useMaxSource) {
            if (NSplit > 0) SplitPoint[NSplit - 1] = j;
            thisSink = SinkBlocks[j];
            thisSource = 0;
            for (int c = -RADIUS; c <= RADIUS; c++) thisSource += SourceBlocks[env.wrap(j - c)];
            NSplit++;
            SplitPoint.push_back(0);
            if (NSplit >= MAXSPLITS) {
                CalcSplitDirects.Stop();
                nf::set_error("ExecuteSlab: too many splits");
                return NF_EINVAL;
            }
        }
    }
    SplitPoint[NSplit - 1] = cpd;
    CalcSplitDirects.Stop();
    if (thisSink > lim.max_sink_blocks || thisSource > lim.max_source_blocks) {
        nf::set_error("Sinks or Sources of the last skewer overflow the maxima");
        return NF_EINVAL;
    }
    SlabNSplit[slab] = NSplit;
    MaxNSplits = std::max(MaxNSplits, NSplit);
    SlabWork &w = work_[slab];
    w.complete = 0;
    if (inflight_slabs_++ == 0) busy_since_ = clock_t_::now();
    for (int n = 0; n < NSplit; n++) {
        int jl = n > 0 ? SplitPoint[n - 1] : 0;
        int jh = SplitPoint[n];
        SICConstruction.Start();
        auto sic = std::make_unique<SetInteractionCollection>(env, lim, slab, jl, jh,
                                                              params.density_kernel_rad2, RADIUS);
        SICConstruction.Stop();
        if (sic->status != NF_OK) return sic->status;
        SICExecute.Start();
        nf_status st = sic->GPUExecute(ctx, env, blocking);
        SICExecute.Stop();
        w.sics.push_back(std::move(sic));
        if (st != NF_OK) return st;
    }
    return NF_OK;
}

int NearFieldDriver::SlabDone(int slab) {
    slab = env.wrap(slab);
    SlabWork &w = work_[slab];
    if (w.complete) return 1;
    if (w.sics.empty()) return 0;
    int done = 1;
    for (auto &s : w.sics) {
        int f = s->CheckCompletion();
        if (f < 0) return -1;
        done = done && f == 1;
    }
    if (done) {
        for (auto &s : w.sics) s->DeviceThreadTimer.Stop();
        w.complete = 1;
        if (--inflight_slabs_ == 0)
            GPUThroughputTime += std::chrono::duration<double>(clock_t_::now() - busy_since_).count();
    }
    return done;
}

nf_status NearFieldDriver::Finalize(int slab) {
    slab = env.wrap(slab);
    if (SlabDone(slab) != 1) {
        nf::set_error("Finalize called for a slab that is not complete");
        return NF_EINVAL;
    }
    FinalizeTimer.Start();
    for (auto &s : work_[slab].sics) {
        DirectInteractions_GPU += s->DirectTotal;
        PaddedDirectInteractions_GPU += s->PaddedDirectTotal;
        GB_to_device += s->bytes_to_device / 1e9;
        GB_from_device += s->bytes_from_device / 1e9;
        DeviceSinks += s->SinkTotal;
        DeviceSources += s->SourceTotal;
        PaddedDeviceSinks += s->PaddedSinkTotal;
        PaddedDeviceSources += s->PaddedSourceTotal;
    }
    work_[slab].sics.clear();
    work_[slab].complete = 0;
    FinalizeTimer.Stop();
    return NF_OK;
}

void NearFieldDriver::AggregateStats() {
    total_GB_to = GB_to_device;
    total_GB_from = GB_from_device;
    total_sinks = (double)DeviceSinks;
    total_sources = (double)DeviceSources;
    total_padded_sinks = (double)PaddedDeviceSinks;
    total_padded_sources = (double)PaddedDeviceSources;
    TotalDirectInteractions_GPU = DirectInteractions_GPU;
    TotalPaddedDirectInteractions_GPU = PaddedDirectInteractions_GPU;
    double s = 0;
    for (int n : SlabNSplit) s += n;
    mean_splits_per_slab = s / env.cpd;
}

}  // namespace nfd

struct nf_driver {
    std::unique_ptr<nfd::NearFieldDriver> d;
};

extern "C" nf_status nf_driver_create(const nf_driver_params *p, nf_driver **out) {
    if (!p || !out) {
        nf::set_error("nf_driver_create: null argument");
        return NF_EINVAL;
    }
    *out = nullptr;
    nf_status st = NF_OK;
    auto drv = std::make_unique<nf_driver>();
    drv->d = std::make_unique<nfd::NearFieldDriver>(*p, &st);
    if (st != NF_OK) return st;
    *out = drv.release();
    return NF_OK;
}

extern "C" nf_status nf_driver_set_slab(nf_driver *drv, int slab, const nf_slab_view *v) {
    if (!drv || !v || !v->posxyz || !v->cellinfo) {
        nf::set_error("nf_driver_set_slab: null argument");
        return NF_EINVAL;
    }
    auto &env = drv->d->env;
    if (slab < 0 || slab >= env.cpd) {
        nf::set_error("nf_driver_set_slab: slab out of range");
        return NF_EINVAL;
    }
    env.slabs[slab] = *v;
    env.present[slab] = 1;
    return NF_OK;
}

extern "C" nf_status nf_driver_execute_slab(nf_driver *drv, int slab, int blocking) {
    if (!drv) {
        nf::set_error("nf_driver_execute_slab: null driver");
        return NF_EINVAL;
    }
    return drv->d->ExecuteSlab(slab, blocking);
}

extern "C" int nf_driver_slab_done(nf_driver *drv, int slab) {
    return drv ? drv->d->SlabDone(slab) : -1;
}

extern "C" nf_status nf_driver_finalize(nf_driver *drv, int slab) {
    if (!drv) {
        nf::set_error("nf_driver_finalize: null driver");
        return NF_EINVAL;
    }
    return drv->d->Finalize(slab);
}

extern "C" nf_status nf_driver_aggregate_stats(nf_driver *drv, nf_driver_stats *s) {
    if (!drv || !s) {
        nf::set_error("nf_driver_aggregate_stats: null argument");
        return NF_EINVAL;
    }
    auto &d = *drv->d;
    d.AggregateStats();
    memset(s, 0, sizeof(*s));
    s->direct_interactions = d.TotalDirectInteractions_GPU;
    s->padded_direct_interactions = d.TotalPaddedDirectInteractions_GPU;
    s->gdi_gpu = d.TotalDirectInteractions_GPU / 1e9;
    s->gdi_padded_gpu = d.TotalPaddedDirectInteractions_GPU / 1e9;
    s->total_gb_to = d.total_GB_to;
    s->total_gb_from = d.total_GB_from;
    s->total_sinks = d.total_sinks;
    s->total_sources = d.total_sources;
    s->total_padded_sinks = d.total_padded_sinks;
    s->total_padded_sources = d.total_padded_sources;
    s->mean_splits_per_slab = d.mean_splits_per_slab;
    s->max_nsplits = d.MaxNSplits;
    s->gpu_throughput_time = d.GPUThroughputTime;
    s->calc_split_s = d.CalcSplitDirects.elapsed;
    s->sic_construction_s = d.SICConstruction.elapsed;
    s->sic_execute_s = d.SICExecute.elapsed;
    s->finalize_s = d.FinalizeTimer.elapsed;
    s->softening_length_internal = d.SofteningLengthInternal;
    s->eps = d.eps;
    s->ngpu = d.NGPU;
    s->nbuffers = d.NBuffers;
    s->max_sink_blocks = d.lim.max_sink_blocks;
    s->max_source_blocks = d.lim.max_source_blocks;
    return NF_OK;
}

extern "C" nf_ctx *nf_driver_context(nf_driver *drv) { return drv ? drv->d->ctx : nullptr; }

extern "C" void nf_driver_destroy(nf_driver *drv) { delete drv; }

extern "C" nf_status nf_driver_plan_sic(nf_driver *drv, int slab, int jlow, int jhigh,
                                        nf_sic_summary *sum, int32_t *sink_set_count,
                                        int32_t *sink_block_parent, int32_t *source_set_count) {
    if (!drv || !sum) {
        nf::set_error("nf_driver_plan_sic: null argument");
        return NF_EINVAL;
    }
    auto &d = *drv->d;
    const int R = d.params.near_field_radius;
    if (slab < 0 || slab >= d.env.cpd || jlow < 0 || jhigh > d.env.cpd || jlow >= jhigh) {
        nf::set_error("nf_driver_plan_sic: bad range");
        return NF_EINVAL;
    }
    for (int c = -R; c <= R; c++)
        if (!d.env.present[d.env.wrap(slab + c)]) {
            nf::set_error("nf_driver_plan_sic: slabs slab-R .. slab+R are not all registered");
            return NF_EINVAL;
        }
    nfd::SetInteractionCollection sic(d.env, d.lim, slab, jlow, jhigh, d.params.density_kernel_rad2, R);
    if (sic.status != NF_OK) return sic.status;
    sum->nsinksets = sic.NSinkSets;
    sum->nsourcesets = sic.NSourceSets;
    sum->nsinkblocks = sic.NSinkBlocks;
    sum->nsourceblocks = sic.NSourceBlocks;
    sum->interaction_count = sic.InteractionCount;
    sum->direct_total = sic.DirectTotal;
    sum->padded_direct_total = sic.PaddedDirectTotal;
    sum->sink_total = sic.SinkTotal;
    sum->source_total = sic.SourceTotal;
    sum->padded_sink_total = sic.PaddedSinkTotal;
    sum->padded_source_total = sic.PaddedSourceTotal;
    if (sink_set_count)
        memcpy(sink_set_count, sic.SinkSetCount.data(), sic.SinkSetCount.size() * sizeof(int32_t));
    if (sink_block_parent)
        memcpy(sink_block_parent, sic.SinkBlockParentPencil.data(),
               sic.SinkBlockParentPencil.size() * sizeof(int32_t));
    if (source_set_count)
        memcpy(source_set_count, sic.SourceSetCount.data(),
               sic.SourceSetCount.size() * sizeof(int32_t));
    return NF_OK;
}
