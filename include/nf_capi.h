/*
 * nf_capi.h -- C ABI of the B200 near-field direct-force library (libnfb200.so).
 *
 * The library computes the abacus near-field direct force: for every sink
 * particle, the softened pairwise acceleration from all particles in the
 * (2R+1)^3 = 5x5x5 neighbouring cells of a periodic box of cpd^3 cells, on
 * float32 positions stored relative to their cell centre.  Output units are
 * the reference's raw near-field output (a = -sum f(r) (src - sink), unit
 * masses; the single spline lacks its 1/eps^3 prefactor, which abacus applies
 * in the kick).
 *
 * Everything crossing this boundary is plain C: opaque handles, POD structs,
 * pointers and sizes, int status codes.  No C++ types, no CUDA runtime types
 * (streams are passed as void*, NULL = the library's own stream).
 *
 * Three layers, each mapped to the reference interface it replaces
 * (paths are within abacusorg/abacus-public):
 *
 *  1. GPU control: nf_get_ngpu / nf_get_device_info / nf_gpu_setup /
 *     nf_gpu_reset replace GetNGPU, GetDeviceInfo, GPUSetup and GPUReset
 *     (singlestep/Direct/GPUControl.cu:267-286, 357-482, 492-510;
 *     declared in singlestep/Direct/DeviceFunctions.h:8-26).
 *
 *  2. Plain drop-in: nf_sic_execute runs one SetInteractionCollection on the
 *     SIC's own pencil layout (the DeviceData arrays of
 *     singlestep/Direct/PencilTask.cu:28-45) and co-adds the pencil partials
 *     into the caller's AccSlab exactly like GPUPencilTask
 *     (PencilTask.cu:154-257, PencilPlan.cc:140-207).  It is what
 *     SetInteractionCollection::GPUExecute (GPUControl.cu:235-261) calls.
 *
 *  3. Batched / serving form: a box whose positions stay resident in HBM
 *     (nf_box_*), one persistent launch per slab range, and a continuous-
 *     batching request loop (nf_server_*).  These replace
 *     NearFieldDriver::ExecuteSlab / SlabDone
 *     (singlestep/Timestep/directdriver.cpp:242-431) for callers that keep
 *     positions on the device.
 */
#ifndef NF_CAPI_H
#define NF_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 2: nf_sic_desc and nf_driver_params end with node_z_start, node_z_size. */
#define NF_ABI_VERSION 2

/* ---------------- status codes ---------------- */
typedef int nf_status;
#define NF_OK 0
#define NF_EINVAL 1      /* bad argument, bad plan, size beyond a limit */
#define NF_ENOMEM 2      /* device or pinned allocation failed */
#define NF_EADMISSION 3  /* serving: request refused by the HBM admission gate */
#define NF_ETIMEDOUT 4   /* a bounded wait ran out */
#define NF_EDEVICE 5     /* a CUDA call failed; the message is in nf_last_error */
#define NF_ENODEV 6      /* no CUDA device */
#define NF_ENOTREADY 7   /* poll: work still in flight */
#define NF_ECANCELLED 8  /* serving: request cancelled or loop stopped */

/* ---------------- softening ---------------- */
/* Softening kernels of singlestep/Direct/DirectGPUKernels.cuh:20-174 and
 * DirectCPUKernels.cc:12-128, selected at run time instead of by
 * configure.ac --with-softening. */
#define NF_SOFT_PLUMMER 0
#define NF_SOFT_SINGLE_SPLINE 1 /* the reference default */
#define NF_SOFT_CUBIC_SPLINE 2
#define NF_SOFT_CUBIC_PLUMMER 3

/* accumulation of each sink's sum */
#define NF_ACC_COMPENSATED 0 /* FP32 chunk partials folded into a TwoSum (hi, lo) pair */
#define NF_ACC_PLAIN 1       /* FP32 chunk partials added into one FP32 running sum */

/* output record per particle (accstruct, singlestep/Direct/GPUControl.cu:134-139) */
#define NF_OUT_FLOAT3 0 /* x, y, z */
#define NF_OUT_FLOAT4 1 /* x, y, z, w (w = FOF density sum when b2 > 0, else 0) */

typedef struct nf_config {
    int device;             /* CUDA ordinal */
    int near_field_radius;  /* R; width 2R+1.  1 <= R <= 2 (NFRADIUS, configure.ac:155-157) */
    int softening;          /* NF_SOFT_* */
    float eps;              /* the reference's kernel parameter (directdriver.cpp:109-117):
                               Plummer eps^2, single spline 1/eps^2, cubic spline 1/eps,
                               cubic Plummer eps^3 */
    float b2;               /* FOF density radius^2 (WriteState.DensityKernelRad2); 0 = off */
    int accumulation;       /* NF_ACC_* */
    int out_kind;           /* NF_OUT_* */
    int sinks_per_lane;     /* 0 = tile shapes from the occupancy; else cap at 1, 2 or 4 */
    int kernel_variant;     /* -1 = autotuned per box; else a fixed kernel shape
                               0 .. nf_kernel_variant_count()-1 */
} nf_config;

typedef struct nf_ctx nf_ctx;
typedef struct nf_box nf_box;

/* Fill *cfg with defaults (device 0, R 2, single spline, compensated, float4,
 * autotuned kernel shape). */
void nf_config_default(nf_config *cfg);

nf_status nf_init(const nf_config *cfg, nf_ctx **out);
void nf_shutdown(nf_ctx *ctx);
/* Message of the last failing call on this thread ("" if none). */
const char *nf_last_error(void);
int nf_abi_version(void);

/* ---------------- 1. GPU control ---------------- */
/* GetNGPU (GPUControl.cu:267-271) */
nf_status nf_get_ngpu(int *ngpu);
/* GetDeviceInfo (GPUControl.cu:274-285): 80% of the smallest device's
 * memory, and the device name. */
nf_status nf_get_device_info(size_t *mem_bytes, char *name, size_t name_len);

/* GPUSetup (GPUControl.cu:357-482): size per-buffer work limits from the
 * buffer byte budget with the reference's bytes-per-block model, create
 * nbuffers = ngpu * buffers_per_device buffers (device memory, pinned host
 * staging, one stream and one worker thread each).  Returns the SIC limits
 * MaxSinkBlocks / MaxSourceBlocks (and, through the optional pointers, MaxNSink,
 * MaxNSource, MaxSinkSize, MaxSourceSize). */
typedef struct nf_gpu_limits {
    int max_sink_blocks, max_source_blocks;
    int max_nsink, max_nsource;
    size_t max_sink_size, max_source_size;
} nf_gpu_limits;
nf_status nf_gpu_setup(nf_ctx *ctx, int cpd, uint64_t max_buffer_bytes, int ngpu,
                       int buffers_per_device, int use_pinned, nf_gpu_limits *limits);
/* GPUReset (GPUControl.cu:492-510): drain the queues, join the workers, free. */
nf_status nf_gpu_reset(nf_ctx *ctx);

/* ---------------- 2. plain drop-in: one SetInteractionCollection ---------------- */
/* Mirrors the SIC fields of singlestep/Direct/SetInteractionCollection.hh:
 * 171-283 that GPUPencilTask reads.  Pencil plans are given per cell
 * (start index in the slab's PosXYZ arrays without ghosts; count), so the
 * library gathers the pencils itself (PencilPlan.cc:22-90, 214-255). */
typedef struct nf_cell_plan {
    uint32_t start; /* CellPencilPlan::start */
    int32_t n;      /* CellPencilPlan::N */
} nf_cell_plan;

typedef struct nf_sic_desc {
    int cpd, nfradius;         /* R; nfwidth = 2R+1 */
    int nk;                    /* Nk: z cells per y row */
    int nsinksets;             /* NSinkSets = j_width * Nk */
    int nsourcesets;           /* NSourceSets = Nk * (j_width + 2R) */
    int nsinkblocks;           /* NSinkBlocks */
    int nsourceblocks;         /* NSourceBlocks */
    int interaction_count;     /* nfwidth * NSinkSets */
    /* per sink pencil */
    const int32_t *sink_set_start;      /* padded start, SinkSetStart */
    const int32_t *sink_set_count;      /* SinkSetCount */
    const uint32_t *sink_set_id_max;    /* SinkSetIdMax */
    const nf_cell_plan *sink_plan;      /* [nsinksets][nfwidth] cells zc-R..zc+R */
    const int32_t *sink_wrapcell;       /* SinkPencilPlan::wrapcell per pencil */
    const int32_t *sink_block_parent;   /* SinkBlockParentPencil[nsinkblocks] */
    /* per source pencil */
    const int32_t *source_set_start;    /* padded start, SourceSetStart */
    const int32_t *source_set_count;    /* SourceSetCount */
    const nf_cell_plan *source_plan;    /* [nsourcesets][nfwidth] cells x-R..x+R */
    /* interactions */
    const int32_t *interaction_list;    /* SinkSourceInteractionList */
    const float *y_offset;              /* SinkSourceYOffset */
    /* slabs (host PosXYZ: X[Nslab] | Y[Nslab] | Z[Nslab]) */
    const float *sink_pos_slab;         /* SinkPosSlab */
    uint64_t sink_nslab;                /* Nslab[R] */
    const float *const *source_pos_slab;/* SourcePosSlab[nfwidth] */
    const uint64_t *source_nslab;       /* Nslab[nfwidth] */
    void *sink_acc_slab;                /* AccSlab (accstruct, out_kind of the context) */
    float b2;
    /* counters written back (SetInteractionCollection.hh:182-183, 243-248) */
    uint64_t *bytes_to_device, *bytes_from_device;
    /* 2D z-split layout (MPI_size_z > 1; PencilOnPencil.cc:37-43, 200-204,
     * PencilPlan.cc:95-138): this node's primary z cells are
     * [node_z_start, node_z_start + node_z_size); Nk = node_z_size + 2R
     * pencils centred from node_z_start - R (index_to_zcen with pad R, no z
     * wrap); sink plans truncated to primary cells with AccSlab starts
     * (startindex), source plans with PosXYZ starts including ghost cells
     * (startindex_with_ghost).  node_z_size = 0: the whole z range (Nk = cpd).
     * Requires node_z_size + 2R <= cpd. */
    int node_z_start, node_z_size;
} nf_sic_desc;

/* Run one SIC (GPUPencilTask): gather pencils, H2D, kernel, D2H, co-add
 * into sink_acc_slab (first pencil of each y row sets, later ones add, the
 * last cell of a non-wrapping pencil sets), then store 1 in *completion.
 * blocking != 0 runs on the calling thread; otherwise the SIC is queued to a
 * worker (queue chosen by the SIC's y centre, GPUControl.cu:240) and the
 * call returns at once.  The descriptor's arrays must stay valid until
 * *completion becomes 1. */
nf_status nf_sic_execute(nf_ctx *ctx, const nf_sic_desc *sic, int jlow, int jhigh,
                         int blocking, volatile int *completion);
/* Wait for every queued SIC (bounded). */
nf_status nf_sic_drain(nf_ctx *ctx, uint64_t timeout_ns);
/* Pencil-kernel time of the SICs completed on this context since the last
 * reset (CUDA events around each SIC's launch, summed), how many SICs and
 * their unpadded pairs; reset != 0 zeroes the counters after reading.  The
 * reference times the same span per SIC with its DeviceData timers
 * (PencilTask.cu:154-257, SetInteractionCollection.hh:243-248).  SICs that
 * run concurrently on several buffers overlap, so their summed kernel time
 * exceeds the wall time the GPU was busy. */
nf_status nf_sic_timing(nf_ctx *ctx, double *kernel_ms, uint64_t *sics, uint64_t *pairs,
                        int reset);

/* ---------------- 2b. NearFieldDriver and the SIC planner ---------------- */
/* The host side of the drop-in: a C++ NearFieldDriver with the reference's
 * methods (singlestep/Timestep/directdriver.cpp:22-95) and a
 * SetInteractionCollection planner (PencilOnPencil.cc:180-418), driven
 * through these entry points.  The abacus globals they read (CP, SB, SS, P)
 * are replaced by per-slab views registered by the caller. */

/* cellinfo, singlestep/DataModel/particlestruct.cpp:334-346 (same layout). */
typedef struct nf_cellinfo {
    uint64_t startindex;
    uint64_t startindex_with_ghost;
    int32_t count;
    int32_t active;
    float mean_square_velocity;
    float max_component_velocity;
    float max_component_acceleration;
} nf_cellinfo;

/* One x-slab as abacus holds it. */
typedef struct nf_slab_view {
    const float *posxyz;          /* PosXYZSlab: X[nslab] | Y[nslab] | Z[nslab] */
    uint64_t nslab;               /* SS->size_with_ghost(slab) */
    const nf_cellinfo *cellinfo;  /* CellInfoSlab: cpd*cpd cells, (y, z) order */
    void *acc;                    /* AccSlab: one accstruct per particle (sink slabs) */
} nf_slab_view;

typedef struct nf_driver_params {
    int device;
    int cpd;
    int64_t np;
    int near_field_radius;         /* P.NearFieldRadius */
    int softening;                 /* NF_SOFT_* (configure --with-softening) */
    double softening_length;       /* ReadState.SofteningLengthNow / BoxSize (Plummer-equivalent) */
    float density_kernel_rad2;     /* WriteState.DensityKernelRad2 (b2; 0 = no density) */
    int direct_bpd;                /* P.DirectBPD */
    double mem_per_gpu_buffer_gb;  /* P.MemPerGPUBufferGB (0 = auto) */
    double max_ram_mb;             /* P.MAXRAMMB (auto buffer sizing) */
    int use_pinned_gpu_memory;     /* P.UsePinnedGPUMemory (-1 = auto) */
    int accumulation;              /* NF_ACC_* */
    int out_kind;                  /* NF_OUT_* (accstruct) */
    /* 2D z-split (MPI_size_z > 1): this node's primary z cells
     * [node_z_start, node_z_start + node_z_size) (node_z_size = 0: all of z).
     * Slab views then only need the cells z in [node_z_start - R,
     * node_z_start + node_z_size + R) filled: startindex numbers primary
     * cells (AccSlab), startindex_with_ghost numbers PosXYZ (ghosts too).
     * Requires node_z_size + 2R <= cpd. */
    int node_z_start, node_z_size;
} nf_driver_params;

/* NearFieldDriver statistics (directdriver.cpp:41-77, filled by Finalize and
 * AggregateStats, directdriver.cpp:434-526). */
typedef struct nf_driver_stats {
    uint64_t direct_interactions;         /* TotalDirectInteractions_GPU */
    uint64_t padded_direct_interactions;  /* TotalPaddedDirectInteractions_GPU */
    double gdi_gpu, gdi_padded_gpu;       /* the above / 1e9 */
    double total_gb_to, total_gb_from;
    double total_sinks, total_sources, total_padded_sinks, total_padded_sources;
    double mean_splits_per_slab;
    int max_nsplits;
    double gpu_throughput_time;           /* s with at least one SIC in flight */
    double calc_split_s, sic_construction_s, sic_execute_s, finalize_s;
    double softening_length_internal;
    float eps;
    int ngpu, nbuffers;
    int max_sink_blocks, max_source_blocks;
} nf_driver_stats;

typedef struct nf_driver nf_driver;

/* NearFieldDriver::NearFieldDriver(int NearFieldRadius) (directdriver.cpp:105-203):
 * eps per softening, GPU count, buffer sizing, GPUSetup. */
nf_status nf_driver_create(const nf_driver_params *p, nf_driver **out);
/* Register slab `slab`'s data (positions, cellinfo, acceleration arena).
 * Slabs slab-R .. slab+R must be registered before ExecuteSlab(slab). */
nf_status nf_driver_set_slab(nf_driver *drv, int slab, const nf_slab_view *view);
/* ExecuteSlab / ExecuteSlabGPU (directdriver.cpp:242-409): split the slab
 * into y-ranges fitting the GPU buffers, build the SICs, queue them. */
nf_status nf_driver_execute_slab(nf_driver *drv, int slab, int blocking);
/* SlabDone (directdriver.cpp:414-431): 1 when every SIC of the slab has
 * completed, 0 while in flight, -1 if one failed. */
int nf_driver_slab_done(nf_driver *drv, int slab);
/* Finalize (directdriver.cpp:434-492): collect SIC statistics, free them. */
nf_status nf_driver_finalize(nf_driver *drv, int slab);
/* AggregateStats (directdriver.cpp:498-526). */
nf_status nf_driver_aggregate_stats(nf_driver *drv, nf_driver_stats *stats);
/* The underlying context (to share with nf_box_* calls). */
nf_ctx *nf_driver_context(nf_driver *drv);
void nf_driver_destroy(nf_driver *drv);

/* The SetInteractionCollection planner alone (no GPU): plan rows
 * [jlow, jhigh) of slab `slab` over registered slabs and return its sizes
 * and counters (NSinkSets, NSourceSets, NSinkBlocks, NSourceBlocks,
 * InteractionCount, DirectTotal, PaddedDirectTotal, SinkTotal, SourceTotal).
 * Arrays, when non-NULL, receive SinkSetCount[nsinksets],
 * SinkBlockParentPencil[nsinkblocks], SourceSetCount[nsourcesets]. */
typedef struct nf_sic_summary {
    int nsinksets, nsourcesets, nsinkblocks, nsourceblocks, interaction_count;
    uint64_t direct_total, padded_direct_total, sink_total, source_total;
    uint64_t padded_sink_total, padded_source_total;
} nf_sic_summary;
nf_status nf_driver_plan_sic(nf_driver *drv, int slab, int jlow, int jhigh, nf_sic_summary *sum,
                             int32_t *sink_set_count, int32_t *sink_block_parent,
                             int32_t *source_set_count);

/* ---------------- 3. batched form: a box resident in HBM ---------------- */
/* Upload a box: cpd^3 cells, particles sorted by cell id ((cx*cpd)+cy)*cpd+cz,
 * float32 positions relative to the cell centre given as three host arrays,
 * cell_start[cpd^3+1] prefix offsets (host).  The library stores float4
 * records in HBM and keeps them until nf_box_destroy. */
nf_status nf_box_create(nf_ctx *ctx, int cpd, int64_t np, const int64_t *cell_start,
                        const float *x, const float *y, const float *z, nf_box **out);
/* Replace the positions of a registered box (same cell counts); x, y, z
 * may be host or device arrays (CUDA unified addressing).  Calls on one
 * context are serialised, but a serving request of the box that is still
 * running reads the positions being replaced: update a box only between
 * its requests (nf_server_wait). */
nf_status nf_box_update(nf_ctx *ctx, nf_box *box, const float *x, const float *y,
                        const float *z);
void nf_box_destroy(nf_ctx *ctx, nf_box *box);
/* One whole step end to end, pipelined: upload new positions (host or
 * device x, y, z, same cell counts), sweep every slab, and copy the
 * records of all particles to out (host or device), as nf_box_update +
 * nf_box_forces(0, cpd) would, but in n_chunks slab chunks (0: 8) so that
 * copies in and out overlap the sweeps of other chunks: chunk k is copied
 * in and ordered, then the slab range whose halo it completes is swept and
 * copied out while the next chunks arrive.  Each chunk needs at least R
 * slabs.  Results equal nf_box_forces(lo, hi) over the same chunk ranges,
 * bit for bit. */
nf_status nf_box_step(nf_ctx *ctx, nf_box *box, const float *x, const float *y, const float *z,
                      void *out, int n_chunks);
/* The same positions as records of three floats per particle (abacus'
 * PosSlab / posstruct layout, cell order) instead of three arrays: the
 * transpose to the device layout happens on the device (the reference
 * transposes on the host into PosXYZ, singlestep/Timestep/pipeline.cpp:
 * 84-124, singlestep/DataModel/cellparticles.cpp:214-226).  Host or device
 * memory. */
nf_status nf_box_update_aos(nf_ctx *ctx, nf_box *box, const float *xyz);
/* Give the box its own softening parameter (same convention as
 * nf_config.eps for the context's softening; 0 = the context's), so that
 * boxes of different particle spacing share one context and one server.
 * Waits for the device and drops the box's cached plans: call it while no
 * sweep or request of this box is in flight. */
nf_status nf_box_set_eps(nf_ctx *ctx, nf_box *box, float eps);
/* Device bytes held by the box (positions + plans + partial buffers). */
size_t nf_box_device_bytes(const nf_box *box);

/* Accelerations of every sink in x-slabs [slab_lo, slab_hi) (0 <= lo < hi <=
 * cpd).  out receives one record per particle of those slabs, in particle
 * order starting at the first particle of slab_lo.  out_on_device selects
 * whether out is a device pointer (0 copies) or host memory (copied back
 * before the call returns).  The work is one persistent CUDA-graph launch
 * per call shape. */
nf_status nf_box_forces(nf_ctx *ctx, nf_box *box, int slab_lo, int slab_hi, void *out,
                        int out_on_device);

/* Exact pair count for slabs [lo, hi) (DirectTotal, PencilOnPencil.cc:412). */
nf_status nf_box_pair_count(nf_ctx *ctx, const nf_box *box, int slab_lo, int slab_hi,
                            uint64_t *pairs);

typedef struct nf_timing {
    float kernel_ms;      /* persistent pair kernel, CUDA events */
    float coadd_ms;       /* partial co-add kernel */
    float total_ms;       /* whole call on the device */
    uint64_t pairs;       /* unpadded pairs */
    uint64_t padded_pairs;/* pairs including null-padded lanes/sources */
    int launches;         /* kernel launches of the call */
    int items;            /* warp work items */
    int variant;          /* kernel shape that ran */
} nf_timing;
/* Timing of the last nf_box_forces on this context. */
nf_status nf_last_timing(nf_ctx *ctx, nf_timing *t);

/* Kernel shapes the autotuner chooses among (sinks per lane, unroll depth,
 * CTAs per SM).  The first nf_box_forces call on a box times every shape on
 * the requested slab range and keeps the fastest for that box. */
int nf_kernel_variant_count(void);
const char *nf_kernel_variant_name(int variant);
/* The box's chosen shape (-1 before tuning) and the kernel time of each
 * candidate during tuning (ms[0 .. n-1]). */
nf_status nf_box_tuning(const nf_box *box, int *variant, float *ms, int n);

/* ---------------- 4. serving: slab requests over resident boxes ---------------- */
/* A request loop with continuous admission: slab requests (one x-slab of
 * one registered box) may be submitted from any thread at any time; a
 * dispatcher admits them, oldest first, as soon as a slot is free and the
 * request's device memory fits the HBM budget, and launches each on its own
 * stream, so requests that arrive while others run overlap with them on the
 * device.  Positions stay resident (nf_box_create); each admitted request
 * holds its own partials, counters and output until it completes.  The
 * result goes to the caller's buffer (host or device); latency is measured
 * from submission to the result being there. */
typedef struct nf_server nf_server;
typedef uint64_t nf_ticket;

typedef struct nf_server_config {
    size_t hbm_budget_bytes;  /* device bytes admitted requests may hold; 0 = 90% of the
                                 device memory free when the server starts */
    int max_inflight;         /* slots: requests on the device at once (default 2: one
                                 running, the next queued behind it; more slots overlap
                                 requests that then share the GPU and all run longer) */
    int max_queued;           /* pending requests beyond which submit fails (default 65536) */
} nf_server_config;

typedef struct nf_server_stats {
    uint64_t submitted, admitted, completed, failed, rejected, cancelled;
    uint64_t pairs;               /* pairs of completed requests */
    double busy_s;                /* wall time with at least one request admitted */
    double p50_ms, p99_ms, mean_ms, max_ms;  /* latency: submit -> result in caller's buffer */
    double queue_p50_ms, queue_p99_ms;       /* submit -> admission */
    int max_concurrent;           /* most requests on the device at once */
    size_t hbm_budget_bytes, hbm_peak_bytes;
} nf_server_stats;

nf_status nf_server_start(nf_ctx *ctx, const nf_server_config *cfg, nf_server **out);
/* Queue one slab request.  `out` receives the slab's records (particle
 * order); it must stay valid until the ticket completes.  NF_EADMISSION if
 * the request alone cannot fit the HBM budget or the queue is full. */
nf_status nf_server_submit(nf_server *srv, nf_box *box, int slab, void *out, int out_on_device,
                           nf_ticket *ticket);
/* *state: 1 completed, 0 pending or running, -1 failed or cancelled. */
nf_status nf_server_poll(nf_server *srv, nf_ticket ticket, int *state);
/* Wait for a ticket (bounded): NF_OK, NF_ETIMEDOUT, NF_ECANCELLED or the
 * request's failure status. */
nf_status nf_server_wait(nf_server *srv, nf_ticket ticket, uint64_t timeout_ns);
/* Cancel a request that has not been admitted yet (NF_EINVAL otherwise). */
nf_status nf_server_cancel(nf_server *srv, nf_ticket ticket);
/* One request's record: what happened to it and when.  Finished requests
 * stay queryable until 65536 newer ones have finished. */
typedef struct nf_request_info {
    int state;          /* 0 queued, 1 running, 2 completed, -1 failed, -2 cancelled */
    nf_status status;   /* failure status (NF_OK otherwise) */
    int slab, slot;     /* the slab; the slot it runs / ran on (-1: not admitted) */
    uint64_t pairs;     /* pairs of the slab (0 until admitted) */
    double submit_ms;   /* submission time, ms since nf_server_start */
    double queue_ms;    /* submit -> admission (-1: not admitted) */
    double run_ms;      /* admission -> result in the caller's buffer (-1: not completed) */
    double total_ms;    /* submit -> result (-1: not completed) */
} nf_request_info;
nf_status nf_server_request_info(nf_server *srv, nf_ticket ticket, nf_request_info *info);
nf_status nf_server_stats_get(nf_server *srv, nf_server_stats *stats);
/* Reset latency statistics (e.g. after warm-up). */
nf_status nf_server_stats_reset(nf_server *srv);
/* Drain or cancel what is queued, wait for what runs (bounded), stop. */
void nf_server_stop(nf_server *srv);

/* Near field of slabs [lo, hi) fused with the step that follows it in
 * abacus: RescaleAndCoAddAcceleration (singlestep/Timestep/kick.cpp:72-107)
 * and KickCell (kick.cpp:30-56), per particle in float, unfused, in the
 * reference's order:
 *     a = (nacc * near_scale + far_acc) * rescale;   w = nacc.w - b2
 *     v += a * kick1;  (cell stats);  v += a * kick2
 * where nacc is the record nf_box_forces returns.  Device pointers, one
 * record per particle of the slabs in particle order: far_acc float3 (NULL:
 * no far field), vel float3 (updated in place), acc_out accstruct (out_kind;
 * NULL: not stored), cell_stats 3 floats per cell of the slabs in cell
 * order (NULL: not computed): mean square velocity after the first half
 * kick, max |v| component, max |a| component (the cellinfo fields
 * mean_square_velocity, max_component_velocity, max_component_acceleration;
 * the mean is summed in a different order than the reference's loop). */
typedef struct nf_kick_params {
    float near_scale; /* single spline: 1/eps_int^3 (kick.cpp:86-96); otherwise 1 */
    float rescale;    /* -3 (Omega_M - Omega_Smooth) / (8 pi N), negated for glass */
    float kick1, kick2;
    float b2;         /* WriteState.DensityKernelRad2, subtracted from w */
} nf_kick_params;
nf_status nf_box_kick(nf_ctx *ctx, nf_box *box, int slab_lo, int slab_hi,
                      const nf_kick_params *kick, const float *far_acc, float *vel,
                      void *acc_out, float *cell_stats);

/* Allocation-free variant of the batched sweep (no counterpart in the
 * reference).  For callers that cannot call cudaMalloc -- code that runs
 * inside another framework's memory pool or caching allocator, or in a
 * process whose device allocations are fixed after start-up.  Nothing is
 * allocated on the device or the host: the scratch (pencil partials and a
 * work counter) is one 32 MiB static device array, held by every GPU that
 * loads this library until the process exits.
 *   pos        device float4 records (x, y, z, unused) in cell order
 *   cell_start device int64 prefix offsets, cpd^3 + 1 entries
 *   out        device records (cfg->out_kind) for the particles of slabs
 *              [slab_lo, slab_hi), in particle order
 *   stream     a cudaStream_t, or NULL for the default stream
 * At most 196608 particles in the requested slabs, and cpd^3 < 2^31; more
 * is NF_EINVAL.  The first call on each device looks up the array's device
 * address with that device current; make that first call before any stream
 * capture.  All calls share the one array and it keeps the last call's
 * contents: calls that overlap on the GPU (other streams, other host
 * threads) race.  Every call first copies the slab range's two particle
 * bounds from cell_start to the host and synchronizes `stream` to read
 * them, so the host waits for all earlier work on `stream`; the sweep and
 * the co-add are then queued on `stream` and the call returns without
 * waiting for them. */
nf_status nf_forces_noalloc(const nf_config *cfg, int cpd, const void *pos,
                            const int64_t *cell_start, int slab_lo, int slab_hi, void *out,
                            void *stream);

/* Run the context's work on the caller's CUDA stream (a cudaStream_t passed
 * as void*); NULL restores the library's own non-blocking stream. */
nf_status nf_set_stream(nf_ctx *ctx, void *stream);

/* FP32 roofline denominator measured on this device: a pure FFMA kernel
 * (8 independent chains of paired f32x2 FMAs per thread, every SM full)
 * timed with CUDA events.
 * burst = best of short runs; sustained = back-to-back for ~seconds_sustained.
 * Results in TFLOP/s (FFMA = 2 flops). */
nf_status nf_measure_fp32_peak(nf_ctx *ctx, double seconds_sustained, double *burst_tflops,
                               double *sustained_tflops);

#ifdef __cplusplus
}
#endif

#endif /* NF_CAPI_H */
