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
 *     batching request loop (nf_serve_*).  These replace
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

#define NF_ABI_VERSION 1

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
    int sinks_per_lane;     /* 0 = autotuned tile shapes; else force 1, 2 or 4 */
    int warps_per_cta;      /* 0 = autotuned; else 4 or 8 */
} nf_config;

typedef struct nf_ctx nf_ctx;
typedef struct nf_box nf_box;

/* Fill *cfg with defaults (device 0, R 2, single spline, compensated, float4). */
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

/* ---------------- 3. batched form: a box resident in HBM ---------------- */
/* Upload a box: cpd^3 cells, particles sorted by cell id ((cx*cpd)+cy)*cpd+cz,
 * float32 positions relative to the cell centre given as three host arrays,
 * cell_start[cpd^3+1] prefix offsets (host).  The library stores float4
 * records in HBM and keeps them until nf_box_destroy. */
nf_status nf_box_create(nf_ctx *ctx, int cpd, int64_t np, const int64_t *cell_start,
                        const float *x, const float *y, const float *z, nf_box **out);
/* Replace the positions of a registered box (same cell counts). */
nf_status nf_box_update(nf_ctx *ctx, nf_box *box, const float *x, const float *y,
                        const float *z);
void nf_box_destroy(nf_ctx *ctx, nf_box *box);
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
} nf_timing;
/* Timing of the last nf_box_forces on this context. */
nf_status nf_last_timing(nf_ctx *ctx, nf_timing *t);

/* Run the context's work on the caller's CUDA stream (a cudaStream_t passed
 * as void*); NULL restores the library's own non-blocking stream. */
nf_status nf_set_stream(nf_ctx *ctx, void *stream);

/* FP32 roofline denominator measured on this device: a pure FFMA kernel
 * (8 independent chains per thread, every SM full) timed with CUDA events.
 * burst = best of short runs; sustained = back-to-back for ~seconds_sustained.
 * Results in TFLOP/s (FFMA = 2 flops). */
nf_status nf_measure_fp32_peak(nf_ctx *ctx, double seconds_sustained, double *burst_tflops,
                               double *sustained_tflops);

#ifdef __cplusplus
}
#endif

#endif /* NF_CAPI_H */
