// nf_internal.h -- host-side internals shared by the library's translation units.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "nf_capi.h"

namespace nf {

// thread-local error text behind nf_last_error()
void set_error(const std::string &msg);
nf_status cuda_fail(cudaError_t e, const char *what);

#define NF_CUDA(call)                                          \
    do {                                                       \
        cudaError_t _e = (call);                               \
        if (_e != cudaSuccess) return nf::cuda_fail(_e, #call); \
    } while (0)

// A pencil partial of one sink and component: a compensated FP32 sum kept as
// (hi, lo), value hi + lo.  The co-add sums the 2R+1 partials of a sink with
// compensated FP32 arithmetic too, so no FP64 enters the accumulation.
typedef float2 Partial;

// One warp work item of the pencil kernel (32 bytes).
struct Item {
    int32_t pencil;      // linear id of the pencil's centre cell (x, y, zc)
    int32_t sink_begin;  // first sink of the tile in the pencil's sink stream
    int32_t nsink;       // sinks in the tile (1 .. 32*S)
    int32_t S;           // sinks per lane: 1, 2 or 4
    int32_t src_begin;   // source stream range [src_begin, src_end)
    int32_t src_end;
    int32_t pad0, pad1;
};

struct Plan {
    int lo = 0, hi = 0;
    int variant = 0;  // kernel shape (index into the variant table)
    int64_t p0 = 0, n_range = 0;
    Item *d_heavy = nullptr;
    int n_heavy_groups = 0;
    Item *d_light = nullptr;
    int n_light = 0;
    int *d_counters = nullptr;
    void *d_out = nullptr;
    size_t out_bytes = 0;
    uint64_t pairs = 0, padded_pairs = 0;
    int grid = 0, warps = 0;
    cudaGraphExec_t graph = nullptr;
};

// The pencil engine, shared by the batched form (nf_box.cu) and the plain
// drop-in (nf_sic.cu).  A launch covers the pencils listed in `items` of a
// box described by float4 positions and a cell prefix array whose linear
// cell id is ((x*cpd)+y)*cpd+z for x in [0, nx).
struct EngineLaunch {
    const float4 *pos = nullptr;
    const int64_t *cs = nullptr;
    int cpd = 0;
    const Item *heavy = nullptr;  // CTA-split groups (WARPS_PER_CTA items each)
    int n_heavy_groups = 0;
    const Item *light = nullptr;
    int n_light = 0;
    int *counters = nullptr;      // 2 ints, zeroed by engine_launch
    Partial *part = nullptr;      // (2R+1) * nc * n_range partials
    int64_t p0 = 0, n_range = 0;  // the sinks' particle range
    int variant = 0;
    int grid = 0;                 // CTAs (0: one full wave)
    float eps = 0.f;              // softening parameter (0: the context's)
};
nf_status engine_launch(nf_ctx *ctx, const EngineLaunch &L, double box_h, cudaStream_t st);
// perm (optional): the caller's index of each packed slot; record p of the
// range [p0, p0 + n) is written at perm[p0 + p] - p0.
nf_status engine_coadd(nf_ctx *ctx, const Partial *part, int64_t n, void *out, cudaStream_t st,
                       float eps = 0.f, const uint32_t *perm = nullptr, int64_t p0 = 0);
nf_status engine_pack(nf_ctx *ctx, const float *x, const float *y, const float *z, int64_t n,
                      float4 *out, cudaStream_t st);
int engine_grid(nf_ctx *ctx, int variant);
int engine_variant_smax(int variant);
int engine_plain_variant();
constexpr int ENGINE_WARPS_PER_CTA = 8;
// SIC size limits from a buffer budget (the reference's bytes-per-block model).
nf_status sic_limits(int out_kind, int cpd, uint64_t max_buffer_bytes, nf_gpu_limits *lim);
// The cached work list of a box's slab range (nf_box.cu).
struct Plan;
}  // namespace nf
struct nf_box;
namespace nf {
nf_status box_plan(nf_ctx *ctx, nf_box *box, int lo, int hi, const Plan **out);

}  // namespace nf

struct nf_box {
    int cpd = 0;
    int64_t np = 0;
    std::vector<int64_t> cell_start;  // host copy, cpd^3 + 1
    float4 *d_pos = nullptr;          // np records (x, y, z, 0), cell order
    int64_t *d_cs = nullptr;          // cell_start on the device
    nf::Partial *d_part = nullptr;    // pencil partials scratch
    float *d_stage = nullptr;         // position upload staging, 3 * np floats
    uint32_t *d_perm = nullptr;       // caller's index of the particle in each packed slot
    void *d_sort = nullptr;           // in-cell ordering scratch (keys, values, sort temp)
    size_t sort_bytes = 0;
    // pipelined step (nf_box_step): copy-in and copy-out streams, per-chunk events
    cudaStream_t s_in = nullptr, s_out = nullptr;
    std::vector<cudaEvent_t> step_ev;
    size_t part_bytes = 0;
    std::map<std::pair<int, int>, std::unique_ptr<nf::Plan>> plans;
    int variant = -1;       // kernel shape chosen by the autotuner (-1: not tuned yet)
    float eps = 0.f;        // the box's own softening parameter (0: the context's)
    float tune_ms[8] = {};  // kernel time of each candidate during tuning
    size_t device_bytes() const;
};

struct nf_ctx {
    nf_config cfg{};
    int device = 0;
    int sms = 0;
    cudaStream_t stream = nullptr;      // where work is enqueued (own or caller's)
    cudaStream_t own_stream = nullptr;  // created by nf_init
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    nf_timing last{};
    std::mutex mu;  // serialises nf_box_forces on one context
    // plain drop-in GPU control (nf_sic.cu)
    struct Sic;
    Sic *sic = nullptr;
};
