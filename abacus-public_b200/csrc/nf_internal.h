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

}  // namespace nf

struct nf_box {
    int cpd = 0;
    int64_t np = 0;
    std::vector<int64_t> cell_start;  // host copy, cpd^3 + 1
    float4 *d_pos = nullptr;          // np records (x, y, z, 0), cell order
    int64_t *d_cs = nullptr;          // cell_start on the device
    double *d_part = nullptr;         // pencil partials scratch
    float *d_stage = nullptr;         // position upload staging, 3 * np floats
    size_t part_bytes = 0;
    std::map<std::pair<int, int>, std::unique_ptr<nf::Plan>> plans;
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
