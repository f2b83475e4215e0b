// nf_ctx.cu -- context, errors and device queries of the C ABI.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "nf_internal.h"

namespace nf {

static thread_local std::string g_err;

void set_error(const std::string &msg) { g_err = msg; }

nf_status cuda_fail(cudaError_t e, const char *what) {
    char buf[512];
    snprintf(buf, sizeof(buf), "%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
    g_err = buf;
    cudaGetLastError();  // clear a non-sticky error so the context stays usable
    if (e == cudaErrorMemoryAllocation) return NF_ENOMEM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return NF_ENODEV;
    return NF_EDEVICE;
}

}  // namespace nf

using namespace nf;

extern "C" const char *nf_last_error(void) { return g_err.c_str(); }
extern "C" int nf_abi_version(void) { return NF_ABI_VERSION; }

extern "C" void nf_config_default(nf_config *cfg) {
    if (!cfg) return;
    memset(cfg, 0, sizeof(*cfg));
    cfg->device = 0;
    cfg->near_field_radius = 2;
    cfg->softening = NF_SOFT_SINGLE_SPLINE;
    cfg->eps = 1.0f;
    cfg->b2 = 0.f;
    cfg->accumulation = NF_ACC_COMPENSATED;
    cfg->out_kind = NF_OUT_FLOAT4;
    cfg->sinks_per_lane = 0;
    cfg->kernel_variant = -1;
}

static nf_status check_config(const nf_config *c) {
    if (c->near_field_radius < 1 || c->near_field_radius > 2) {
        set_error("near_field_radius must be 1 or 2");
        return NF_EINVAL;
    }
    if (c->softening < NF_SOFT_PLUMMER || c->softening > NF_SOFT_CUBIC_PLUMMER) {
        set_error("unknown softening");
        return NF_EINVAL;
    }
    if (!std::isfinite(c->eps) || c->eps <= 0.f) {
        set_error("eps must be finite and positive (directdriver.cpp:119)");
        return NF_EINVAL;
    }
    if (!std::isfinite(c->b2) || c->b2 < 0.f) {
        set_error("b2 must be finite and >= 0");
        return NF_EINVAL;
    }
    if (c->accumulation != NF_ACC_COMPENSATED && c->accumulation != NF_ACC_PLAIN) {
        set_error("unknown accumulation mode");
        return NF_EINVAL;
    }
    if (c->out_kind != NF_OUT_FLOAT3 && c->out_kind != NF_OUT_FLOAT4) {
        set_error("unknown output record kind");
        return NF_EINVAL;
    }
    if (c->sinks_per_lane != 0 && c->sinks_per_lane != 1 && c->sinks_per_lane != 2 &&
        c->sinks_per_lane != 4) {
        set_error("sinks_per_lane must be 0, 1, 2 or 4");
        return NF_EINVAL;
    }
    if (c->kernel_variant < -1 || c->kernel_variant >= nf_kernel_variant_count()) {
        set_error("kernel_variant out of range");
        return NF_EINVAL;
    }
    if (c->out_kind == NF_OUT_FLOAT3 && c->b2 > 0.f) {
        set_error("the density channel needs NF_OUT_FLOAT4 records");
        return NF_EINVAL;
    }
    return NF_OK;
}

extern "C" nf_status nf_get_ngpu(int *ngpu) {
    if (!ngpu) {
        set_error("nf_get_ngpu: null argument");
        return NF_EINVAL;
    }
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        *ngpu = 0;
        return cuda_fail(e, "cudaGetDeviceCount");
    }
    *ngpu = n;
    return n > 0 ? NF_OK : NF_ENODEV;
}

extern "C" nf_status nf_get_device_info(size_t *mem_bytes, char *name, size_t name_len) {
    int n = 0;
    nf_status st = nf_get_ngpu(&n);
    if (st != NF_OK) return st;
    size_t mem = SIZE_MAX;
    cudaDeviceProp p;
    for (int g = 0; g < n; g++) {
        NF_CUDA(cudaGetDeviceProperties(&p, g));
        size_t m = (size_t)(0.8 * (double)p.totalGlobalMem);
        if (m < mem) mem = m;
    }
    if (mem_bytes) *mem_bytes = mem;
    if (name && name_len) {
        strncpy(name, p.name, name_len - 1);
        name[name_len - 1] = 0;
    }
    return NF_OK;
}

extern "C" nf_status nf_init(const nf_config *cfg, nf_ctx **out) {
    if (!cfg || !out) {
        set_error("nf_init: null argument");
        return NF_EINVAL;
    }
    *out = nullptr;
    nf_status st = check_config(cfg);
    if (st != NF_OK) return st;
    int n = 0;
    st = nf_get_ngpu(&n);
    if (st != NF_OK) return st;
    if (cfg->device < 0 || cfg->device >= n) {
        set_error("nf_init: device ordinal out of range");
        return NF_EINVAL;
    }
    NF_CUDA(cudaSetDevice(cfg->device));
    nf_ctx *ctx = new nf_ctx;
    ctx->cfg = *cfg;
    ctx->device = cfg->device;
    cudaError_t e = cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, cfg->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking);
    ctx->stream = ctx->own_stream;
    for (int i = 0; i < 4 && e == cudaSuccess; i++) e = cudaEventCreate(&ctx->ev[i]);
    if (e != cudaSuccess) {
        nf_status s2 = cuda_fail(e, "nf_init");
        nf_shutdown(ctx);
        return s2;
    }
    *out = ctx;
    return NF_OK;
}

void nf_sic_shutdown(nf_ctx *ctx);  // nf_sic.cu

extern "C" void nf_shutdown(nf_ctx *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    nf_sic_shutdown(ctx);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (int i = 0; i < 4; i++)
        if (ctx->ev[i]) cudaEventDestroy(ctx->ev[i]);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
}

extern "C" nf_status nf_set_stream(nf_ctx *ctx, void *stream) {
    if (!ctx) {
        set_error("nf_set_stream: null context");
        return NF_EINVAL;
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    return NF_OK;
}

// FP32 throughput probe: 8 independent chains of paired FMAs (f32x2, two
// FMAs per instruction) per thread, 16 per loop trip, so that loop control
// takes under 1 % of the issue slots and the FMA pipe alone sets the rate.
constexpr int PEAK_CHAINS = 8, PEAK_UNROLL = 16;

__global__ void ffma_peak_kernel(float *out, int iters, float a, float b) {
    float2 x[PEAK_CHAINS];
#pragma unroll
    for (int c = 0; c < PEAK_CHAINS; c++)
        x[c] = make_float2(threadIdx.x * 1e-3f + 0.1f * c, threadIdx.x * 1e-3f - 0.1f * c);
    const float2 a2 = make_float2(a, a), b2 = make_float2(b, b);
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int u = 0; u < PEAK_UNROLL; u++)
#pragma unroll
            for (int c = 0; c < PEAK_CHAINS; c++) x[c] = __ffma2_rn(x[c], a2, b2);
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < PEAK_CHAINS; c++) s += x[c].x + x[c].y;
    if (s == 1234.5f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the chains live
}

extern "C" nf_status nf_measure_fp32_peak(nf_ctx *ctx, double seconds_sustained,
                                          double *burst_tflops, double *sustained_tflops) {
    if (!ctx) {
        set_error("nf_measure_fp32_peak: null context");
        return NF_EINVAL;
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    NF_CUDA(cudaSetDevice(ctx->device));
    const int threads = 256, blocks = ctx->sms * 8, iters = 4096;
    float *out = nullptr;
    NF_CUDA(cudaMalloc(&out, (size_t)blocks * threads * sizeof(float)));
    // FMA = 2 flops, two FMAs per paired instruction
    const double flops = 2.0 * 2.0 * PEAK_CHAINS * PEAK_UNROLL * (double)iters * blocks * threads;
    cudaStream_t s = ctx->stream;
    float best = 1e30f;
    cudaError_t e = cudaSuccess;
    for (int r = 0; r < 6 && e == cudaSuccess; r++) {  // first run warms up
        cudaEventRecord(ctx->ev[0], s);
        ffma_peak_kernel<<<blocks, threads, 0, s>>>(out, iters, 0.9999f, 1e-4f);
        cudaEventRecord(ctx->ev[1], s);
        e = cudaEventSynchronize(ctx->ev[1]);
        float ms = 0;
        cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
        if (r > 0 && ms < best) best = ms;
    }
    if (e != cudaSuccess) {
        cudaFree(out);
        return cuda_fail(e, "ffma_peak_kernel");
    }
    if (burst_tflops) *burst_tflops = flops / (best * 1e-3) / 1e12;
    int reps = (int)std::max(1.0, seconds_sustained * 1e3 / best);
    cudaEventRecord(ctx->ev[0], s);
    for (int r = 0; r < reps; r++)
        ffma_peak_kernel<<<blocks, threads, 0, s>>>(out, iters, 0.9999f, 1e-4f);
    cudaEventRecord(ctx->ev[1], s);
    e = cudaEventSynchronize(ctx->ev[1]);
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
    cudaFree(out);
    if (e != cudaSuccess) return cuda_fail(e, "ffma_peak_kernel");
    if (sustained_tflops) *sustained_tflops = flops * reps / (ms * 1e-3) / 1e12;
    return NF_OK;
}

extern "C" nf_status nf_last_timing(nf_ctx *ctx, nf_timing *t) {
    if (!ctx || !t) {
        set_error("nf_last_timing: null argument");
        return NF_EINVAL;
    }
    *t = ctx->last;
    return NF_OK;
}
