// nf_sic.cu -- plain drop-in: GPU control and one SetInteractionCollection.
// (filled in by the drop-in layer; the batched form does not depend on it)
#include "nf_internal.h"

using namespace nf;

struct nf_ctx::Sic {};

void nf_sic_shutdown(nf_ctx *ctx) {
    if (!ctx || !ctx->sic) return;
    delete ctx->sic;
    ctx->sic = nullptr;
}

extern "C" nf_status nf_gpu_setup(nf_ctx *ctx, int, uint64_t, int, int, int, nf_gpu_limits *) {
    (void)ctx;
    set_error("nf_gpu_setup: not built yet");
    return NF_EINVAL;
}

extern "C" nf_status nf_gpu_reset(nf_ctx *ctx) {
    nf_sic_shutdown(ctx);
    return NF_OK;
}

extern "C" nf_status nf_sic_execute(nf_ctx *, const nf_sic_desc *, int, int, int, volatile int *) {
    set_error("nf_sic_execute: not built yet");
    return NF_EINVAL;
}

extern "C" nf_status nf_sic_drain(nf_ctx *, uint64_t) { return NF_OK; }
