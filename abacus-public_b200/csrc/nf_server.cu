// nf_server.cu -- serving: slab requests over resident boxes with continuous
// admission.
//
// A dispatcher thread admits queued requests oldest first whenever a slot is
// free and the request's device memory (pencil partials, counters, output)
// fits the HBM budget, and launches each admitted request on its slot's own
// stream: the box's cached slab plan (built and autotuned on first use)
// drives one persistent pencil-kernel launch, the co-add and the copy to the
// caller's buffer.  Requests admitted while others run overlap with them on
// the device (a persistent grid's tail is filled by the next request's
// CTAs; copies overlap kernels).  A host callback after the copy marks the
// request complete and frees its slot; latency is submit -> that callback.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <unordered_map>

#include "nf_internal.h"

namespace nf {

using sclock = std::chrono::steady_clock;

struct Req;

struct Slot {
    int index = 0;
    cudaStream_t stream = nullptr;
    double *part = nullptr;
    void *out = nullptr;
    int *counters = nullptr;
    size_t part_cap = 0, out_cap = 0;  // bytes
    Req *req = nullptr;
    size_t bytes() const { return part_cap + out_cap + (part_cap ? 256 : 0); }
};

struct Req {
    nf_ticket id = 0;
    nf_box *box = nullptr;
    int slab = 0;
    void *out = nullptr;
    int on_dev = 0;
    int state = 0;  // 0 queued, 1 running, 2 done, -1 failed, -2 cancelled
    nf_status status = NF_OK;
    sclock::time_point t_submit, t_admit, t_done;
    uint64_t pairs = 0;
    Slot *slot = nullptr;
    struct nf_server *srv = nullptr;
};

}  // namespace nf

using namespace nf;

struct nf_server {
    nf_ctx *ctx = nullptr;
    nf_server_config cfg{};
    std::mutex mu;
    std::condition_variable cv, cv_done;
    std::deque<Req *> pending;
    std::unordered_map<nf_ticket, std::unique_ptr<Req>> reqs;
    std::vector<Slot> slots;
    size_t budget = 0, held = 0, peak = 0;
    nf_ticket next_id = 1;
    bool stop = false;
    int running = 0, max_running = 0;
    std::thread dispatcher;
    // statistics
    uint64_t submitted = 0, admitted = 0, completed = 0, failed = 0, rejected = 0, cancelled = 0;
    uint64_t pairs = 0;
    std::vector<double> lat_ms, queue_ms;
    double busy_s = 0;
    sclock::time_point busy_since;
};

static size_t rec_bytes(const nf_ctx *ctx) { return ctx->cfg.out_kind == NF_OUT_FLOAT4 ? 16 : 12; }

static void CUDART_CB on_done(void *arg) {
    Req *r = (Req *)arg;
    nf_server *s = r->srv;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        r->t_done = sclock::now();
        r->state = 2;
        r->slot->req = nullptr;
        r->slot = nullptr;
        s->completed++;
        s->pairs += r->pairs;
        s->lat_ms.push_back(std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count());
        s->queue_ms.push_back(std::chrono::duration<double, std::milli>(r->t_admit - r->t_submit).count());
        if (--s->running == 0)
            s->busy_s += std::chrono::duration<double>(r->t_done - s->busy_since).count();
    }
    s->cv.notify_all();
    s->cv_done.notify_all();
}

// Booking for one admission: the slot to (re)allocate and idle slots whose
// buffers are released to stay within the budget.  Decided with s->mu held;
// the CUDA calls happen after the lock is dropped (cudaFree waits for device
// work, including host callbacks that take s->mu).
struct Booking {
    Slot *slot = nullptr;
    size_t part = 0, out = 0;  // new capacities (0: keep the slot's buffers)
    std::vector<Slot *> release;
};

static bool book_slot(nf_server *s, Slot &sl, size_t part_need, size_t out_need, Booking &bk) {
    bk = Booking{};
    bk.slot = &sl;
    if (sl.part_cap >= part_need && sl.out_cap >= out_need && sl.counters) return true;
    size_t gp = std::max(part_need, sl.part_cap), go = std::max(out_need, sl.out_cap);
    size_t held = s->held - sl.bytes() + gp + go + 256;
    for (auto &o : s->slots) {
        if (held <= s->budget) break;
        if (&o == &sl || o.req || !o.part_cap) continue;
        bk.release.push_back(&o);
        held -= o.bytes();
    }
    if (held > s->budget) return false;
    bk.part = gp;
    bk.out = go;
    for (Slot *o : bk.release) {  // book the new total now
        s->held -= o->bytes();
        o->part_cap = o->out_cap = 0;
    }
    s->held = s->held - sl.bytes() + gp + go + 256;
    s->peak = std::max(s->peak, s->held);
    return true;
}

// Carry out a booking (no lock held).
static nf_status apply_booking(Booking &bk) {
    for (Slot *o : bk.release) {
        cudaFree(o->part);
        cudaFree(o->out);
        cudaFree(o->counters);
        o->part = nullptr;
        o->out = nullptr;
        o->counters = nullptr;
    }
    if (!bk.part) return NF_OK;
    Slot &sl = *bk.slot;
    cudaFree(sl.part);
    cudaFree(sl.out);
    cudaFree(sl.counters);
    sl.part = nullptr;
    sl.out = nullptr;
    sl.counters = nullptr;
    if (cudaMalloc(&sl.part, bk.part) != cudaSuccess || cudaMalloc(&sl.out, bk.out) != cudaSuccess ||
        cudaMalloc(&sl.counters, 256) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(sl.part);
        cudaFree(sl.out);
        cudaFree(sl.counters);
        sl.part = nullptr;
        sl.out = nullptr;
        sl.counters = nullptr;
        set_error("nf_server: device allocation failed within the HBM budget");
        return NF_ENOMEM;
    }
    sl.part_cap = bk.part;
    sl.out_cap = bk.out;
    return NF_OK;
}

static nf_status launch_request(nf_server *s, Req *r, Slot &sl, const Plan *pl) {
    nf_ctx *ctx = s->ctx;
    EngineLaunch L;
    L.pos = r->box->d_pos;
    L.cs = r->box->d_cs;
    L.cpd = r->box->cpd;
    L.heavy = pl->d_heavy;
    L.n_heavy_groups = pl->n_heavy_groups;
    L.light = pl->d_light;
    L.n_light = pl->n_light;
    L.counters = sl.counters;
    L.part = sl.part;
    L.p0 = pl->p0;
    L.n_range = pl->n_range;
    L.variant = pl->variant;
    L.grid = pl->grid;
    nf_status st = engine_launch(ctx, L, 0.0, sl.stream);
    if (st == NF_OK) st = engine_coadd(ctx, sl.part, pl->n_range, sl.out, sl.stream);
    if (st != NF_OK) return st;
    size_t bytes = (size_t)pl->n_range * rec_bytes(ctx);
    if (bytes)
        NF_CUDA(cudaMemcpyAsync(r->out, sl.out, bytes,
                                r->on_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                sl.stream));
    NF_CUDA(cudaLaunchHostFunc(sl.stream, on_done, r));
    return NF_OK;
}

static void fail_admitted(nf_server *s, Req *r, Slot *sl, nf_status st) {
    // called with s->mu held
    if (sl) {
        s->held -= sl->bytes();
        sl->part_cap = sl->out_cap = 0;
        sl->req = nullptr;
    }
    r->slot = nullptr;
    r->state = -1;
    r->status = st;
    s->failed++;
    if (--s->running == 0)
        s->busy_s += std::chrono::duration<double>(sclock::now() - s->busy_since).count();
    s->cv_done.notify_all();
}

static void dispatcher_main(nf_server *s) {
    cudaSetDevice(s->ctx->device);
    const int W = 2 * s->ctx->cfg.near_field_radius + 1;
    const int nc = s->ctx->cfg.b2 > 0.f ? 4 : 3;
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        s->cv.wait(lk, [&] {
            if (s->stop) return true;
            if (s->pending.empty()) return false;
            for (auto &sl : s->slots)
                if (!sl.req) return true;
            return false;
        });
        if (s->stop) break;
        Req *r = s->pending.front();
        // the slab's plan (built, and the box tuned, outside the lock on first use)
        lk.unlock();
        const Plan *pl = nullptr;
        nf_status st = box_plan(s->ctx, r->box, r->slab, r->slab + 1, &pl);
        lk.lock();
        if (r->state != 0) continue;  // cancelled meanwhile
        if (st != NF_OK) {
            s->pending.pop_front();
            r->state = -1;
            r->status = st;
            s->failed++;
            s->cv_done.notify_all();
            continue;
        }
        size_t part_need = (size_t)W * nc * (size_t)pl->n_range * sizeof(double) + 16;
        size_t out_need = (size_t)pl->n_range * rec_bytes(s->ctx) + 16;
        Slot *pick = nullptr;  // a free slot, preferring one already large enough
        for (auto &sl : s->slots)
            if (!sl.req && (!pick || (sl.part_cap >= part_need && pick->part_cap < part_need)))
                pick = &sl;
        Booking bk;
        if (!pick || !book_slot(s, *pick, part_need, out_need, bk)) {
            if (s->running == 0) {  // nothing in flight will free memory
                s->pending.pop_front();
                r->state = -1;
                r->status = NF_EADMISSION;
                s->rejected++;
                s->cv_done.notify_all();
                continue;
            }
            s->cv.wait_for(lk, std::chrono::milliseconds(1));  // until a request completes
            continue;
        }
        s->pending.pop_front();
        r->state = 1;
        r->slot = pick;
        r->pairs = pl->pairs;
        r->t_admit = sclock::now();
        pick->req = r;
        s->admitted++;
        if (s->running++ == 0) s->busy_since = r->t_admit;
        s->max_running = std::max(s->max_running, s->running);
        lk.unlock();
        st = apply_booking(bk);
        if (st == NF_OK) st = launch_request(s, r, *pick, pl);
        lk.lock();
        if (st != NF_OK) fail_admitted(s, r, pick, st);
    }
}

extern "C" nf_status nf_server_start(nf_ctx *ctx, const nf_server_config *cfg, nf_server **out) {
    if (!ctx || !out) {
        set_error("nf_server_start: null argument");
        return NF_EINVAL;
    }
    *out = nullptr;
    NF_CUDA(cudaSetDevice(ctx->device));
    auto s = std::make_unique<nf_server>();
    s->ctx = ctx;
    if (cfg) s->cfg = *cfg;
    if (s->cfg.max_inflight <= 0) s->cfg.max_inflight = 8;
    if (s->cfg.max_queued <= 0) s->cfg.max_queued = 65536;
    if (s->cfg.max_inflight > 256) {
        set_error("nf_server_start: max_inflight above 256");
        return NF_EINVAL;
    }
    size_t freeb = 0, total = 0;
    NF_CUDA(cudaMemGetInfo(&freeb, &total));
    s->budget = s->cfg.hbm_budget_bytes ? s->cfg.hbm_budget_bytes : (size_t)(0.9 * (double)freeb);
    s->slots.resize(s->cfg.max_inflight);
    for (int i = 0; i < s->cfg.max_inflight; i++) {
        s->slots[i].index = i;
        cudaError_t e = cudaStreamCreateWithFlags(&s->slots[i].stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            for (auto &sl : s->slots)
                if (sl.stream) cudaStreamDestroy(sl.stream);
            return cuda_fail(e, "nf_server_start");
        }
    }
    s->dispatcher = std::thread(dispatcher_main, s.get());
    *out = s.release();
    return NF_OK;
}

extern "C" nf_status nf_server_submit(nf_server *s, nf_box *box, int slab, void *out,
                                      int out_on_device, nf_ticket *ticket) {
    if (!s || !box || !out || !ticket || slab < 0 || slab >= box->cpd) {
        set_error("nf_server_submit: bad argument");
        return NF_EINVAL;
    }
    const int W = 2 * s->ctx->cfg.near_field_radius + 1;
    const int nc = s->ctx->cfg.b2 > 0.f ? 4 : 3;
    int64_t c2 = (int64_t)box->cpd * box->cpd;
    int64_t n = box->cell_start[(slab + 1) * c2] - box->cell_start[slab * c2];
    size_t need = (size_t)W * nc * n * sizeof(double) + (size_t)n * rec_bytes(s->ctx) + 512;
    std::lock_guard<std::mutex> lk(s->mu);
    s->submitted++;
    if (need > s->budget || (int)s->pending.size() >= s->cfg.max_queued) {
        s->rejected++;
        set_error(need > s->budget ? "nf_server_submit: request larger than the HBM budget"
                                   : "nf_server_submit: queue full");
        return NF_EADMISSION;
    }
    auto r = std::make_unique<Req>();
    r->id = s->next_id++;
    r->box = box;
    r->slab = slab;
    r->out = out;
    r->on_dev = out_on_device;
    r->srv = s;
    r->t_submit = sclock::now();
    *ticket = r->id;
    s->pending.push_back(r.get());
    s->reqs[r->id] = std::move(r);
    s->cv.notify_all();
    return NF_OK;
}

extern "C" nf_status nf_server_poll(nf_server *s, nf_ticket t, int *state) {
    if (!s || !state) {
        set_error("nf_server_poll: null argument");
        return NF_EINVAL;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(t);
    if (it == s->reqs.end()) {
        set_error("nf_server_poll: unknown ticket");
        return NF_EINVAL;
    }
    int st = it->second->state;
    *state = st == 2 ? 1 : (st < 0 ? -1 : 0);
    return NF_OK;
}

extern "C" nf_status nf_server_wait(nf_server *s, nf_ticket t, uint64_t timeout_ns) {
    if (!s) {
        set_error("nf_server_wait: null server");
        return NF_EINVAL;
    }
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(t);
    if (it == s->reqs.end()) {
        set_error("nf_server_wait: unknown ticket");
        return NF_EINVAL;
    }
    Req *r = it->second.get();
    bool ok = s->cv_done.wait_for(lk, std::chrono::nanoseconds(timeout_ns),
                                  [&] { return r->state == 2 || r->state < 0; });
    if (!ok) {
        set_error("nf_server_wait: request still pending at the timeout");
        return NF_ETIMEDOUT;
    }
    if (r->state == -2) {
        set_error("nf_server_wait: request cancelled");
        return NF_ECANCELLED;
    }
    if (r->state == -1) {
        set_error("nf_server_wait: request failed");
        return r->status != NF_OK ? r->status : NF_EDEVICE;
    }
    return NF_OK;
}

extern "C" nf_status nf_server_cancel(nf_server *s, nf_ticket t) {
    if (!s) {
        set_error("nf_server_cancel: null server");
        return NF_EINVAL;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(t);
    if (it == s->reqs.end() || it->second->state != 0) {
        set_error("nf_server_cancel: only queued requests can be cancelled");
        return NF_EINVAL;
    }
    Req *r = it->second.get();
    s->pending.erase(std::remove(s->pending.begin(), s->pending.end(), r), s->pending.end());
    r->state = -2;
    s->cancelled++;
    s->cv_done.notify_all();
    return NF_OK;
}

static double pct(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    double pos = q / 100.0 * (v.size() - 1);
    size_t i = (size_t)pos;
    double f = pos - i;
    return i + 1 < v.size() ? v[i] * (1 - f) + v[i + 1] * f : v[i];
}

extern "C" nf_status nf_server_stats_get(nf_server *s, nf_server_stats *o) {
    if (!s || !o) {
        set_error("nf_server_stats_get: null argument");
        return NF_EINVAL;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    memset(o, 0, sizeof(*o));
    o->submitted = s->submitted;
    o->admitted = s->admitted;
    o->completed = s->completed;
    o->failed = s->failed;
    o->rejected = s->rejected;
    o->cancelled = s->cancelled;
    o->pairs = s->pairs;
    o->busy_s = s->busy_s + (s->running ? std::chrono::duration<double>(sclock::now() - s->busy_since).count() : 0.0);
    o->p50_ms = pct(s->lat_ms, 50);
    o->p99_ms = pct(s->lat_ms, 99);
    double sum = 0, mx = 0;
    for (double v : s->lat_ms) {
        sum += v;
        mx = std::max(mx, v);
    }
    o->mean_ms = s->lat_ms.empty() ? 0 : sum / s->lat_ms.size();
    o->max_ms = mx;
    o->queue_p50_ms = pct(s->queue_ms, 50);
    o->queue_p99_ms = pct(s->queue_ms, 99);
    o->max_concurrent = s->max_running;
    o->hbm_budget_bytes = s->budget;
    o->hbm_peak_bytes = s->peak;
    return NF_OK;
}

extern "C" nf_status nf_server_stats_reset(nf_server *s) {
    if (!s) {
        set_error("nf_server_stats_reset: null server");
        return NF_EINVAL;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    s->submitted = s->admitted = s->completed = s->failed = s->rejected = s->cancelled = 0;
    s->pairs = 0;
    s->lat_ms.clear();
    s->queue_ms.clear();
    s->busy_s = 0;
    if (s->running) s->busy_since = sclock::now();
    s->max_running = s->running;
    return NF_OK;
}

extern "C" void nf_server_stop(nf_server *s) {
    if (!s) return;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        for (Req *r : s->pending) {
            r->state = -2;
            s->cancelled++;
        }
        s->pending.clear();
        s->cv_done.wait_for(lk, std::chrono::seconds(60), [&] { return s->running == 0; });
        s->stop = true;
    }
    s->cv.notify_all();
    s->cv_done.notify_all();
    if (s->dispatcher.joinable()) s->dispatcher.join();
    cudaSetDevice(s->ctx->device);
    for (auto &sl : s->slots) {
        if (sl.stream) {
            cudaStreamSynchronize(sl.stream);
            cudaStreamDestroy(sl.stream);
        }
        cudaFree(sl.part);
        cudaFree(sl.out);
        cudaFree(sl.counters);
    }
    delete s;
}
