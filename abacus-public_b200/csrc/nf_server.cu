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
//
// Slot memory comes from a memory pool owned by the server and is
// allocated and freed stream-ordered on the slot's stream, so growing one
// slot never waits for the requests running on the others (a plain
// cudaFree would synchronise the whole device).  A slot that must grow is
// sized for the largest slab of the request's box when the budget allows,
// so each slot grows at most once per box geometry.
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
    Partial *part = nullptr;
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
    int slot_index = -1;  // the slot it ran on (kept after completion)
    int waiters = 0;      // threads inside nf_server_wait on this request
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
    cudaMemPool_t pool = nullptr;
    sclock::time_point t_start;
    std::deque<nf_ticket> finished;  // retired oldest first beyond NF_SERVER_HISTORY
    // statistics
    uint64_t submitted = 0, admitted = 0, completed = 0, failed = 0, rejected = 0, cancelled = 0;
    uint64_t pairs = 0;
    std::vector<double> lat_ms, queue_ms;
    double busy_s = 0;
    sclock::time_point busy_since;
};

static size_t rec_bytes(const nf_ctx *ctx) { return ctx->cfg.out_kind == NF_OUT_FLOAT4 ? 16 : 12; }

// Finished requests kept for poll/wait/request_info before the oldest are
// forgotten (their tickets then read as unknown).
static constexpr size_t NF_SERVER_HISTORY = 1u << 16;

// A request reached a final state (s->mu held): remember it, and forget the
// oldest finished ones beyond the history bound that nobody waits on.
static void finish(nf_server *s, Req *r) {
    s->finished.push_back(r->id);
    while (s->finished.size() > NF_SERVER_HISTORY) {
        auto it = s->reqs.find(s->finished.front());
        if (it != s->reqs.end()) {
            if (it->second->waiters > 0) break;
            s->reqs.erase(it);
        }
        s->finished.pop_front();
    }
}

static void CUDART_CB on_done(void *arg) {
    Req *r = (Req *)arg;
    nf_server *s = r->srv;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        r->t_done = sclock::now();
        r->state = 2;
        r->slot_index = r->slot->index;
        r->slot->req = nullptr;
        r->slot = nullptr;
        s->completed++;
        s->pairs += r->pairs;
        s->lat_ms.push_back(std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count());
        s->queue_ms.push_back(std::chrono::duration<double, std::milli>(r->t_admit - r->t_submit).count());
        if (--s->running == 0)
            s->busy_s += std::chrono::duration<double>(r->t_done - s->busy_since).count();
        finish(s, r);
    }
    s->cv.notify_all();
    s->cv_done.notify_all();
}

// Booking for one admission: the slot to (re)allocate and idle slots whose
// buffers are released to stay within the budget.  Decided with s->mu held;
// the CUDA calls happen after the lock is dropped.
struct Booking {
    Slot *slot = nullptr;
    size_t part = 0, out = 0;  // new capacities (0: keep the slot's buffers)
    std::vector<Slot *> release;
    std::vector<void *> release_ptrs;  // their buffers, taken at booking time
};

// Device bytes of a slab request: partials (one record of nc (hi, lo) pairs per
// sink and pencil slot) and the output records.
static void request_bytes(const nf_server *s, int64_t nsink, size_t *part, size_t *out) {
    const int W = 2 * s->ctx->cfg.near_field_radius + 1;
    const int nc = s->ctx->cfg.b2 > 0.f ? 4 : 3;
    *part = (size_t)W * nc * (size_t)nsink * sizeof(Partial) + 16;
    *out = (size_t)nsink * rec_bytes(s->ctx) + 16;
}

static int64_t largest_slab(const nf_box *box) {
    const int64_t c2 = (int64_t)box->cpd * box->cpd;
    int64_t m = 0;
    for (int x = 0; x < box->cpd; x++)
        m = std::max(m, box->cell_start[(x + 1) * c2] - box->cell_start[x * c2]);
    return m;
}

// Try to book capacities gp/go for slot sl, releasing idle slots' buffers
// as needed; false (nothing changed) if the budget cannot hold them.
static bool try_book(nf_server *s, Slot &sl, size_t gp, size_t go, Booking &bk) {
    size_t held = s->held - sl.bytes() + gp + go + 256;
    std::vector<Slot *> rel;
    for (auto &o : s->slots) {
        if (held <= s->budget) break;
        if (&o == &sl || o.req || !o.part_cap) continue;
        rel.push_back(&o);
        held -= o.bytes();
    }
    if (held > s->budget) return false;
    bk.part = gp;
    bk.out = go;
    for (Slot *o : rel) {  // book the new total now; the buffers go back after the unlock
        o->part_cap = o->out_cap = 0;
        bk.release.push_back(o);
        bk.release_ptrs.insert(bk.release_ptrs.end(), {o->part, o->out, o->counters});
        o->part = nullptr;
        o->out = nullptr;
        o->counters = nullptr;
    }
    s->held = held;
    s->peak = std::max(s->peak, s->held);
    sl.part_cap = gp;  // booked; allocated by apply_booking
    sl.out_cap = go;
    return true;
}

static bool book_slot(nf_server *s, Slot &sl, const nf_box *box, size_t part_need,
                      size_t out_need, Booking &bk) {
    bk = Booking{};
    bk.slot = &sl;
    if (sl.part_cap >= part_need && sl.out_cap >= out_need && sl.counters) return true;
    // grow to the box's largest slab if the budget allows, else to this request
    size_t pm, om;
    request_bytes(s, largest_slab(box), &pm, &om);
    pm = std::max({pm, part_need, sl.part_cap});
    om = std::max({om, out_need, sl.out_cap});
    if (try_book(s, sl, pm, om, bk)) return true;
    return try_book(s, sl, std::max(part_need, sl.part_cap), std::max(out_need, sl.out_cap), bk);
}

// Carry out a booking (no lock held): stream-ordered frees and allocations
// from the server's pool.  The released slots are idle; their buffers are
// freed on their own streams, behind the work those streams last ran.
static nf_status apply_booking(nf_server *s, Booking &bk) {
    for (size_t i = 0; i < bk.release.size(); i++)
        for (int k = 0; k < 3; k++)
            if (bk.release_ptrs[3 * i + k]) cudaFreeAsync(bk.release_ptrs[3 * i + k], bk.release[i]->stream);
    if (!bk.part) return NF_OK;
    Slot &sl = *bk.slot;
    cudaStream_t st = sl.stream;
    if (sl.part) cudaFreeAsync(sl.part, st);
    if (sl.out) cudaFreeAsync(sl.out, st);
    if (sl.counters) cudaFreeAsync(sl.counters, st);
    sl.part = nullptr;
    sl.out = nullptr;
    sl.counters = nullptr;
    void *p = nullptr, *o = nullptr, *c = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&p, bk.part, s->pool, st);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync(&o, bk.out, s->pool, st);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync(&c, 256, s->pool, st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        for (void *q : {p, o, c})
            if (q) cudaFreeAsync(q, st);
        set_error("nf_server: device allocation failed within the HBM budget");
        return NF_ENOMEM;
    }
    sl.part = (Partial *)p;
    sl.out = o;
    sl.counters = (int *)c;
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
    L.eps = r->box->eps;
    nf_status st = engine_launch(ctx, L, 0.0, sl.stream);
    if (st == NF_OK) st = engine_coadd(ctx, sl.part, pl->n_range, sl.out, sl.stream, r->box->eps, r->box->d_perm,
                                          pl->p0);
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
    finish(s, r);
    s->cv_done.notify_all();
}

static void dispatcher_main(nf_server *s) {
    cudaSetDevice(s->ctx->device);
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
            finish(s, r);
            s->cv_done.notify_all();
            continue;
        }
        size_t part_need, out_need;
        request_bytes(s, pl->n_range, &part_need, &out_need);
        Slot *pick = nullptr;  // a free slot, preferring one already large enough
        for (auto &sl : s->slots)
            if (!sl.req && (!pick || (sl.part_cap >= part_need && pick->part_cap < part_need)))
                pick = &sl;
        Booking bk;
        if (!pick || !book_slot(s, *pick, r->box, part_need, out_need, bk)) {
            if (s->running == 0) {  // nothing in flight will free memory
                s->pending.pop_front();
                r->state = -1;
                r->status = NF_EADMISSION;
                s->rejected++;
                finish(s, r);
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
        st = apply_booking(s, bk);
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
    // two slots by default: one request running and the next already queued
    // on the device behind it.  More slots overlap persistent launches that
    // share the GPU, which stretches every request's run time.
    if (s->cfg.max_inflight <= 0) s->cfg.max_inflight = 2;
    if (s->cfg.max_queued <= 0) s->cfg.max_queued = 65536;
    if (s->cfg.max_inflight > 256) {
        set_error("nf_server_start: max_inflight above 256");
        return NF_EINVAL;
    }
    size_t freeb = 0, total = 0;
    NF_CUDA(cudaMemGetInfo(&freeb, &total));
    s->budget = s->cfg.hbm_budget_bytes ? s->cfg.hbm_budget_bytes : (size_t)(0.9 * (double)freeb);
    // the slots' memory pool: freed blocks stay in the pool (up to the
    // budget) for the next growth instead of going back to the driver
    cudaMemPoolProps pp{};
    pp.allocType = cudaMemAllocationTypePinned;
    pp.location.type = cudaMemLocationTypeDevice;
    pp.location.id = ctx->device;
    NF_CUDA(cudaMemPoolCreate(&s->pool, &pp));
    uint64_t keep = s->budget;
    cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    s->t_start = sclock::now();
    s->slots.resize(s->cfg.max_inflight);
    for (int i = 0; i < s->cfg.max_inflight; i++) {
        s->slots[i].index = i;
        cudaError_t e = cudaStreamCreateWithFlags(&s->slots[i].stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            for (auto &sl : s->slots)
                if (sl.stream) cudaStreamDestroy(sl.stream);
            cudaMemPoolDestroy(s->pool);
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
    int64_t c2 = (int64_t)box->cpd * box->cpd;
    size_t pb, ob;
    request_bytes(s, box->cell_start[(slab + 1) * c2] - box->cell_start[slab * c2], &pb, &ob);
    size_t need = pb + ob + 256;
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
    r->waiters++;  // keeps the record while this thread sleeps
    bool ok = s->cv_done.wait_for(lk, std::chrono::nanoseconds(timeout_ns),
                                  [&] { return r->state == 2 || r->state < 0; });
    r->waiters--;
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
    finish(s, r);
    s->cv_done.notify_all();
    return NF_OK;
}

extern "C" nf_status nf_server_request_info(nf_server *s, nf_ticket t, nf_request_info *info) {
    if (!s || !info) {
        set_error("nf_server_request_info: null argument");
        return NF_EINVAL;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(t);
    if (it == s->reqs.end()) {
        set_error("nf_server_request_info: unknown ticket");
        return NF_EINVAL;
    }
    const Req *r = it->second.get();
    auto ms = [](sclock::time_point a, sclock::time_point b) {
        return std::chrono::duration<double, std::milli>(b - a).count();
    };
    memset(info, 0, sizeof(*info));
    info->state = r->state;
    info->status = r->status;
    info->slab = r->slab;
    info->slot = r->slot ? r->slot->index : r->slot_index;
    info->pairs = r->pairs;
    info->submit_ms = ms(s->t_start, r->t_submit);
    const bool admitted = r->state == 1 || r->state == 2 || (r->state == -1 && r->pairs);
    info->queue_ms = admitted ? ms(r->t_submit, r->t_admit) : -1.0;
    info->run_ms = r->state == 2 ? ms(r->t_admit, r->t_done) : -1.0;
    info->total_ms = r->state == 2 ? ms(r->t_submit, r->t_done) : -1.0;
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
        if (!sl.stream) continue;
        for (void *q : {(void *)sl.part, sl.out, (void *)sl.counters})
            if (q) cudaFreeAsync(q, sl.stream);
        cudaStreamSynchronize(sl.stream);
        cudaStreamDestroy(sl.stream);
    }
    if (s->pool) cudaMemPoolDestroy(s->pool);
    delete s;
}
