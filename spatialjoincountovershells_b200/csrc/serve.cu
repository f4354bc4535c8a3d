// Serving loop: halo-query requests of uneven size against device-resident
// particle indexes, admitted by free device memory and run concurrently.
//
// A dispatcher thread owns K slots, one CUDA stream each.  A request waits in
// a FIFO until a slot is free and its device-memory need (halos, sorted
// halos, sort scratch, counts) fits in what the running requests leave of the
// budget; it is then admitted: its halos are copied in, prepared (radius
// table, shell lookup, Morton sort), counted against every index and its u32
// counts copied back, all on the slot's stream, so admitted requests overlap
// on the device (continuous batching: a request arriving while others run is
// admitted as soon as a slot and memory free up, not when the batch drains).
// Completion is detected by polling the slot's event; latency is measured on
// the host clock from submission to detected completion.
//
// The reference has no serving mode; each request computes exactly what
// sjcs_query_create + sjcs_query_count per index + read-back compute (same
// kernels, same arithmetic), so a request's counts do not depend on what else
// runs beside it.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "sjcs_internal.cuh"

namespace sjcs {
namespace {

double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

bool pinned(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

struct Request {
    uint64_t ticket = 0;
    const float* halo_xyz = nullptr;
    size_t stride = 12;
    uint64_t nhalos = 0;
    std::vector<float> r2;
    int flags = 0;
    uint32_t* out = nullptr;
    bool out_pinned = false;
    uint64_t mem = 0;
    double t_submit = 0, t_admit = 0, t_done = 0;
    int status = SJCS_OK;
    std::string msg;  // error message of a failed request
    bool done = false;
};

struct Slot {
    cudaStream_t s = nullptr;
    cudaEvent_t ev_done = nullptr;
    Request* req = nullptr;
    sjcs_query q{};
    float* d_raw = nullptr;
    uint32_t* stage = nullptr;  // pinned staging of counts for pageable outputs
    size_t stage_elems = 0;
};

}  // namespace
}  // namespace sjcs

struct sjcs_server {
    uint32_t magic;
    sjcs_ctx* ctx;
    std::vector<const sjcs_index*> idx;
    std::vector<sjcs::Slot> slots;
    uint64_t budget = 0, in_use = 0, peak = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<sjcs::Request*> queue;
    std::map<uint64_t, sjcs::Request*> reqs;
    uint64_t next_ticket = 1;
    uint64_t submitted = 0, completed = 0;
    uint32_t inflight = 0, max_inflight = 0;
    bool stop = false;
    std::thread th;
};

namespace sjcs {
namespace {

constexpr uint32_t kServerMagic = 0x534a5653u;  // "SJVS"

bool valid_server(const sjcs_server* s) { return s && s->magic == kServerMagic; }

uint64_t request_bytes(uint64_t nhalos, size_t stride, int nrads) {
    // per halo: raw halo + sorted halo + Morton sort records (2 x (4 + 16) B)
    // + counts + queue-schedule scratch (12 B) + sort histogram (1 B);
    // fixed: radius table, shell lookup table, scan partials
    return nhalos * (uint64_t)(stride + 16 + 40 + 4 * (uint64_t)nrads + 13) + 65536 + 8 * (uint64_t)nrads;
}

// Queue one admitted request's work on its slot's stream (dispatcher thread, unlocked).
int enqueue(sjcs_server* srv, Slot& sl) {
    Request* r = sl.req;
    cudaStream_t s = sl.s;
    const uint64_t n = r->nhalos;
    const int nrads = (int)r->r2.size();
    sl.q = sjcs_query{};
    sl.q.magic = 0;  // internal: never handed out
    sl.q.ctx = srv->ctx;
    sl.d_raw = nullptr;
    const size_t raw_bytes = n ? (size_t)((n - 1) * r->stride + 12) : 16;
    SJCS_CUDA_TRY(cudaMallocAsync(&sl.d_raw, raw_bytes, s));
    if (n) SJCS_CUDA_TRY(cudaMemcpyAsync(sl.d_raw, r->halo_xyz, raw_bytes, cudaMemcpyHostToDevice, s));
    int rc = query_prepare(srv->ctx, sl.d_raw, r->stride, n, r->r2.data(), nrads, r->flags, &sl.q, s);
    if (rc) return rc;
    if (n) {
        std::lock_guard<std::mutex> lk(srv->ctx->mu);  // launch set-up and the tuned-schedule cache
        // grid indexes of one cell grid under the static schedule: one fused
        // pass (each halo planned once for all of them)
        const size_t k = srv->idx.size();
        bool fuse = k >= 2 && k <= (size_t)kMaxFusedIndexes;
        for (size_t i = 0; fuse && i < k; ++i) {
            const sjcs_index* a = srv->idx[0];
            const sjcs_index* b = srv->idx[i];
            fuse = b->kind == SJCS_INDEX_GRID && b->geom.ncells == a->geom.ncells && b->geom.G[0] == a->geom.G[0] &&
                   b->geom.G[1] == a->geom.G[1] && b->geom.G[2] == a->geom.G[2];
        }
        if (fuse) fuse = schedule_for(srv->ctx, &sl.q, srv->idx[0]).mode != SJCS_SCHED_QUEUE;
        if (fuse) {
            rc = launch_shell_count_multi(srv->ctx, &sl.q, srv->idx.data(), (int)k, s);
            if (rc) return rc;
        } else {
            for (const sjcs_index* ix : srv->idx) {
                const Schedule sc = schedule_for(srv->ctx, &sl.q, ix);
                rc = ix->kind == SJCS_INDEX_GRID ? launch_shell_count(srv->ctx, &sl.q, ix, s, &sc)
                                                 : launch_morton_count(srv->ctx, &sl.q, ix, s, &sc);
                if (rc) return rc;
            }
        }
    }
    const size_t cnt = (size_t)n * (size_t)nrads;
    if (cnt) {
        uint32_t* dst = r->out;
        if (!r->out_pinned) {
            if (sl.stage_elems < cnt) {
                if (sl.stage) cudaFreeHost(sl.stage);
                sl.stage = nullptr;
                sl.stage_elems = 0;
                SJCS_CUDA_TRY(cudaMallocHost(&sl.stage, cnt * sizeof(uint32_t)));
                sl.stage_elems = cnt;
            }
            dst = sl.stage;
        }
        SJCS_CUDA_TRY(cudaMemcpyAsync(dst, sl.q.counts, cnt * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    }
    cudaFreeAsync(sl.d_raw, s);
    cudaFreeAsync(sl.q.halos, s);
    cudaFreeAsync(sl.q.counts, s);
    cudaFreeAsync(sl.q.d_r2, s);
    if (sl.q.d_lut) cudaFreeAsync(sl.q.d_lut, s);
    SJCS_CUDA_TRY(cudaEventRecord(sl.ev_done, s));
    return SJCS_OK;
}

// Free what a failed enqueue left allocated on the slot's stream.
void release_partial(Slot& sl) {
    cudaStream_t s = sl.s;
    if (sl.d_raw) cudaFreeAsync(sl.d_raw, s);
    if (sl.q.halos) cudaFreeAsync(sl.q.halos, s);
    if (sl.q.counts) cudaFreeAsync(sl.q.counts, s);
    if (sl.q.d_r2) cudaFreeAsync(sl.q.d_r2, s);
    if (sl.q.d_lut) cudaFreeAsync(sl.q.d_lut, s);
    cudaGetLastError();
}

// The dispatcher holds the server mutex only while it changes shared state;
// copies, launches and result copies run unlocked (slots belong to this
// thread alone, and a request's fields are its own until `done` is set).
void dispatcher(sjcs_server* srv) {
    cudaSetDevice(srv->ctx->device);
    std::unique_lock<std::mutex> lk(srv->mu);
    std::vector<Slot*> finished, admitted;
    for (;;) {
        // completions
        finished.clear();
        for (Slot& sl : srv->slots)
            if (sl.req && cudaEventQuery(sl.ev_done) != cudaErrorNotReady) finished.push_back(&sl);
        if (!finished.empty()) {
            lk.unlock();
            for (Slot* sl : finished) {
                Request* r = sl->req;
                const cudaError_t e = cudaEventQuery(sl->ev_done);
                if (e != cudaSuccess && r->status == SJCS_OK) {
                    r->status = SJCS_ERR_CUDA;
                    r->msg = std::string("request failed on the device: ") + cudaGetErrorString(e);
                } else if (r->status == SJCS_OK && !r->out_pinned && r->nhalos) {
                    std::memcpy(r->out, sl->stage, (size_t)r->nhalos * r->r2.size() * sizeof(uint32_t));
                }
            }
            lk.lock();
            for (Slot* sl : finished) {
                Request* r = sl->req;
                r->t_done = now_ms();
                r->done = true;
                sl->req = nullptr;
                srv->in_use -= r->mem;
                --srv->inflight;
                ++srv->completed;
            }
            srv->cv_done.notify_all();
        }
        // admissions, first come first served
        admitted.clear();
        for (Slot& sl : srv->slots) {
            if (sl.req || srv->queue.empty()) continue;
            Request* r = srv->queue.front();
            if (srv->inflight > 0 && srv->in_use + r->mem > srv->budget) break;  // wait for memory
            srv->queue.pop_front();
            sl.req = r;
            r->t_admit = now_ms();
            srv->in_use += r->mem;
            srv->peak = std::max(srv->peak, srv->in_use);
            ++srv->inflight;
            srv->max_inflight = std::max(srv->max_inflight, srv->inflight);
            admitted.push_back(&sl);
        }
        if (!admitted.empty()) {
            lk.unlock();
            for (Slot* sl : admitted) {
                const int rc = enqueue(srv, *sl);
                if (rc) {
                    // it completes with its error once the stream has drained
                    sl->req->status = rc;
                    sl->req->msg = sjcs_last_error();
                    release_partial(*sl);
                    cudaEventRecord(sl->ev_done, sl->s);
                }
            }
            lk.lock();
        }
        if (srv->stop && srv->queue.empty() && srv->inflight == 0) break;
        if (finished.empty() && admitted.empty()) {
            // in flight: poll again shortly; idle: sleep until a submission
            if (srv->inflight) srv->cv_work.wait_for(lk, std::chrono::microseconds(50));
            else srv->cv_work.wait_for(lk, std::chrono::milliseconds(20));
        }
    }
}

}  // namespace
}  // namespace sjcs

using namespace sjcs;

extern "C" {

int sjcs_server_create(sjcs_ctx* ctx, sjcs_index* const* indexes, int nindexes, const sjcs_server_opts* opts,
                       sjcs_server** out) {
    if (!ctx || ctx->magic != kCtxMagic) return fail(SJCS_ERR_STATE, "invalid context");
    if (!out) return fail(SJCS_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (nindexes < 0 || (nindexes && !indexes)) return fail(SJCS_ERR_INVALID, "bad index list");
    for (int i = 0; i < nindexes; ++i)
        if (!indexes[i] || indexes[i]->magic != kIndexMagic || indexes[i]->ctx != ctx)
            return fail(SJCS_ERR_STATE, "index %d does not belong to this context", i);
    sjcs_server_opts o{};
    if (opts) o = *opts;
    for (int i = 0; i < 4; ++i)
        if (o.reserved[i]) return fail(SJCS_ERR_INVALID, "reserved option fields must be zero");
    if (o.slots > 64) return fail(SJCS_ERR_INVALID, "at most 64 slots");
    SJCS_CUDA_TRY(cudaSetDevice(ctx->device));
    // the indexes must be built before any request reads them
    for (int i = 0; i < nindexes; ++i) SJCS_CUDA_TRY(cudaEventSynchronize(indexes[i]->ev_ready));
    sjcs_server* srv = new (std::nothrow) sjcs_server();
    if (!srv) return fail(SJCS_ERR_NOMEM, "out of host memory");
    srv->magic = kServerMagic;
    srv->ctx = ctx;
    srv->idx.assign(indexes, indexes + nindexes);
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    srv->budget = o.mem_budget ? o.mem_budget : (uint64_t)(0.8 * (double)free_b);
    srv->slots.resize(o.slots ? o.slots : 4);
    for (Slot& sl : srv->slots) {
        cudaStreamCreateWithFlags(&sl.s, cudaStreamNonBlocking);
        cudaEventCreateWithFlags(&sl.ev_done, cudaEventDisableTiming);
    }
    srv->th = std::thread(dispatcher, srv);
    *out = srv;
    return SJCS_OK;
}

int sjcs_server_submit(sjcs_server* srv, const float* halo_xyz, size_t stride_bytes, uint64_t nhalos,
                       const float* r2, int nrads, int flags, uint32_t* out_counts, uint64_t* ticket) {
    if (!valid_server(srv)) return fail(SJCS_ERR_STATE, "invalid server");
    if (!ticket) return fail(SJCS_ERR_INVALID, "ticket is NULL");
    if (nhalos && (!halo_xyz || !out_counts)) return fail(SJCS_ERR_INVALID, "halo_xyz or out_counts is NULL");
    if (!r2 || nrads <= 0) return fail(SJCS_ERR_INVALID, "radius table is empty");
    if (stride_bytes < 12 || stride_bytes % 4) return fail(SJCS_ERR_INVALID, "stride_bytes must be a multiple of 4 and >= 12");
    if (nhalos > 0xffffffffull) return fail(SJCS_ERR_INVALID, "too many halos");
    if (flags & ~SJCS_QUERY_PERIODIC) return fail(SJCS_ERR_INVALID, "unknown query flags 0x%x", flags);
    {
        // the request's counts are summed over every index into uint32
        uint64_t bound = 0;
        for (const sjcs_index* ix : srv->idx) bound += count_call_bound(flags, r2[nrads - 1], ix->n);
        if (bound > 0xffffffffull)
            return fail(SJCS_ERR_INVALID,
                        "the request's counts could reach %llu, beyond its uint32 output; serve fewer particles",
                        (unsigned long long)bound);
    }
    Request* r = new (std::nothrow) Request();
    if (!r) return fail(SJCS_ERR_NOMEM, "out of host memory");
    r->halo_xyz = halo_xyz;
    r->stride = stride_bytes;
    r->nhalos = nhalos;
    r->r2.assign(r2, r2 + nrads);
    r->flags = flags;
    r->out = out_counts;
    r->out_pinned = nhalos && pinned(out_counts);
    r->mem = request_bytes(nhalos, stride_bytes, nrads);
    r->t_submit = now_ms();
    std::lock_guard<std::mutex> lk(srv->mu);
    if (r->mem > srv->budget) {
        const uint64_t need = r->mem, budget = srv->budget;
        delete r;
        return fail(SJCS_ERR_NOMEM, "request needs %llu device bytes; the server's budget is %llu",
                    (unsigned long long)need, (unsigned long long)budget);
    }
    r->ticket = srv->next_ticket++;
    srv->reqs[r->ticket] = r;
    srv->queue.push_back(r);
    ++srv->submitted;
    *ticket = r->ticket;
    srv->cv_work.notify_one();
    return SJCS_OK;
}

int sjcs_server_wait(sjcs_server* srv, uint64_t ticket, sjcs_request_info* info) {
    if (!valid_server(srv)) return fail(SJCS_ERR_STATE, "invalid server");
    std::unique_lock<std::mutex> lk(srv->mu);
    auto it = srv->reqs.find(ticket);
    if (it == srv->reqs.end()) return fail(SJCS_ERR_INVALID, "unknown ticket %llu", (unsigned long long)ticket);
    Request* r = it->second;
    srv->cv_done.wait(lk, [&] { return r->done; });
    if (info) {
        info->queue_ms = r->t_admit - r->t_submit;
        info->service_ms = r->t_done - r->t_admit;
        info->latency_ms = r->t_done - r->t_submit;
        info->status = r->status;
    }
    const int st = r->status;
    const std::string msg = r->msg;
    srv->reqs.erase(it);
    delete r;
    if (st) return fail(st, "%s", msg.c_str());
    return SJCS_OK;
}

int sjcs_server_stats(sjcs_server* srv, sjcs_server_info* out) {
    if (!valid_server(srv) || !out) return fail(SJCS_ERR_INVALID, "invalid argument");
    std::lock_guard<std::mutex> lk(srv->mu);
    sjcs_server_info s{};
    s.submitted = srv->submitted;
    s.completed = srv->completed;
    s.queued = srv->queue.size();
    s.inflight = srv->inflight;
    s.max_inflight = srv->max_inflight;
    s.slots = (uint32_t)srv->slots.size();
    s.budget_bytes = srv->budget;
    s.in_use_bytes = srv->in_use;
    s.peak_bytes = srv->peak;
    *out = s;
    return SJCS_OK;
}

int sjcs_server_destroy(sjcs_server* srv) {
    if (!valid_server(srv)) return fail(SJCS_ERR_STATE, "invalid server");
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->stop = true;
        srv->cv_work.notify_one();
    }
    srv->th.join();  // drains every submitted request
    cudaSetDevice(srv->ctx->device);
    for (Slot& sl : srv->slots) {
        cudaStreamSynchronize(sl.s);
        if (sl.stage) cudaFreeHost(sl.stage);
        cudaEventDestroy(sl.ev_done);
        cudaStreamDestroy(sl.s);
    }
    for (auto& kv : srv->reqs) delete kv.second;  // completed but never waited for
    srv->magic = 0;
    delete srv;
    return SJCS_OK;
}

}  // extern "C"
