// extern "C" entry points of libsjcs.so (declared in include/sjcs.h).
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "morton.cuh"
#include "sjcs_internal.cuh"

namespace sjcs {

static thread_local std::string g_last_error;
static std::atomic<uint64_t> g_launches{0};

void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

void set_error(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
}

int fail(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

namespace {

// out = the 64-bit totals: the u32 accumulators plus, after a fold, the
// folded part (folded == nullptr: none yet).
__global__ void k_widen_u32_u64(const uint32_t* __restrict__ in, uint64_t m,
                                const unsigned long long* __restrict__ folded, unsigned long long* __restrict__ out) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride)
        out[i] = (unsigned long long)in[i] + (folded ? folded[i] : 0ull);
}

// One fold: the 64-bit totals take the u32 accumulators, which restart at 0.
__global__ void k_fold_counts(uint32_t* __restrict__ c32, uint64_t m, unsigned long long* __restrict__ c64) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        c64[i] += c32[i];
        c32[i] = 0u;
    }
}

__global__ void k_fill_f32(float* __restrict__ p, uint64_t m, float v) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) p[i] = v;
}

bool valid_ctx(const sjcs_ctx* c) { return c && c->magic == kCtxMagic; }
bool valid_index(const sjcs_index* i) { return i && i->magic == kIndexMagic; }
bool valid_query(const sjcs_query* q) { return q && q->magic == kQueryMagic; }

int set_device(const sjcs_ctx* ctx) {
    SJCS_CUDA_TRY(cudaSetDevice(ctx->device));
    return SJCS_OK;
}

bool is_pinned(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// Parallel host copy/add of a widened chunk into the caller's array.
void host_store(uint64_t* dst, const uint64_t* src, uint64_t m, bool add) {
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const unsigned nt = (m < (1u << 20)) ? 1u : hw;
    auto work = [&](unsigned t) {
        const uint64_t lo = m * t / nt, hi = m * (t + 1) / nt;
        if (add)
            for (uint64_t i = lo; i < hi; ++i) dst[i] += src[i];
        else
            std::memcpy(dst + lo, src + lo, (hi - lo) * sizeof(uint64_t));
    };
    if (nt == 1) {
        work(0);
        return;
    }
    std::vector<std::thread> th;
    th.reserve(nt);
    for (unsigned t = 0; t < nt; ++t) th.emplace_back(work, t);
    for (auto& x : th) x.join();
}

// Shell lookup table over the bit patterns of squared distances (see
// sjcs_query::d_lut).  Built only for strictly increasing, finite,
// non-negative tables whose closest pair of values is far enough apart in bit
// space to give at most 4096 slots; otherwise the kernel binary-searches.
void build_shell_lut(const float* r2, int nrads, std::vector<uint32_t>* lut, uint32_t* k0_out, int* shift_out) {
    constexpr size_t kMaxSlots = 4096;
    lut->clear();
    if (nrads < 2) return;
    uint32_t prev = 0;
    uint32_t min_gap = 0xffffffffu;
    for (int i = 0; i < nrads; ++i) {
        if (!std::isfinite(r2[i])) return;
        uint32_t b;
        std::memcpy(&b, &r2[i], 4);
        if (b & 0x80000000u) return;  // negative or -0.0: bit order is not value order
        if (i > 0) {
            if (b <= prev) return;  // repeated value
            min_gap = std::min(min_gap, b - prev);
        }
        prev = b;
    }
    uint32_t k0, kmax;
    std::memcpy(&k0, &r2[0], 4);
    std::memcpy(&kmax, &r2[nrads - 1], 4);
    int shift = 0;
    while (shift < 31 && (2u << shift) <= min_gap) ++shift;  // 2^shift <= min_gap
    const uint64_t nslots = ((uint64_t)(kmax - 1 - k0) >> shift) + 1;
    if (nslots > kMaxSlots) return;
    lut->resize(nslots);
    for (uint64_t j = 0; j < nslots; ++j) {
        const uint32_t key = k0 + (uint32_t)(j << shift);
        float v;
        std::memcpy(&v, &key, 4);
        (*lut)[j] = (uint32_t)(std::upper_bound(r2, r2 + nrads, v) - r2);  // #{r2[i] <= v}
    }
    *k0_out = k0;
    *shift_out = shift;
}

}  // namespace

constexpr uint32_t kParamSlots = 8;
constexpr size_t kParamSlotBytes = 64 << 10;

// Copy `bytes` of host memory to dst on stream s without the host waiting for
// s: through a page-locked slot of the context (the slot's previous copy is
// long done unless 8 newer ones are still queued); larger tables fall back to
// a pageable copy.
int upload_params(sjcs_ctx* ctx, void* dst, const void* src, size_t bytes, cudaStream_t s) {
    if (bytes == 0) return SJCS_OK;
    if (bytes > kParamSlotBytes) {
        SJCS_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
        return SJCS_OK;
    }
    std::lock_guard<std::mutex> lk(ctx->param_mu);
    if (!ctx->param_ring) {
        SJCS_CUDA_TRY(cudaMallocHost(&ctx->param_ring, kParamSlots * kParamSlotBytes));
        ctx->param_ev.assign(kParamSlots, nullptr);
        for (auto& e : ctx->param_ev) SJCS_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    const uint32_t slot = ctx->param_next++ % kParamSlots;
    char* p = ctx->param_ring + (size_t)slot * kParamSlotBytes;
    SJCS_CUDA_TRY(cudaEventSynchronize(ctx->param_ev[slot]));
    std::memcpy(p, src, bytes);
    SJCS_CUDA_TRY(cudaMemcpyAsync(dst, p, bytes, cudaMemcpyHostToDevice, s));
    SJCS_CUDA_TRY(cudaEventRecord(ctx->param_ev[slot], s));
    return SJCS_OK;
}

int query_prepare(sjcs_ctx* ctx, const float* d_halo_xyz, size_t stride, uint64_t nhalos, const float* r2,
                  int nrads, int flags, sjcs_query* q, cudaStream_t s) {
    q->nhalos = nhalos;
    q->nrads = nrads;
    q->flags = flags;
    int pad = 1;
    while (pad < nrads) pad <<= 1;
    q->pad = pad;
    bool mono = true;
    for (int i = 0; i < nrads; ++i) {
        if (std::isnan(r2[i])) mono = false;
        if (i + 1 < nrads && !(r2[i] <= r2[i + 1])) mono = false;
    }
    q->monotone = mono;
    q->r2max = r2[nrads - 1];
    q->R = (float)std::sqrt((double)r2[nrads - 1]);
    q->half = (flags & SJCS_QUERY_PERIODIC) ? q->R : r2[nrads - 1];
    SJCS_CUDA_TRY(cudaMallocAsync(&q->d_r2, (size_t)pad * sizeof(float), s));
    k_fill_f32<<<(pad + 255) / 256, 256, 0, s>>>(q->d_r2, (uint64_t)pad, INFINITY);
    SJCS_LAUNCH_CHECK();
    int rc = upload_params(ctx, q->d_r2, r2, (size_t)nrads * sizeof(float), s);
    if (rc) return rc;
    std::vector<uint32_t> lut;
    if (mono) build_shell_lut(r2, nrads, &lut, &q->lut_k0, &q->lut_shift);
    q->nlut = (int)lut.size();
    if (!lut.empty()) {
        SJCS_CUDA_TRY(cudaMallocAsync(&q->d_lut, lut.size() * sizeof(uint32_t), s));
        rc = upload_params(ctx, q->d_lut, lut.data(), lut.size() * sizeof(uint32_t), s);
        if (rc) return rc;
    }
    const uint64_t ncnt = nhalos * (uint64_t)nrads;
    SJCS_CUDA_TRY(cudaMallocAsync(&q->counts, (ncnt ? ncnt : 1) * sizeof(uint32_t), s));
    if (ncnt) SJCS_CUDA_TRY(cudaMemsetAsync(q->counts, 0, ncnt * sizeof(uint32_t), s));
    SJCS_CUDA_TRY(cudaMallocAsync(&q->halos, (nhalos ? nhalos : 1) * sizeof(float4), s));
    return sort_halos(ctx, d_halo_xyz, stride, nhalos, q->halos, s);
}

namespace {

int check_query_args(sjcs_ctx* ctx, const float* halo_xyz, size_t stride, uint64_t nhalos, const float* r2,
                     int nrads, int flags, sjcs_query** out) {
    if (!valid_ctx(ctx)) return fail(SJCS_ERR_STATE, "invalid context");
    if (!out) return fail(SJCS_ERR_INVALID, "out is NULL");
    if (nhalos && !halo_xyz) return fail(SJCS_ERR_INVALID, "halo_xyz is NULL");
    if (!r2 || nrads <= 0) return fail(SJCS_ERR_INVALID, "radius table is empty");
    if (stride < 3 * sizeof(float) || (stride % sizeof(float)) != 0)
        return fail(SJCS_ERR_INVALID, "stride_bytes must be a multiple of 4 and >= 12 (got %zu)", stride);
    if (nhalos > 0xffffffffull) return fail(SJCS_ERR_INVALID, "too many halos (%llu)", (unsigned long long)nhalos);
    if (flags & ~SJCS_QUERY_PERIODIC) return fail(SJCS_ERR_INVALID, "unknown query flags 0x%x", flags);
    return SJCS_OK;
}

void clear_count_events(sjcs_query* q) {
    for (cudaEvent_t e : q->count_events) cudaEventDestroy(e);
    q->count_events.clear();
}

sjcs_query* new_query(sjcs_ctx* ctx) {
    sjcs_query* q = new (std::nothrow) sjcs_query();
    if (!q) return nullptr;
    q->magic = kQueryMagic;
    q->ctx = ctx;
    cudaEventCreate(&q->ev_last);
    cudaEventCreate(&q->ev_d0);
    cudaEventCreate(&q->ev_d1);
    cudaEventCreateWithFlags(&q->ev_rq, cudaEventDisableTiming);
    return q;
}

// Work that writes or frees q's counts waits, on stream s, for an
// asynchronous read of them (a no-op once the read has finished).
cudaError_t after_reads(const sjcs_query* q, cudaStream_t s) {
    return q->read_queued ? cudaStreamWaitEvent(s, q->ev_d1, 0) : cudaSuccess;
}

// Before a count call that can add up to `add` to an accumulator: fold the
// u32 accumulators into the 64-bit totals (on stream s) if the call could
// otherwise carry one past q->fold_limit.  Called after after_reads(q, s).
int fold_before_count(sjcs_ctx* ctx, sjcs_query* q, uint64_t add, cudaStream_t s) {
    if (add > q->fold_limit)
        return fail(SJCS_ERR_INVALID,
                    "one count call could add %llu to a 32-bit accumulator (limit %llu): use indexes of fewer "
                    "particles",
                    (unsigned long long)add, (unsigned long long)q->fold_limit);
    if (q->bound + add <= q->fold_limit) {
        q->bound += add;
        return SJCS_OK;
    }
    const uint64_t m = q->nhalos * (uint64_t)q->nrads;
    if (m) {
        if (!q->counts64) {
            SJCS_CUDA_TRY(cudaMallocAsync(&q->counts64, m * sizeof(unsigned long long), s));
            SJCS_CUDA_TRY(cudaMemsetAsync(q->counts64, 0, m * sizeof(unsigned long long), s));
        }
        k_fold_counts<<<ctx->num_sms * 8, 256, 0, s>>>(q->counts, m, q->counts64);
        SJCS_LAUNCH_CHECK();
    }
    ++q->folds;
    q->bound = add;
    return SJCS_OK;
}

void free_query(sjcs_query* q) {
    if (!q) return;
    cudaStream_t s = q->ctx->s_count;
    after_reads(q, s);
    if (q->halos) cudaFreeAsync(q->halos, s);
    if (q->counts) cudaFreeAsync(q->counts, s);
    if (q->counts64) cudaFreeAsync(q->counts64, s);
    if (q->d_r2) cudaFreeAsync(q->d_r2, s);
    if (q->d_lut) cudaFreeAsync(q->d_lut, s);
    cudaStreamSynchronize(s);
    if (q->h_stage) cudaFreeHost(q->h_stage);
    clear_count_events(q);
    cudaEventDestroy(q->ev_last);
    cudaEventDestroy(q->ev_d0);
    cudaEventDestroy(q->ev_d1);
    cudaEventDestroy(q->ev_rq);
    q->magic = 0;
    delete q;
}

sjcs_index* new_index(sjcs_ctx* ctx) {
    sjcs_index* idx = new (std::nothrow) sjcs_index();
    if (!idx) return nullptr;
    idx->magic = kIndexMagic;
    idx->ctx = ctx;
    cudaEventCreate(&idx->ev_start);
    cudaEventCreate(&idx->ev_h2d);
    cudaEventCreate(&idx->ev_ready);
    cudaEventCreate(&idx->ev_train0);
    return idx;
}

void free_index(sjcs_index* idx) {
    if (!idx) return;
    sjcs_ctx* ctx = idx->ctx;
    // Frees are ordered after the build (build stream) and after every count
    // queued on the count stream that reads this index.
    cudaStreamWaitEvent(ctx->s_count, idx->ev_ready, 0);
    if (idx->pts) cudaFreeAsync(idx->pts, ctx->s_count);
    if (idx->cell_start) cudaFreeAsync(idx->cell_start, ctx->s_count);
    if (idx->leaves) cudaFreeAsync(idx->leaves, ctx->s_count);
    if (idx->root) cudaFreeAsync(idx->root, ctx->s_count);
    cudaEventDestroy(idx->ev_train0);
    cudaEventDestroy(idx->ev_start);
    cudaEventDestroy(idx->ev_h2d);
    cudaEventDestroy(idx->ev_ready);
    idx->magic = 0;
    delete idx;
}

// Unless builds may overlap counts: the build kernels queued next on s wait
// for every count queued so far (the copies queued before them do not).
void order_after_counts(sjcs_ctx* ctx, cudaStream_t s) {
    if (ctx->overlap || !ctx->ev_counts) return;
    if (cudaEventRecord(ctx->ev_counts, ctx->s_count) == cudaSuccess) cudaStreamWaitEvent(s, ctx->ev_counts, 0);
    cudaGetLastError();
}

// Validated copy of the build options.
int check_opts(const sjcs_index_opts* opts, sjcs_index_opts* o_out) {
    sjcs_index_opts o{};
    if (opts) o = *opts;
    if (o.kind != SJCS_INDEX_GRID && o.kind != SJCS_INDEX_LEARNED && o.kind != SJCS_INDEX_MORTON)
        return fail(SJCS_ERR_INVALID, "unsupported index kind %d", o.kind);
    for (int i = 0; i < 3; ++i)
        if (o.reserved[i]) return fail(SJCS_ERR_INVALID, "reserved option fields must be zero");
    if (o.flags & ~(uint32_t)SJCS_INDEX_VERIFY) return fail(SJCS_ERR_INVALID, "unknown index flags 0x%x", o.flags);
    if (!(o.radius_hint >= 0.0f)) return fail(SJCS_ERR_INVALID, "radius_hint must be >= 0");
    const bool morton = o.kind != SJCS_INDEX_GRID;
    if (morton && (o.grid[0] > (uint32_t)kMaxMortonLevel || o.grid[1] || o.grid[2]))
        return fail(SJCS_ERR_INVALID, "Morton index: grid[0] is the cell level (0 = automatic, 1..%d), grid[1] and grid[2] must be zero",
                    kMaxMortonLevel);
    if (!morton && (o.grid[0] || o.grid[1] || o.grid[2]) &&
        (!o.grid[0] || !o.grid[1] || !o.grid[2] || o.grid[0] > 65535 || o.grid[1] > 65535 || o.grid[2] > 65535 ||
         (uint64_t)o.grid[0] * o.grid[1] * o.grid[2] > (1ull << 31)))
        return fail(SJCS_ERR_INVALID, "grid must be all zero or three values in [1,65535] with <= 2^31 cells");
    *o_out = o;
    return SJCS_OK;
}

// Queue the build kernels of an index over device particles on stream s.
int enqueue_build(sjcs_ctx* ctx, sjcs_index* idx, const float* d_xyz, uint64_t n, const sjcs_index_opts& o,
                  cudaStream_t s) {
    if (o.kind != SJCS_INDEX_GRID) {
        const int level = o.grid[0] ? (int)o.grid[0] : morton_auto_level(n, o.radius_hint);
        return build_morton_index(ctx, d_xyz, n, level, o.kind == SJCS_INDEX_LEARNED,
                                  (o.flags & SJCS_INDEX_VERIFY) != 0, idx, s);
    }
    return build_grid_index(ctx, d_xyz, n, auto_grid(n, o.radius_hint, o.grid), idx, s);
}

// Copy a host file to new device memory on the upload stream and make the
// build stream wait for it: uploads of later files never queue behind builds
// that wait for counts, so the copy engine stays busy.  idx's ev_start and
// ev_h2d bracket the copy.  The caller frees *d on the build stream.
int upload(sjcs_ctx* ctx, sjcs_index* idx, const void* host, size_t bytes, void** d) {
    cudaStream_t u = ctx->s_h2d;
    *d = nullptr;
    cudaEventRecord(idx->ev_start, u);
    cudaError_t e = cudaMallocAsync(d, bytes, u);
    if (e != cudaSuccess) {
        *d = nullptr;
        cudaGetLastError();
        return fail(SJCS_ERR_NOMEM, "device allocation of %llu bytes for the upload failed: %s",
                    (unsigned long long)bytes, cudaGetErrorString(e));
    }
    e = cudaMemcpyAsync(*d, host, bytes, cudaMemcpyHostToDevice, u);
    if (e == cudaSuccess) e = cudaEventRecord(idx->ev_h2d, u);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->s_build, idx->ev_h2d, 0);
    if (e != cudaSuccess) {
        cudaFreeAsync(*d, u);
        *d = nullptr;
        return fail(SJCS_ERR_CUDA, "host-to-device copy failed: %s", cudaGetErrorString(e));
    }
    idx->had_h2d = true;
    return SJCS_OK;
}

int index_build_common(sjcs_ctx* ctx, const float* xyz, bool host, uint64_t n, const sjcs_index_opts* opts,
                       sjcs_index** out) {
    if (!valid_ctx(ctx)) return fail(SJCS_ERR_STATE, "invalid context");
    if (!out) return fail(SJCS_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (n && !xyz) return fail(SJCS_ERR_INVALID, "xyz is NULL");
    if (n > 0xffffffffull) return fail(SJCS_ERR_INVALID, "too many particles for one index (%llu)", (unsigned long long)n);
    sjcs_index_opts o{};
    int rc = check_opts(opts, &o);
    if (rc) return rc;
    rc = set_device(ctx);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(ctx->mu);
    sjcs_index* idx = new_index(ctx);
    if (!idx) return fail(SJCS_ERR_NOMEM, "out of host memory");
    idx->kind = o.kind;
    idx->n = n;
    cudaStream_t s = ctx->s_build;
    const float* d_xyz = xyz;
    void* up = nullptr;
    if (host && n) {
        rc = upload(ctx, idx, xyz, n * 3 * sizeof(float), &up);
        if (rc) {
            free_index(idx);
            return rc;
        }
        d_xyz = static_cast<const float*>(up);
    } else {
        cudaEventRecord(idx->ev_start, s);
        cudaEventRecord(idx->ev_h2d, s);
    }
    order_after_counts(ctx, s);
    rc = enqueue_build(ctx, idx, d_xyz, n, o, s);
    if (up) cudaFreeAsync(up, s);  // after the build, in stream order
    if (rc) {
        free_index(idx);
        return rc;
    }
    cudaEventRecord(idx->ev_ready, s);
    *out = idx;
    return SJCS_OK;
}

uint32_t pow2_ceil(uint32_t v) {
    uint32_t r = 1;
    while (r < v && r < (1u << 30)) r <<= 1;
    return r;
}

// Key of a workload shape for the autotuned-schedule cache.
std::string shape_key(const sjcs_query* q, const sjcs_index* idx) {
    auto lg = [](uint64_t v) { int k = 0; while ((1ull << k) < v && k < 63) ++k; return k; };
    char buf[128];
    uint32_t rbits;
    std::memcpy(&rbits, &q->R, sizeof(rbits));
    std::snprintf(buf, sizeof(buf), "k%d n%d h%d r%08x s%d p%d", idx->kind, lg(idx->n), lg(q->nhalos), rbits,
                  q->nrads, q->flags & SJCS_QUERY_PERIODIC);
    return buf;
}

}  // namespace

Schedule resolve(const sjcs_schedule& in) {
    Schedule sc{};
    sc.mode = in.mode == SJCS_SCHED_QUEUE ? SJCS_SCHED_QUEUE : SJCS_SCHED_STATIC;
    sc.piece = pow2_ceil(in.piece ? in.piece : 32768u);
    sc.max_pieces = in.max_pieces ? in.max_pieces : 64u;
    sc.single = pow2_ceil(in.single ? in.single : std::max(1u, sc.piece / 8u));
    return sc;
}

// The schedule a count call uses (ctx->mu held).
Schedule schedule_for(sjcs_ctx* ctx, const sjcs_query* q, const sjcs_index* idx) {
    sjcs_schedule sc = q->sched;
    if (sc.mode == SJCS_SCHED_AUTO) {
        auto it = ctx->tuned.find(shape_key(q, idx));
        sc = it != ctx->tuned.end() ? it->second : sjcs_schedule{SJCS_SCHED_STATIC, 0, 0, 0};
    }
    return resolve(sc);
}

namespace {

}  // namespace
}  // namespace sjcs

struct sjcs_step {
    uint32_t magic;
    sjcs_ctx* ctx;
    sjcs_query* q;
    cudaGraph_t graph;
    cudaGraphExec_t exec;
    cudaEvent_t ev_pre, ev0, ev1;
    size_t kernels;  // kernel nodes in the graph
    bool launched;
    uint64_t n;      // particles per launch
};

namespace sjcs {
namespace {
constexpr uint32_t kStepMagic = 0x534a5358u;  // "SJSX"
bool valid_step(const sjcs_step* s) { return s && s->magic == kStepMagic; }

// Stream work of one file step, queued while s_build is capturing.
int capture_step_body(sjcs_ctx* ctx, sjcs_query* q, const float* host_xyz, uint64_t n, const sjcs_index_opts& o,
                      sjcs_index* idx, cudaEvent_t join1, cudaEvent_t join2) {
    cudaStream_t sb = ctx->s_build, sc = ctx->s_count;
    float* d = nullptr;
    SJCS_CUDA_TRY(cudaMallocAsync(&d, n * 3 * sizeof(float), sb));
    SJCS_CUDA_TRY(cudaMemcpyAsync(d, host_xyz, n * 3 * sizeof(float), cudaMemcpyHostToDevice, sb));
    int rc = enqueue_build(ctx, idx, d, n, o, sb);
    SJCS_CUDA_TRY(cudaFreeAsync(d, sb));
    if (rc) return rc;
    SJCS_CUDA_TRY(cudaEventRecord(join1, sb));
    SJCS_CUDA_TRY(cudaStreamWaitEvent(sc, join1, 0));
    const Schedule sched = schedule_for(ctx, q, idx);
    rc = idx->kind == SJCS_INDEX_GRID ? launch_shell_count(ctx, q, idx, sc, &sched)
                                      : launch_morton_count(ctx, q, idx, sc, &sched);
    if (idx->pts) SJCS_CUDA_TRY(cudaFreeAsync(idx->pts, sc));
    if (idx->cell_start) SJCS_CUDA_TRY(cudaFreeAsync(idx->cell_start, sc));
    if (idx->leaves) SJCS_CUDA_TRY(cudaFreeAsync(idx->leaves, sc));
    if (idx->root) SJCS_CUDA_TRY(cudaFreeAsync(idx->root, sc));
    idx->pts = nullptr;
    idx->cell_start = nullptr;
    idx->leaves = nullptr;
    idx->root = nullptr;
    SJCS_CUDA_TRY(cudaEventRecord(join2, sc));
    SJCS_CUDA_TRY(cudaStreamWaitEvent(sb, join2, 0));
    return rc;
}
}  // namespace
}  // namespace sjcs

using namespace sjcs;

extern "C" {

const char* sjcs_last_error(void) { return g_last_error.c_str(); }

const char* sjcs_version(void) { return "sjcs-b200 0.1 (sm_100a)"; }

int sjcs_ctx_create(int device, sjcs_ctx** out) {
    if (!out) return fail(SJCS_ERR_INVALID, "out is NULL");
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(SJCS_ERR_CUDA, "no CUDA device available (%s)", cudaGetErrorString(e));
    }
    if (device < 0 || device >= ndev) return fail(SJCS_ERR_INVALID, "device %d out of range [0,%d)", device, ndev);
    SJCS_CUDA_TRY(cudaSetDevice(device));
    int major = 0;
    SJCS_CUDA_TRY(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
    if (major < 10) return fail(SJCS_ERR_CUDA, "device %d is sm_%d0-class; this library is built for sm_100a", device, major);
    sjcs_ctx* ctx = new (std::nothrow) sjcs_ctx();
    if (!ctx) return fail(SJCS_ERR_NOMEM, "out of host memory");
    ctx->magic = kCtxMagic;
    ctx->device = device;
    cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
    SJCS_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->s_build, cudaStreamNonBlocking));
    SJCS_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->s_count, cudaStreamNonBlocking));
    SJCS_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->s_read, cudaStreamNonBlocking));
    SJCS_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->s_h2d, cudaStreamNonBlocking));
    SJCS_CUDA_TRY(cudaEventCreateWithFlags(&ctx->ev_counts, cudaEventDisableTiming));
    // Keep freed stream-ordered memory cached in the pool: every file's index
    // and scratch reuse the previous file's pages without new cudaMalloc calls.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    cudaGetLastError();
    *out = ctx;
    return SJCS_OK;
}

int sjcs_ctx_destroy(sjcs_ctx* ctx) {
    if (!valid_ctx(ctx)) return fail(SJCS_ERR_STATE, "invalid context");
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->s_build);
    cudaStreamSynchronize(ctx->s_count);
    cudaStreamSynchronize(ctx->s_read);
    cudaStreamSynchronize(ctx->s_h2d);
    cudaStreamDestroy(ctx->s_build);
    cudaStreamDestroy(ctx->s_count);
    cudaStreamDestroy(ctx->s_read);
    cudaStreamDestroy(ctx->s_h2d);
    for (cudaEvent_t e : ctx->ring_ev)
        if (e) cudaEventDestroy(e);
    if (ctx->ring) cudaFreeHost(ctx->ring);
    for (cudaEvent_t e : ctx->param_ev)
        if (e) cudaEventDestroy(e);
    if (ctx->param_ring) cudaFreeHost(ctx->param_ring);
    if (ctx->ev_counts) cudaEventDestroy(ctx->ev_counts);
    ctx->magic = 0;
    delete ctx;
    return SJCS_OK;
}

int sjcs_ctx_sync(sjcs_ctx* ctx) {
    if (!valid_ctx(ctx)) return fail(SJCS_ERR_STATE, "invalid context");
    int rc = set_device(ctx);
    if (rc) return rc;
    SJCS_CUDA_TRY(cudaStreamSynchronize(ctx->s_build));
    SJCS_CUDA_TRY(cudaStreamSynchronize(ctx->s_count));
    SJCS_CUDA_TRY(cudaStreamSynchronize(ctx->s_read));
    SJCS_CUDA_TRY(cudaStreamSynchronize(ctx->s_h2d));
    return SJCS_OK;
}

int sjcs_ctx_stream(const sjcs_ctx* ctx, int which, void** stream) {
    if (!valid_ctx(ctx) || !stream || (which != 0 && which != 1)) return fail(SJCS_ERR_INVALID, "invalid argument");
    *stream = (void*)(which == 0 ? ctx->s_build : ctx->s_count);
    return SJCS_OK;
}

int sjcs_ctx_set_overlap(sjcs_ctx* ctx, int overlap) {
    if (!valid_ctx(ctx)) return fail(SJCS_ERR_STATE, "invalid context");
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->overlap = overlap != 0;
    return SJCS_OK;
}

uint64_t sjcs_launch_counter(void) { return g_launches.load(); }

int sjcs_ctx_reserve(sjcs_ctx* ctx, uint64_t bytes) {
    if (!valid_ctx(ctx)) return fail(SJCS_ERR_STATE, "invalid context");
    int rc = set_device(ctx);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(ctx->mu);
    SJCS_CUDA_TRY(cudaStreamSynchronize(ctx->s_build));
    SJCS_CUDA_TRY(cudaStreamSynchronize(ctx->s_count));
    if (bytes == 0) return SJCS_OK;
    void* p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, bytes, ctx->s_count);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(SJCS_ERR_NOMEM, "cannot reserve %llu bytes: %s", (unsigned long long)bytes, cudaGetErrorString(e));
    }
    SJCS_CUDA_TRY(cudaFreeAsync(p, ctx->s_count));
    SJCS_CUDA_TRY(cudaStreamSynchronize(ctx->s_count));
    return SJCS_OK;
}

int sjcs_ctx_trim(sjcs_ctx* ctx) {
    if (!valid_ctx(ctx)) return fail(SJCS_ERR_STATE, "invalid context");
    int rc = set_device(ctx);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(ctx->mu);
    SJCS_CUDA_TRY(cudaStreamSynchronize(ctx->s_build));
    SJCS_CUDA_TRY(cudaStreamSynchronize(ctx->s_count));
    cudaMemPool_t pool;
    SJCS_CUDA_TRY(cudaDeviceGetDefaultMemPool(&pool, ctx->device));
    SJCS_CUDA_TRY(cudaMemPoolTrimTo(pool, 0));
    return SJCS_OK;
}

int sjcs_ctx_memory(sjcs_ctx* ctx, uint64_t* free_bytes, uint64_t* pool_bytes) {
    if (!valid_ctx(ctx)) return fail(SJCS_ERR_STATE, "invalid context");
    int rc = set_device(ctx);
    if (rc) return rc;
    if (free_bytes) {
        size_t f = 0, t = 0;
        SJCS_CUDA_TRY(cudaMemGetInfo(&f, &t));
        *free_bytes = f;
    }
    if (pool_bytes) {
        cudaMemPool_t pool;
        SJCS_CUDA_TRY(cudaDeviceGetDefaultMemPool(&pool, ctx->device));
        uint64_t v = 0;
        SJCS_CUDA_TRY(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &v));
        *pool_bytes = v;
    }
    return SJCS_OK;
}

int sjcs_ctx_num_sms(const sjcs_ctx* ctx, int* out) {
    if (!valid_ctx(ctx) || !out) return fail(SJCS_ERR_INVALID, "invalid argument");
    *out = ctx->num_sms;
    return SJCS_OK;
}

int sjcs_host_alloc(size_t bytes, void** out) {
    if (!out) return fail(SJCS_ERR_INVALID, "out is NULL");
    *out = nullptr;
    cudaError_t e = cudaMallocHost(out, bytes ? bytes : 1);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(SJCS_ERR_NOMEM, "pinned allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    }
    return SJCS_OK;
}

int sjcs_host_free(void* p) {
    if (!p) return SJCS_OK;
    SJCS_CUDA_TRY(cudaFreeHost(p));
    return SJCS_OK;
}

int sjcs_index_build(sjcs_ctx* ctx, const float* xyz, uint64_t n, const sjcs_index_opts* opts, sjcs_index** out) {
    return index_build_common(ctx, xyz, true, n, opts, out);
}

int sjcs_index_build_device(sjcs_ctx* ctx, const float* d_xyz, uint64_t n, const sjcs_index_opts* opts,
                            sjcs_index** out) {
    return index_build_common(ctx, d_xyz, false, n, opts, out);
}

namespace {
constexpr size_t kIngestChunk = 8u << 20;  // bytes per read and per copy
constexpr unsigned kIngestThreads = 8;      // reader threads = staging slots

// Read [off, off + len) of fd completely.
bool pread_all(int fd, char* dst, uint64_t off, uint64_t len) {
    uint64_t done = 0;
    while (done < len) {
        const ssize_t r = pread(fd, dst + done, (size_t)(len - done), (off_t)(off + done));
        if (r <= 0) return false;
        done += (uint64_t)r;
    }
    return true;
}

// bytes of fd into new device memory *d on the upload stream: reader thread t
// takes chunks t, t + T, ... through its own staging slot, waiting for the
// slot's previous copy before overwriting it.  idx's ev_start / ev_h2d
// bracket the copies and the build stream waits for them.  Called with
// ctx->ring_mu held.
// The page-locked staging slots and their events (once per context; called
// with ctx->ring_mu held).
int ensure_ring(sjcs_ctx* ctx) {
    if (ctx->ring) return SJCS_OK;
    SJCS_CUDA_TRY(cudaMallocHost(&ctx->ring, (size_t)kIngestThreads * kIngestChunk));
    ctx->ring_ev.assign(kIngestThreads, nullptr);
    for (auto& e : ctx->ring_ev) SJCS_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return SJCS_OK;
}

int ingest_file(sjcs_ctx* ctx, sjcs_index* idx, int fd, uint64_t bytes, void** d) {
    cudaStream_t u = ctx->s_h2d;
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const unsigned T = std::min(kIngestThreads, hw);
    int rc = ensure_ring(ctx);
    if (rc) return rc;
    *d = nullptr;
    cudaEventRecord(idx->ev_start, u);
    cudaError_t e = cudaMallocAsync(d, bytes, u);
    if (e != cudaSuccess) {
        *d = nullptr;
        cudaGetLastError();
        return fail(SJCS_ERR_NOMEM, "device allocation of %llu bytes for the file failed: %s",
                    (unsigned long long)bytes, cudaGetErrorString(e));
    }
    const uint64_t nchunks = (bytes + kIngestChunk - 1) / kIngestChunk;
    std::atomic<int> bad_read{0}, bad_cuda{0};
    auto worker = [&](unsigned t) {
        char* slot = ctx->ring + (size_t)t * kIngestChunk;
        for (uint64_t c = t; c < nchunks && !bad_read && !bad_cuda; c += T) {
            const uint64_t off = c * kIngestChunk, len = std::min<uint64_t>(kIngestChunk, bytes - off);
            if (cudaEventSynchronize(ctx->ring_ev[t]) != cudaSuccess) { bad_cuda = 1; return; }
            if (!pread_all(fd, slot, off, len)) { bad_read = 1; return; }
            if (cudaMemcpyAsync(static_cast<char*>(*d) + off, slot, len, cudaMemcpyHostToDevice, u) != cudaSuccess ||
                cudaEventRecord(ctx->ring_ev[t], u) != cudaSuccess) {
                bad_cuda = 1;
                return;
            }
        }
    };
    std::vector<std::thread> th;
    th.reserve(T);
    for (unsigned t = 1; t < T; ++t) th.emplace_back(worker, t);
    worker(0);
    for (auto& x : th) x.join();
    if (bad_read || bad_cuda) {
        cudaStreamSynchronize(u);  // copies out of the staging slots are done before they are reused
        cudaFreeAsync(*d, u);
        *d = nullptr;
        cudaGetLastError();
        return bad_read ? fail(SJCS_ERR_INVALID, "short read of the particle file")
                        : fail(SJCS_ERR_CUDA, "host-to-device copy of the particle file failed");
    }
    cudaEventRecord(idx->ev_h2d, u);
    SJCS_CUDA_TRY(cudaStreamWaitEvent(ctx->s_build, idx->ev_h2d, 0));
    idx->had_h2d = true;
    return SJCS_OK;
}
}  // namespace

int sjcs_ctx_prepare_files(sjcs_ctx* ctx, uint64_t max_particles) {
    if (!valid_ctx(ctx)) return fail(SJCS_ERR_STATE, "invalid context");
    int rc = set_device(ctx);
    if (rc) return rc;
    {
        std::lock_guard<std::mutex> lk(ctx->ring_mu);
        rc = ensure_ring(ctx);
        if (rc) return rc;
    }
    // one file's upload (12 B), sorted particles (16 B), the partition
    // build's records (16 B) and middle digits (2 B) per particle, its
    // segment tables, and the largest automatic cell table (2^28 + 1 entries)
    const uint64_t bytes = max_particles * 48ull + (268435457ull * 4ull) + (64ull << 20);
    return max_particles ? sjcs_ctx_reserve(ctx, bytes) : SJCS_OK;
}

int sjcs_index_build_file(sjcs_ctx* ctx, const char* path, const sjcs_index_opts* opts, sjcs_index** out) {
    if (!valid_ctx(ctx)) return fail(SJCS_ERR_STATE, "invalid context");
    if (!out) return fail(SJCS_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!path) return fail(SJCS_ERR_INVALID, "path is NULL");
    sjcs_index_opts o{};
    int rc = check_opts(opts, &o);
    if (rc) return rc;
    const int fd = open(path, O_RDONLY);
    struct stat st;
    if (fd < 0 || fstat(fd, &st) != 0) {
        if (fd >= 0) close(fd);
        return fail(SJCS_ERR_INVALID, "ERROR: file %s not found in readDecodedParticles()", path);
    }
    const uint64_t n = (uint64_t)st.st_size / (3 * sizeof(float));
    if (n > 0xffffffffull) {
        close(fd);
        return fail(SJCS_ERR_INVALID, "too many particles for one index (%llu)", (unsigned long long)n);
    }
    rc = set_device(ctx);
    if (rc) {
        close(fd);
        return rc;
    }
    sjcs_index* idx = new_index(ctx);
    if (!idx) {
        close(fd);
        return fail(SJCS_ERR_NOMEM, "out of host memory");
    }
    idx->kind = o.kind;
    idx->n = n;
    void* d = nullptr;
    if (n) {
        std::lock_guard<std::mutex> lk(ctx->ring_mu);
        rc = ingest_file(ctx, idx, fd, n * 3 * sizeof(float), &d);
    }
    close(fd);
    if (rc) {
        free_index(idx);
        return rc;
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaStream_t s = ctx->s_build;
    if (!n) {
        cudaEventRecord(idx->ev_start, s);
        cudaEventRecord(idx->ev_h2d, s);
    }
    order_after_counts(ctx, s);
    rc = enqueue_build(ctx, idx, static_cast<const float*>(d), n, o, s);
    if (d) cudaFreeAsync(d, s);  // after the build, in stream order
    if (rc) {
        free_index(idx);
        return rc;
    }
    cudaEventRecord(idx->ev_ready, s);
    *out = idx;
    return SJCS_OK;
}

int sjcs_index_build_compressed(sjcs_ctx* ctx, const uint16_t* uv, uint64_t n, const void* gadget_header,
                                const sjcs_index_opts* opts, sjcs_index** out) {
    if (!valid_ctx(ctx)) return fail(SJCS_ERR_STATE, "invalid context");
    if (!out) return fail(SJCS_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (n && !uv) return fail(SJCS_ERR_INVALID, "uv is NULL");
    if (n > 0xffffffffull) return fail(SJCS_ERR_INVALID, "too many particles for one index (%llu)", (unsigned long long)n);
    GadgetDecode g{};
    int rc = gadget_decode_params(gadget_header, &g);
    if (rc) return rc;
    sjcs_index_opts o{};
    rc = check_opts(opts, &o);
    if (rc) return rc;
    rc = set_device(ctx);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(ctx->mu);
    sjcs_index* idx = new_index(ctx);
    if (!idx) return fail(SJCS_ERR_NOMEM, "out of host memory");
    idx->kind = o.kind;
    idx->n = n;
    cudaStream_t s = ctx->s_build;
    void* up = nullptr;
    if (n) {
        rc = upload(ctx, idx, uv, n * 3 * sizeof(uint16_t), &up);
        if (rc) {
            free_index(idx);
            return rc;
        }
    } else {
        cudaEventRecord(idx->ev_start, s);
        cudaEventRecord(idx->ev_h2d, s);
    }
    const uint16_t* d_uv = static_cast<const uint16_t*>(up);
    StreamScratch scr(s);
    float* d_xyz = nullptr;
    cudaError_t e = scr.alloc(&d_xyz, n * 3 * sizeof(float));
    if (e != cudaSuccess) {
        if (up) cudaFreeAsync(up, s);
        free_index(idx);
        return fail(SJCS_ERR_NOMEM, "device allocation for %llu compressed particles failed: %s",
                    (unsigned long long)n, cudaGetErrorString(e));
    }
    order_after_counts(ctx, s);
    rc = launch_decode(d_uv, n, g, d_xyz, s);
    if (!rc) rc = enqueue_build(ctx, idx, d_xyz, n, o, s);
    if (up) cudaFreeAsync(up, s);  // after the decode, in stream order
    if (rc) {
        free_index(idx);
        return rc;
    }
    cudaEventRecord(idx->ev_ready, s);
    *out = idx;
    return SJCS_OK;
}

int sjcs_decode_compressed(sjcs_ctx* ctx, const uint16_t* uv, uint64_t n, const void* gadget_header, float* xyz) {
    if (!valid_ctx(ctx)) return fail(SJCS_ERR_STATE, "invalid context");
    if (n && (!uv || !xyz)) return fail(SJCS_ERR_INVALID, "uv or xyz is NULL");
    GadgetDecode g{};
    int rc = gadget_decode_params(gadget_header, &g);
    if (rc) return rc;
    rc = set_device(ctx);
    if (rc) return rc;
    if (n == 0) return SJCS_OK;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaStream_t s = ctx->s_build;
    {
        StreamScratch scr(s);
        uint16_t* d_uv = nullptr;
        float* d_xyz = nullptr;
        SJCS_CUDA_TRY(scr.alloc(&d_uv, n * 3 * sizeof(uint16_t)));
        SJCS_CUDA_TRY(scr.alloc(&d_xyz, n * 3 * sizeof(float)));
        SJCS_CUDA_TRY(cudaMemcpyAsync(d_uv, uv, n * 3 * sizeof(uint16_t), cudaMemcpyHostToDevice, s));
        rc = launch_decode(d_uv, n, g, d_xyz, s);
        if (rc) return rc;
        SJCS_CUDA_TRY(cudaMemcpyAsync(xyz, d_xyz, n * 3 * sizeof(float), cudaMemcpyDeviceToHost, s));
    }
    SJCS_CUDA_TRY(cudaStreamSynchronize(s));
    return SJCS_OK;
}

int sjcs_index_wait(sjcs_index* idx) {
    if (!valid_index(idx)) return fail(SJCS_ERR_STATE, "invalid index");
    SJCS_CUDA_TRY(cudaEventSynchronize(idx->ev_ready));
    return SJCS_OK;
}

int sjcs_index_size(const sjcs_index* idx, uint64_t* out) {
    if (!valid_index(idx) || !out) return fail(SJCS_ERR_INVALID, "invalid argument");
    *out = idx->n;
    return SJCS_OK;
}

int sjcs_index_grid(const sjcs_index* idx, uint32_t out[3]) {
    if (!valid_index(idx) || !out) return fail(SJCS_ERR_INVALID, "invalid argument");
    for (int a = 0; a < 3; ++a) out[a] = (uint32_t)idx->geom.G[a];
    return SJCS_OK;
}

int sjcs_index_learned_info(sjcs_index* idx, sjcs_learned_info* out) {
    if (!valid_index(idx) || !out) return fail(SJCS_ERR_INVALID, "invalid argument");
    if (idx->kind != SJCS_INDEX_LEARNED) return fail(SJCS_ERR_INVALID, "not a learned index");
    int rc = set_device(idx->ctx);
    if (rc) return rc;
    SJCS_CUDA_TRY(cudaEventSynchronize(idx->ev_ready));
    LearnedRoot r{};
    SJCS_CUDA_TRY(cudaMemcpy(&r, idx->root, sizeof(r), cudaMemcpyDeviceToHost));
    sjcs_learned_info info{};
    info.level = (uint32_t)idx->level;
    info.leaves = kLeaves;
    info.nonempty = r.nonempty;
    info.max_err = r.max_err;
    info.mean_err = r.nonempty ? (double)r.sum_err / (double)r.nonempty : 0.0;
    info.checked = r.checked;
    info.mismatches = r.mismatches;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, idx->ev_h2d, idx->ev_train0) == cudaSuccess) info.sort_ms = ms;
    if (cudaEventElapsedTime(&ms, idx->ev_train0, idx->ev_ready) == cudaSuccess) info.train_ms = ms;
    cudaGetLastError();
    *out = info;
    return SJCS_OK;
}

int sjcs_index_timing(const sjcs_index* idx, sjcs_timing* out) {
    if (!valid_index(idx) || !out) return fail(SJCS_ERR_INVALID, "invalid argument");
    SJCS_CUDA_TRY(cudaEventSynchronize(idx->ev_ready));
    sjcs_timing t{};
    float ms = 0.f;
    if (idx->had_h2d && cudaEventElapsedTime(&ms, idx->ev_start, idx->ev_h2d) == cudaSuccess) t.h2d_ms = ms;
    if (cudaEventElapsedTime(&ms, idx->ev_h2d, idx->ev_ready) == cudaSuccess) t.build_ms = ms;
    cudaGetLastError();
    *out = t;
    return SJCS_OK;
}

int sjcs_index_destroy(sjcs_index* idx) {
    if (!valid_index(idx)) return fail(SJCS_ERR_STATE, "invalid index");
    sjcs_ctx* ctx = idx->ctx;
    cudaSetDevice(ctx->device);
    std::lock_guard<std::mutex> lk(ctx->mu);
    free_index(idx);
    return SJCS_OK;
}

int sjcs_query_create(sjcs_ctx* ctx, const float* halo_xyz, size_t stride_bytes, uint64_t nhalos, const float* r2,
                      int nrads, int flags, sjcs_query** out) {
    int rc = check_query_args(ctx, halo_xyz, stride_bytes, nhalos, r2, nrads, flags, out);
    if (rc) return rc;
    *out = nullptr;
    rc = set_device(ctx);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(ctx->mu);
    sjcs_query* q = new_query(ctx);
    if (!q) return fail(SJCS_ERR_NOMEM, "out of host memory");
    cudaStream_t s = ctx->s_count, u = ctx->s_h2d;
    float* d_raw = nullptr;
    // The last halo needs only its 12 coordinate bytes, not a whole stride.
    const size_t bytes = nhalos ? (size_t)(nhalos - 1) * stride_bytes + 3 * sizeof(float) : 0;
    if (nhalos) {
        // on the upload stream, so the copy overlaps counts already queued on
        // the count stream; the count stream waits for it
        cudaEvent_t ev = nullptr;
        cudaError_t e = cudaMallocAsync(&d_raw, bytes, u);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_raw, halo_xyz, bytes, cudaMemcpyHostToDevice, u);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventRecord(ev, u);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s, ev, 0);
        if (ev) cudaEventDestroy(ev);
        if (e != cudaSuccess) {
            if (d_raw) cudaFreeAsync(d_raw, u);
            free_query(q);
            return fail(SJCS_ERR_CUDA, "halo upload failed: %s", cudaGetErrorString(e));
        }
    }
    rc = query_prepare(ctx, d_raw, stride_bytes, nhalos, r2, nrads, flags, q, s);
    if (d_raw) cudaFreeAsync(d_raw, s);  // after the halo sort that reads it
    if (rc) {
        free_query(q);
        return rc;
    }
    *out = q;
    return SJCS_OK;
}

int sjcs_query_create_device(sjcs_ctx* ctx, const float* d_halo_xyz, size_t stride_bytes, uint64_t nhalos,
                             const float* r2, int nrads, int flags, sjcs_query** out) {
    int rc = check_query_args(ctx, d_halo_xyz, stride_bytes, nhalos, r2, nrads, flags, out);
    if (rc) return rc;
    *out = nullptr;
    rc = set_device(ctx);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(ctx->mu);
    sjcs_query* q = new_query(ctx);
    if (!q) return fail(SJCS_ERR_NOMEM, "out of host memory");
    rc = query_prepare(ctx, d_halo_xyz, stride_bytes, nhalos, r2, nrads, flags, q, ctx->s_count);
    if (rc) {
        free_query(q);
        return rc;
    }
    *out = q;
    return SJCS_OK;
}

int sjcs_query_count(sjcs_ctx* ctx, sjcs_query* q, const sjcs_index* idx) {
    if (!valid_ctx(ctx)) return fail(SJCS_ERR_STATE, "invalid context");
    if (!valid_query(q) || q->ctx != ctx) return fail(SJCS_ERR_STATE, "query does not belong to this context");
    if (!valid_index(idx) || idx->ctx != ctx) return fail(SJCS_ERR_STATE, "index does not belong to this context");
    int rc = set_device(ctx);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaStream_t s = ctx->s_count;
    SJCS_CUDA_TRY(cudaStreamWaitEvent(s, idx->ev_ready, 0));
    SJCS_CUDA_TRY(after_reads(q, s));
    rc = fold_before_count(ctx, q, count_call_bound(q->flags, q->r2max, idx->n), s);
    if (rc) return rc;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    SJCS_CUDA_TRY(cudaEventCreate(&e0));
    SJCS_CUDA_TRY(cudaEventCreate(&e1));
    q->count_events.push_back(e0);
    q->count_events.push_back(e1);
    cudaEventRecord(e0, s);
    const Schedule sc = schedule_for(ctx, q, idx);
    rc = idx->kind == SJCS_INDEX_GRID ? launch_shell_count(ctx, q, idx, s, &sc) : launch_morton_count(ctx, q, idx, s, &sc);
    cudaEventRecord(e1, s);
    cudaEventRecord(q->ev_last, s);
    return rc;
}

int sjcs_query_count_many(sjcs_ctx* ctx, sjcs_query* q, const sjcs_index* const* idx, int k) {
    if (!valid_ctx(ctx)) return fail(SJCS_ERR_STATE, "invalid context");
    if (!valid_query(q) || q->ctx != ctx) return fail(SJCS_ERR_STATE, "query does not belong to this context");
    if (k < 0 || (k > 0 && !idx)) return fail(SJCS_ERR_INVALID, "idx is NULL or k < 0");
    for (int i = 0; i < k; ++i)
        if (!valid_index(idx[i]) || idx[i]->ctx != ctx)
            return fail(SJCS_ERR_STATE, "index %d does not belong to this context", i);
    int rc = set_device(ctx);
    if (rc) return rc;
    // Fused: runs of up to kMaxFused grid indexes of one geometry under the
    // static schedule whose counts fit the accumulators together; anything
    // else is counted index by index.
    for (int i = 0; i < k;) {
        int j = i + 1;
        const sjcs_index* a = idx[i];
        bool fuse = a->kind == SJCS_INDEX_GRID;
        if (fuse) {
            std::lock_guard<std::mutex> lk(ctx->mu);
            fuse = schedule_for(ctx, q, a).mode != SJCS_SCHED_QUEUE;
        }
        uint64_t add = count_call_bound(q->flags, q->r2max, a->n);
        while (fuse && j < k && j - i < kMaxFusedIndexes) {
            const sjcs_index* b = idx[j];
            const uint64_t add_b = count_call_bound(q->flags, q->r2max, b->n);
            if (b->kind != SJCS_INDEX_GRID || b->geom.ncells != a->geom.ncells || b->geom.G[0] != a->geom.G[0] ||
                b->geom.G[1] != a->geom.G[1] || b->geom.G[2] != a->geom.G[2] || add + add_b > q->fold_limit)
                break;
            add += add_b;
            ++j;
        }
        if (j - i == 1) {
            rc = sjcs_query_count(ctx, q, a);
            if (rc) return rc;
            i = j;
            continue;
        }
        std::lock_guard<std::mutex> lk(ctx->mu);
        cudaStream_t s = ctx->s_count;
        for (int t = i; t < j; ++t) SJCS_CUDA_TRY(cudaStreamWaitEvent(s, idx[t]->ev_ready, 0));
        SJCS_CUDA_TRY(after_reads(q, s));
        rc = fold_before_count(ctx, q, add, s);
        if (rc) return rc;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        SJCS_CUDA_TRY(cudaEventCreate(&e0));
        SJCS_CUDA_TRY(cudaEventCreate(&e1));
        q->count_events.push_back(e0);
        q->count_events.push_back(e1);
        cudaEventRecord(e0, s);
        rc = launch_shell_count_multi(ctx, q, idx + i, j - i, s);
        cudaEventRecord(e1, s);
        cudaEventRecord(q->ev_last, s);
        if (rc) return rc;
        i = j;
    }
    return SJCS_OK;
}

int sjcs_step_create(sjcs_ctx* ctx, sjcs_query* q, const float* host_xyz, uint64_t n, const sjcs_index_opts* opts,
                     sjcs_step** out) {
    if (!valid_ctx(ctx)) return fail(SJCS_ERR_STATE, "invalid context");
    if (!valid_query(q) || q->ctx != ctx) return fail(SJCS_ERR_STATE, "query does not belong to this context");
    if (!out) return fail(SJCS_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!host_xyz || n == 0) return fail(SJCS_ERR_INVALID, "a step needs a host buffer of n >= 1 particles");
    if (n > 0xffffffffull) return fail(SJCS_ERR_INVALID, "too many particles for one index (%llu)", (unsigned long long)n);
    sjcs_index_opts o{};
    int rc = check_opts(opts, &o);
    if (rc) return rc;
    rc = set_device(ctx);
    if (rc) return rc;
    cudaPointerAttributes pa{};
    if (cudaPointerGetAttributes(&pa, host_xyz) != cudaSuccess || pa.type != cudaMemoryTypeHost) {
        cudaGetLastError();
        return fail(SJCS_ERR_INVALID, "the step's particle buffer must be pinned host memory (sjcs_host_alloc)");
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    sjcs_step* st = new (std::nothrow) sjcs_step();
    if (!st) return fail(SJCS_ERR_NOMEM, "out of host memory");
    st->magic = kStepMagic;
    st->ctx = ctx;
    st->q = q;
    st->n = n;
    cudaEventCreate(&st->ev_pre);
    cudaEventCreate(&st->ev0);
    cudaEventCreate(&st->ev1);
    cudaEvent_t join1 = nullptr, join2 = nullptr;
    cudaEventCreateWithFlags(&join1, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&join2, cudaEventDisableTiming);
    sjcs_index* idx = new_index(ctx);
    idx->kind = o.kind;
    idx->n = n;
    cudaError_t e = cudaStreamBeginCapture(ctx->s_build, cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) {
        rc = fail(SJCS_ERR_CUDA, "stream capture could not start: %s", cudaGetErrorString(e));
    } else {
        rc = capture_step_body(ctx, q, host_xyz, n, o, idx, join1, join2);
        cudaGraph_t g = nullptr;
        e = cudaStreamEndCapture(ctx->s_build, &g);
        if (!rc && e != cudaSuccess) rc = fail(SJCS_ERR_CUDA, "stream capture failed: %s", cudaGetErrorString(e));
        st->graph = g;
        if (!rc) {
            e = cudaGraphInstantiate(&st->exec, g, 0);
            if (e != cudaSuccess) rc = fail(SJCS_ERR_CUDA, "graph instantiation failed: %s", cudaGetErrorString(e));
            size_t nn = 0;
            if (!rc && cudaGraphGetNodes(g, nullptr, &nn) == cudaSuccess && nn) {
                std::vector<cudaGraphNode_t> nodes(nn);
                if (cudaGraphGetNodes(g, nodes.data(), &nn) == cudaSuccess)
                    for (cudaGraphNode_t nd : nodes) {
                        cudaGraphNodeType t;
                        if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++st->kernels;
                    }
            }
        }
    }
    cudaGetLastError();
    // The index object only described the captured buffers; its memory
    // belongs to the graph.
    idx->pts = nullptr;
    idx->cell_start = nullptr;
    idx->leaves = nullptr;
    idx->root = nullptr;
    free_index(idx);
    cudaEventDestroy(join1);
    cudaEventDestroy(join2);
    if (rc) {
        if (st->exec) cudaGraphExecDestroy(st->exec);
        if (st->graph) cudaGraphDestroy(st->graph);
        cudaEventDestroy(st->ev_pre);
        cudaEventDestroy(st->ev0);
        cudaEventDestroy(st->ev1);
        st->magic = 0;
        delete st;
        return rc;
    }
    *out = st;
    return SJCS_OK;
}

int sjcs_step_launch(sjcs_ctx* ctx, sjcs_step* st) {
    if (!valid_ctx(ctx)) return fail(SJCS_ERR_STATE, "invalid context");
    if (!valid_step(st) || st->ctx != ctx) return fail(SJCS_ERR_STATE, "step does not belong to this context");
    if (!valid_query(st->q)) return fail(SJCS_ERR_STATE, "the step's query was destroyed");
    int rc = set_device(ctx);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(ctx->mu);
    // the 32-bit accumulators are folded first if this file could overflow them
    SJCS_CUDA_TRY(after_reads(st->q, ctx->s_count));
    rc = fold_before_count(ctx, st->q, count_call_bound(st->q->flags, st->q->r2max, st->n), ctx->s_count);
    if (rc) return rc;
    // after everything queued so far on both streams (halo preparation,
    // earlier counts and read-backs of the query)
    SJCS_CUDA_TRY(cudaEventRecord(st->ev_pre, ctx->s_count));
    SJCS_CUDA_TRY(cudaStreamWaitEvent(ctx->s_build, st->ev_pre, 0));
    SJCS_CUDA_TRY(after_reads(st->q, ctx->s_build));
    SJCS_CUDA_TRY(cudaEventRecord(st->ev0, ctx->s_build));
    SJCS_CUDA_TRY(cudaGraphLaunch(st->exec, ctx->s_build));
    for (size_t k = 0; k < st->kernels; ++k) note_launch();
    SJCS_CUDA_TRY(cudaEventRecord(st->ev1, ctx->s_build));
    SJCS_CUDA_TRY(cudaStreamWaitEvent(ctx->s_count, st->ev1, 0));
    SJCS_CUDA_TRY(cudaEventRecord(st->q->ev_last, ctx->s_count));
    st->launched = true;
    return SJCS_OK;
}

int sjcs_step_wait(sjcs_step* st) {
    if (!valid_step(st)) return fail(SJCS_ERR_STATE, "invalid step");
    if (st->launched) SJCS_CUDA_TRY(cudaEventSynchronize(st->ev1));
    return SJCS_OK;
}

int sjcs_step_time(sjcs_step* st, float* ms) {
    if (!valid_step(st) || !ms) return fail(SJCS_ERR_INVALID, "invalid argument");
    *ms = 0.0f;
    if (!st->launched) return SJCS_OK;
    SJCS_CUDA_TRY(cudaEventSynchronize(st->ev1));
    SJCS_CUDA_TRY(cudaEventElapsedTime(ms, st->ev0, st->ev1));
    return SJCS_OK;
}

int sjcs_step_destroy(sjcs_step* st) {
    if (!valid_step(st)) return fail(SJCS_ERR_STATE, "invalid step");
    set_device(st->ctx);
    if (st->launched) cudaEventSynchronize(st->ev1);
    cudaGraphExecDestroy(st->exec);
    cudaGraphDestroy(st->graph);
    cudaEventDestroy(st->ev_pre);
    cudaEventDestroy(st->ev0);
    cudaEventDestroy(st->ev1);
    st->magic = 0;
    delete st;
    return SJCS_OK;
}

int sjcs_query_set_schedule(sjcs_ctx* ctx, sjcs_query* q, const sjcs_schedule* sched) {
    if (!valid_ctx(ctx)) return fail(SJCS_ERR_STATE, "invalid context");
    if (!valid_query(q) || q->ctx != ctx) return fail(SJCS_ERR_STATE, "query does not belong to this context");
    if (!sched) return fail(SJCS_ERR_INVALID, "schedule is NULL");
    if (sched->mode < SJCS_SCHED_AUTO || sched->mode > SJCS_SCHED_QUEUE)
        return fail(SJCS_ERR_INVALID, "unknown schedule mode %d", sched->mode);
    if (sched->piece > (1u << 30) || sched->single > (1u << 30) || sched->max_pieces > 65536u)
        return fail(SJCS_ERR_INVALID, "schedule sizes out of range (piece, single <= 2^30, max_pieces <= 65536)");
    std::lock_guard<std::mutex> lk(ctx->mu);
    q->sched = *sched;
    return SJCS_OK;
}

int sjcs_query_get_schedule(const sjcs_query* q, sjcs_schedule* out) {
    if (!valid_query(q) || !out) return fail(SJCS_ERR_INVALID, "invalid argument");
    *out = q->sched;
    return SJCS_OK;
}

int sjcs_autotune(sjcs_ctx* ctx, sjcs_query* q, const sjcs_index* idx, sjcs_schedule* chosen, float* trial_ms,
                  int max_trials, int* ntrials) {
    if (!valid_ctx(ctx)) return fail(SJCS_ERR_STATE, "invalid context");
    if (!valid_query(q) || q->ctx != ctx) return fail(SJCS_ERR_STATE, "query does not belong to this context");
    if (!valid_index(idx) || idx->ctx != ctx) return fail(SJCS_ERR_STATE, "index does not belong to this context");
    if (trial_ms && max_trials < 0) return fail(SJCS_ERR_INVALID, "max_trials < 0");
    int rc = set_device(ctx);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(ctx->mu);
    std::vector<sjcs_schedule> cand{{SJCS_SCHED_STATIC, 0, 0, 0}};
    for (uint32_t pc : {2048u, 8192u, 32768u, 131072u}) cand.push_back(sjcs_schedule{SJCS_SCHED_QUEUE, pc, 64u, 0});
    cand.push_back(sjcs_schedule{SJCS_SCHED_QUEUE, 32768u, 256u, 0});
    std::vector<float> ms(cand.size(), 0.0f);
    cudaStream_t s = ctx->s_count;
    SJCS_CUDA_TRY(cudaStreamWaitEvent(s, idx->ev_ready, 0));
    // trials count into scratch accumulators; the query's own stay untouched
    uint32_t* saved = q->counts;
    uint32_t* tmp = nullptr;
    const size_t bytes = (size_t)q->nhalos * (size_t)q->nrads * sizeof(uint32_t);
    SJCS_CUDA_TRY(cudaMallocAsync(&tmp, bytes ? bytes : 16, s));
    q->counts = tmp;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto run = [&](const sjcs_schedule& c, float* out_ms) -> int {
        const Schedule sc = resolve(c);
        cudaEventRecord(e0, s);
        int r = idx->kind == SJCS_INDEX_GRID ? launch_shell_count(ctx, q, idx, s, &sc)
                                             : launch_morton_count(ctx, q, idx, s, &sc);
        cudaEventRecord(e1, s);
        if (r) return r;
        if (cudaEventSynchronize(e1) != cudaSuccess) return fail(SJCS_ERR_CUDA, "autotune trial failed");
        float t = 0.0f;
        cudaEventElapsedTime(&t, e0, e1);
        *out_ms = t;
        return SJCS_OK;
    };
    float warm = 0.0f;
    rc = run(cand[0], &warm);  // warm-up (caches, clocks, lazy module loading)
    const int reps = warm < 5.0f ? 3 : 1;
    for (size_t i = 0; i < cand.size() && !rc; ++i) {
        float best = 0.0f;
        for (int r = 0; r < reps && !rc; ++r) {
            float t = 0.0f;
            rc = run(cand[i], &t);
            best = (r == 0 || t < best) ? t : best;
        }
        ms[i] = best;
    }
    q->counts = saved;
    cudaFreeAsync(tmp, s);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    size_t bi = 0;
    for (size_t i = 1; i < cand.size(); ++i)
        if (ms[i] < ms[bi]) bi = i;
    q->sched = cand[bi];
    ctx->tuned[shape_key(q, idx)] = cand[bi];
    if (chosen) *chosen = cand[bi];
    if (trial_ms)
        for (int i = 0; i < max_trials && i < (int)cand.size(); ++i) trial_ms[i] = ms[i];
    if (ntrials) *ntrials = (int)cand.size();
    return SJCS_OK;
}

int sjcs_query_wait(sjcs_query* q) {
    if (!valid_query(q)) return fail(SJCS_ERR_STATE, "invalid query");
    SJCS_CUDA_TRY(cudaEventSynchronize(q->ev_last));
    return SJCS_OK;
}

int sjcs_query_read_counts(sjcs_ctx* ctx, sjcs_query* q, uint64_t* counts, int accumulate) {
    if (!valid_ctx(ctx)) return fail(SJCS_ERR_STATE, "invalid context");
    if (!valid_query(q) || q->ctx != ctx) return fail(SJCS_ERR_STATE, "query does not belong to this context");
    const uint64_t m = q->nhalos * (uint64_t)q->nrads;
    if (m && !counts) return fail(SJCS_ERR_INVALID, "counts is NULL");
    int rc = set_device(ctx);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaStream_t s = ctx->s_count;
    if (m == 0) return SJCS_OK;
    StreamScratch scr(s);
    unsigned long long* wide = nullptr;
    SJCS_CUDA_TRY(scr.alloc(&wide, m * sizeof(uint64_t)));
    cudaEventRecord(q->ev_d0, s);
    k_widen_u32_u64<<<ctx->num_sms * 8, 256, 0, s>>>(q->counts, m, q->counts64, wide);
    SJCS_LAUNCH_CHECK();
    if (!accumulate && is_pinned(counts)) {
        SJCS_CUDA_TRY(cudaMemcpyAsync(counts, wide, m * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
        cudaEventRecord(q->ev_d1, s);
        SJCS_CUDA_TRY(cudaStreamSynchronize(s));
    } else {
        // Double-buffered pinned staging; host threads store (or add) chunk
        // k while the copy engine brings chunk k+1.
        const uint64_t chunk = 8ull << 20;  // elements (64 MB)
        if (!q->h_stage) {
            SJCS_CUDA_TRY(cudaMallocHost(&q->h_stage, 2 * chunk * sizeof(uint64_t)));
            q->h_stage_elems = 2 * chunk;
        }
        uint64_t* stage = reinterpret_cast<uint64_t*>(q->h_stage);
        cudaEvent_t done[2];
        cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming);
        cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming);
        const uint64_t nchunks = (m + chunk - 1) / chunk;
        int err = SJCS_OK;
        for (uint64_t c = 0; c <= nchunks && !err; ++c) {
            if (c < nchunks) {
                const uint64_t off = c * chunk, len = std::min(chunk, m - off);
                cudaError_t e = cudaMemcpyAsync(stage + (c & 1) * chunk, wide + off, len * sizeof(uint64_t),
                                                cudaMemcpyDeviceToHost, s);
                if (e == cudaSuccess) e = cudaEventRecord(done[c & 1], s);
                if (e != cudaSuccess) err = fail(SJCS_ERR_CUDA, "count read-back failed: %s", cudaGetErrorString(e));
            }
            if (c > 0 && !err) {
                const uint64_t p = c - 1, off = p * chunk, len = std::min(chunk, m - off);
                cudaError_t e = cudaEventSynchronize(done[p & 1]);
                if (e != cudaSuccess) err = fail(SJCS_ERR_CUDA, "count read-back failed: %s", cudaGetErrorString(e));
                else host_store(counts + off, stage + (p & 1) * chunk, len, accumulate != 0);
            }
        }
        cudaEventRecord(q->ev_d1, s);
        cudaStreamSynchronize(s);
        cudaEventDestroy(done[0]);
        cudaEventDestroy(done[1]);
        if (err) return err;
    }
    float ms = 0.f;
    q->last_d2h_ms = (cudaEventElapsedTime(&ms, q->ev_d0, q->ev_d1) == cudaSuccess) ? ms : 0.f;
    cudaGetLastError();
    return SJCS_OK;
}

int sjcs_query_read_counts_async(sjcs_ctx* ctx, sjcs_query* q, uint64_t* counts) {
    if (!valid_ctx(ctx)) return fail(SJCS_ERR_STATE, "invalid context");
    if (!valid_query(q) || q->ctx != ctx) return fail(SJCS_ERR_STATE, "query does not belong to this context");
    const uint64_t m = q->nhalos * (uint64_t)q->nrads;
    if (m == 0) return SJCS_OK;
    if (!counts) return fail(SJCS_ERR_INVALID, "counts is NULL");
    int rc = set_device(ctx);
    if (rc) return rc;
    if (!is_pinned(counts) || !is_pinned(counts + (m - 1)))
        return fail(SJCS_ERR_INVALID, "counts must be page-locked host memory for an asynchronous read");
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaStream_t s = ctx->s_read;
    // after everything queued on the count stream so far: q's upload and counts
    SJCS_CUDA_TRY(cudaEventRecord(q->ev_rq, ctx->s_count));
    SJCS_CUDA_TRY(cudaStreamWaitEvent(s, q->ev_rq, 0));
    StreamScratch scr(s);  // freed in stream order after the copy
    unsigned long long* wide = nullptr;
    SJCS_CUDA_TRY(scr.alloc(&wide, m * sizeof(uint64_t)));
    SJCS_CUDA_TRY(cudaEventRecord(q->ev_d0, s));
    k_widen_u32_u64<<<ctx->num_sms * 8, 256, 0, s>>>(q->counts, m, q->counts64, wide);
    SJCS_LAUNCH_CHECK();
    SJCS_CUDA_TRY(cudaMemcpyAsync(counts, wide, m * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    SJCS_CUDA_TRY(cudaEventRecord(q->ev_d1, s));
    q->read_queued = true;
    return SJCS_OK;
}

int sjcs_query_read_counts32_async(sjcs_ctx* ctx, sjcs_query* q, uint32_t* counts) {
    if (!valid_ctx(ctx)) return fail(SJCS_ERR_STATE, "invalid context");
    if (!valid_query(q) || q->ctx != ctx) return fail(SJCS_ERR_STATE, "query does not belong to this context");
    const uint64_t m = q->nhalos * (uint64_t)q->nrads;
    if (m == 0) return SJCS_OK;
    if (!counts) return fail(SJCS_ERR_INVALID, "counts is NULL");
    int rc = set_device(ctx);
    if (rc) return rc;
    if (!is_pinned(counts) || !is_pinned(counts + (m - 1)))
        return fail(SJCS_ERR_INVALID, "counts must be page-locked host memory for an asynchronous read");
    std::lock_guard<std::mutex> lk(ctx->mu);
    // without a fold every accumulated count is <= the query's bound <=
    // 2^32 - 1, so the 32-bit accumulators are the totals themselves
    if (q->folds)
        return fail(SJCS_ERR_INVALID, "the counts were folded into 64-bit totals %u time(s): read them as uint64",
                    q->folds);
    cudaStream_t s = ctx->s_read;
    SJCS_CUDA_TRY(cudaEventRecord(q->ev_rq, ctx->s_count));
    SJCS_CUDA_TRY(cudaStreamWaitEvent(s, q->ev_rq, 0));
    SJCS_CUDA_TRY(cudaEventRecord(q->ev_d0, s));
    SJCS_CUDA_TRY(cudaMemcpyAsync(counts, q->counts, m * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    SJCS_CUDA_TRY(cudaEventRecord(q->ev_d1, s));
    q->read_queued = true;
    return SJCS_OK;
}

int sjcs_query_wait_read(sjcs_query* q) {
    if (!valid_query(q)) return fail(SJCS_ERR_STATE, "invalid query");
    if (!q->read_queued) return SJCS_OK;
    SJCS_CUDA_TRY(cudaEventSynchronize(q->ev_d1));
    float ms = 0.f;
    q->last_d2h_ms = (cudaEventElapsedTime(&ms, q->ev_d0, q->ev_d1) == cudaSuccess) ? ms : 0.f;
    cudaGetLastError();
    return SJCS_OK;
}

int sjcs_query_device_counts(const sjcs_query* q, uint32_t** d_counts) {
    if (!valid_query(q) || !d_counts) return fail(SJCS_ERR_INVALID, "invalid argument");
    *d_counts = q->counts;
    return SJCS_OK;
}

int sjcs_query_reset(sjcs_ctx* ctx, sjcs_query* q) {
    if (!valid_ctx(ctx)) return fail(SJCS_ERR_STATE, "invalid context");
    if (!valid_query(q) || q->ctx != ctx) return fail(SJCS_ERR_STATE, "query does not belong to this context");
    int rc = set_device(ctx);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(ctx->mu);
    const uint64_t m = q->nhalos * (uint64_t)q->nrads;
    SJCS_CUDA_TRY(after_reads(q, ctx->s_count));
    if (m) SJCS_CUDA_TRY(cudaMemsetAsync(q->counts, 0, m * sizeof(uint32_t), ctx->s_count));
    if (m && q->counts64) SJCS_CUDA_TRY(cudaMemsetAsync(q->counts64, 0, m * sizeof(unsigned long long), ctx->s_count));
    SJCS_CUDA_TRY(cudaStreamSynchronize(ctx->s_count));
    q->bound = 0;
    q->folds = 0;
    clear_count_events(q);
    return SJCS_OK;
}

int sjcs_query_set_fold_limit(sjcs_ctx* ctx, sjcs_query* q, uint64_t limit) {
    if (!valid_ctx(ctx)) return fail(SJCS_ERR_STATE, "invalid context");
    if (!valid_query(q) || q->ctx != ctx) return fail(SJCS_ERR_STATE, "query does not belong to this context");
    if (limit < 1 || limit > 0xffffffffull)
        return fail(SJCS_ERR_INVALID, "the fold limit must lie in [1, 2^32 - 1] (got %llu)", (unsigned long long)limit);
    std::lock_guard<std::mutex> lk(ctx->mu);
    q->fold_limit = limit;
    return SJCS_OK;
}

int sjcs_query_folds(const sjcs_query* q, uint32_t* out) {
    if (!valid_query(q) || !out) return fail(SJCS_ERR_INVALID, "invalid argument");
    *out = q->folds;
    return SJCS_OK;
}

int sjcs_query_timing(const sjcs_query* q, sjcs_timing* out) {
    if (!valid_query(q) || !out) return fail(SJCS_ERR_INVALID, "invalid argument");
    SJCS_CUDA_TRY(cudaEventSynchronize(q->ev_last));
    sjcs_timing t{};
    for (size_t i = 0; i + 1 < q->count_events.size(); i += 2) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, q->count_events[i], q->count_events[i + 1]) == cudaSuccess) t.count_ms += ms;
        t.count_calls++;
    }
    t.d2h_ms = q->last_d2h_ms;
    cudaGetLastError();
    *out = t;
    return SJCS_OK;
}

int sjcs_query_destroy(sjcs_query* q) {
    if (!valid_query(q)) return fail(SJCS_ERR_STATE, "invalid query");
    sjcs_ctx* ctx = q->ctx;
    cudaSetDevice(ctx->device);
    std::lock_guard<std::mutex> lk(ctx->mu);
    free_query(q);
    return SJCS_OK;
}

int sjcs_multi_range_count(sjcs_ctx* ctx, const sjcs_index* idx, const float* halo_xyz, size_t stride_bytes,
                           uint64_t nhalos, const float* r2, int nrads, int flags, uint64_t* counts) {
    if (nhalos && !counts) return fail(SJCS_ERR_INVALID, "counts is NULL");
    sjcs_query* q = nullptr;
    int rc = sjcs_query_create(ctx, halo_xyz, stride_bytes, nhalos, r2, nrads, flags, &q);
    if (rc) return rc;
    rc = sjcs_query_count(ctx, q, idx);
    if (!rc) rc = sjcs_query_read_counts(ctx, q, counts, 1);
    sjcs_query_destroy(q);
    return rc;
}

int sjcs_radius_table(double minrad, double maxrad, int nrads, float* r2) {
    if (nrads <= 0 || !r2) return fail(SJCS_ERR_INVALID, "nrads must be > 0 and r2 non-NULL");
    if (minrad > maxrad) std::swap(minrad, maxrad);
    // Logspace(2.0, log2(min), log2(max), n, r): the reference is built with
    // -O2 -march=native, which contracts a + i*c into one fused multiply-add.
    const double a = std::log2(minrad), b = std::log2(maxrad);
    const double c = (b - a) / (nrads - 1);
    for (int i = 0; i < nrads - 1; ++i) r2[i] = (float)std::pow(2.0, std::fma((double)i, c, a));
    r2[nrads - 1] = (float)std::pow(2.0, b);
    for (int i = 0; i < nrads; ++i) r2[i] = r2[i] * r2[i];
    return SJCS_OK;
}

}  // extern "C"
