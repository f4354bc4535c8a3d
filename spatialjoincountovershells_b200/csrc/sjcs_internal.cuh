// Internal declarations shared by the CUDA translation units of libsjcs.so.
//
// Data layout in HBM (one particle file = one index):
//   pts[n]                float4 (x, y, z, cell key bits; the LSD build leaves 0),
//                         particles grouped by cell in cell order, so a warp
//                         reading 32 consecutive candidates issues one
//                         coalesced 128-bit load per lane
//   cell_start[ncells+1]  u32, first sorted slot of every cell; cells are
//                         numbered x-fastest ((cz*Gy + cy)*Gx + cx), so one
//                         (cy, cz) row of cells is one contiguous slot range.
// A query holds the halos sorted along a Morton curve (float4 x,y,z,orig-id)
// and u32 count accumulators [nhalos][nrads] in the caller's halo order.
#pragma once

#include <cuda_runtime.h>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/sjcs.h"

namespace sjcs {

// Periodic box edge of the reference (LOW_BOUND / UPP_BOUND,
// include/objects/RTree/Mbr.h:7-8).
constexpr float kBoxLow = 0.0f;
constexpr float kBoxUpp = 1000.0f;

void set_error(const char* fmt, ...);
int fail(int code, const char* fmt, ...);
void note_launch();  // counts this library's kernel launches (sjcs_launch_counter)

#define SJCS_CUDA_TRY(expr)                                                            \
    do {                                                                               \
        cudaError_t e_ = (expr);                                                       \
        if (e_ != cudaSuccess)                                                         \
            return ::sjcs::fail(SJCS_ERR_CUDA, "%s:%d: %s: %s", __FILE__, __LINE__,   \
                                #expr, cudaGetErrorString(e_));                        \
    } while (0)

#define SJCS_LAUNCH_CHECK()                                                            \
    do {                                                                               \
        ::sjcs::note_launch();                                                         \
        cudaError_t e_ = cudaGetLastError();                                           \
        if (e_ != cudaSuccess)                                                         \
            return ::sjcs::fail(SJCS_ERR_CUDA, "%s:%d: kernel launch: %s", __FILE__,   \
                                __LINE__, cudaGetErrorString(e_));                     \
    } while (0)

// Stream-ordered scratch: every buffer allocated through it is released with
// cudaFreeAsync on the same stream when the holder goes out of scope, so
// error returns do not leak and no host synchronisation is needed.
struct StreamScratch {
    cudaStream_t s;
    std::vector<void*> ptrs;
    explicit StreamScratch(cudaStream_t st) : s(st) {}
    StreamScratch(const StreamScratch&) = delete;
    StreamScratch& operator=(const StreamScratch&) = delete;
    template <class T>
    cudaError_t alloc(T** p, size_t bytes) {
        cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(p), bytes ? bytes : 16, s);
        if (e == cudaSuccess) ptrs.push_back(static_cast<void*>(*p));
        return e;
    }
    ~StreamScratch() {
        for (void* p : ptrs) cudaFreeAsync(p, s);
    }
};

// Uniform cell grid over [0,1000)^3.  Coordinates outside the box clamp into
// the edge cells, so the cell of any value is monotone in the value and a
// query box [lo, hi] always covers the cells of every point inside it.
struct GridGeom {
    float inv_h[3];   // cells per unit length, G/1000 in fp32
    int G[3];         // cells per axis
    uint64_t ncells;  // G[0]*G[1]*G[2]
};

__device__ __forceinline__ int cell_of(float v, float inv_h, int G) {
    // __fmul_rn: never contracted, so build and query compute the same cell.
    float t = floorf(__fmul_rn(v, inv_h));
    t = fminf(fmaxf(t, 0.0f), (float)(G - 1));  // fmaxf(NaN, 0) == 0
    return (int)t;
}

__device__ __forceinline__ uint32_t cell_key(const GridGeom& g, float x, float y, float z) {
    const uint32_t cx = (uint32_t)cell_of(x, g.inv_h[0], g.G[0]);
    const uint32_t cy = (uint32_t)cell_of(y, g.inv_h[1], g.G[1]);
    const uint32_t cz = (uint32_t)cell_of(z, g.inv_h[2], g.G[2]);
    return (cz * (uint32_t)g.G[1] + cy) * (uint32_t)g.G[0] + cx;
}

// 10-bit-per-axis Morton code used only to order halos for cache locality.
__device__ __forceinline__ uint32_t spread3_10(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}
__device__ __forceinline__ uint32_t morton30(float x, float y, float z) {
    const float s = 1024.0f / 1000.0f;
    const uint32_t qx = (uint32_t)cell_of(x, s, 1024);
    const uint32_t qy = (uint32_t)cell_of(y, s, 1024);
    const uint32_t qz = (uint32_t)cell_of(z, s, 1024);
    return spread3_10(qx) | (spread3_10(qy) << 1) | (spread3_10(qz) << 2);
}

}  // namespace sjcs

// ---- opaque ABI objects ----------------------------------------------------

struct sjcs_ctx {
    uint32_t magic;
    int device;
    int num_sms;
    cudaStream_t s_build;  // particle copies + index builds
    cudaStream_t s_count;  // halo upload/sort, shell counts, count read-back
    cudaStream_t s_read = nullptr;  // asynchronous count read-back
    cudaStream_t s_h2d = nullptr;   // uploads of host particle files
    std::mutex mu;
    std::map<std::string, sjcs_schedule> tuned;  // autotuned schedules by workload shape
    bool overlap = false;    // builds' kernels may run beside queued counts
    cudaEvent_t ev_counts = nullptr;  // marks the counts queued so far (build ordering)
    // File ingest (sjcs_index_build_file): pinned staging slots, one per
    // reader thread, each with the event of the last copy out of it.
    std::mutex ring_mu;
    char* ring = nullptr;
    std::vector<cudaEvent_t> ring_ev;
    // Small parameter uploads (radius and shell tables): page-locked slots,
    // each with the event of the last copy out of it, because a copy from
    // pageable memory may make the host wait for its stream.
    std::mutex param_mu;
    char* param_ring = nullptr;
    std::vector<cudaEvent_t> param_ev;
    uint32_t param_next = 0;
};

namespace sjcs {
struct LearnedLeaf;
struct LearnedRoot;
}

struct sjcs_index {
    uint32_t magic;
    sjcs_ctx* ctx;
    int kind;
    uint64_t n;
    sjcs::GridGeom geom;   // grid kind
    float4* pts;           // n sorted particles
    uint32_t* cell_start;  // grid: geom.ncells + 1 entries; Morton kinds: 8^level + 1 entries
    int level;             // Morton kinds: cell level of the offset table and of the lookups
    bool verify;           // learned kind: the model was checked against the table
    sjcs::LearnedLeaf* leaves;  // learned kind: 4096 leaves
    sjcs::LearnedRoot* root;    // learned kind: root model and training statistics
    cudaEvent_t ev_start, ev_h2d, ev_ready, ev_train0;  // ev_train0: sort done, training starts
    bool had_h2d;
};

struct sjcs_query {
    uint32_t magic;
    sjcs_ctx* ctx;
    uint64_t nhalos;
    int nrads;
    int flags;
    int pad;            // power of two >= nrads (binary-search table size)
    bool monotone;      // r2 non-decreasing and free of NaN: fast binning
    float R;            // (float)sqrt((double)r2[nrads-1]), as MultiRangeCount.c:19
    float half;         // query half-width: R (periodic) or r2[nrads-1] (non-periodic, MultiRangeCount.c:81)
    float r2max;
    float4* halos;      // Morton-sorted halos, .w = original index bits
    uint32_t* counts;   // [nhalos][nrads], caller's halo order
    float* d_r2;        // [pad], entries past nrads = +inf
    // Shell lookup on the bit pattern of dist (non-negative floats order like
    // their bits): slot j covers keys [lut_k0 + j<<lut_shift, ...+1<<lut_shift)
    // and holds #{i : r2[i] <= first value of the slot}; every slot holds at
    // most one table value, so one compare against r2[slot value] finishes.
    uint32_t* d_lut;    // [nlut]; nlut == 0: no LUT, binary search instead
    int nlut;
    uint32_t lut_k0;
    int lut_shift;
    uint32_t* h_stage;  // pinned staging for count read-back
    size_t h_stage_elems;
    std::vector<cudaEvent_t> count_events;  // (start, end) pairs, one per count call since reset
    cudaEvent_t ev_last;                    // end of the last count call
    cudaEvent_t ev_d0, ev_d1;
    cudaEvent_t ev_rq = nullptr;  // s_count's work when an asynchronous read was queued
    bool read_queued = false;     // an asynchronous read ended at ev_d1 (maybe still running)
    float last_d2h_ms;
    sjcs_schedule sched;  // count schedule (SJCS_SCHED_AUTO by default)
    // 64-bit totals.  The u32 accumulators hold the counts since the last
    // fold; before a count call could push one of them past fold_limit, the
    // query adds them into counts64 (allocated at the first fold) and clears
    // them, so the totals never wrap, whatever the number of files.
    unsigned long long* counts64 = nullptr;
    uint64_t bound = 0;                    // upper bound of any u32 accumulator since the last fold
    uint64_t fold_limit = 0xffffffffull;   // largest value a u32 accumulator may reach
    uint32_t folds = 0;
};

namespace sjcs {
// Largest amount one count of n particles can add to a single (halo, shell)
// accumulator.  A particle is counted at most once per periodic image, and
// it can lie inside two images' query boxes only when a box is at least 1000
// wide (R >= 500; 499 leaves room for the fp32 rounding of the box bounds),
// so below that every particle counts at most once.  Non-periodic queries
// search one image.
inline uint64_t count_call_bound(int flags, float r2max, uint64_t n) {
    const float R = (float)std::sqrt((double)r2max);
    const bool multi = (flags & SJCS_QUERY_PERIODIC) && !(R < 499.0f);  // NaN R: assume the worst
    return multi ? 8 * n : n;
}

constexpr uint32_t kCtxMagic = 0x534a4358u;    // "SJCX"
constexpr uint32_t kIndexMagic = 0x534a4958u;  // "SJIX"
constexpr uint32_t kQueryMagic = 0x534a5158u;  // "SJQX"

// index_build.cu
int build_grid_index(sjcs_ctx* ctx, const float* d_xyz, uint64_t n, const GridGeom& g,
                     sjcs_index* idx, cudaStream_t s);
GridGeom auto_grid(uint64_t n, float radius_hint, const uint32_t* grid_req);

// learned_index.cu: Morton kinds (plain Morton offset table, learned rank model)
int morton_auto_level(uint64_t n, float radius_hint);
int build_morton_index(sjcs_ctx* ctx, const float* d_xyz, uint64_t n, int level, bool learned, bool verify,
                       sjcs_index* idx, cudaStream_t s);

// morton_count.cu (sc as for launch_shell_count)
struct Schedule;
int launch_morton_count(sjcs_ctx* ctx, const sjcs_query* q, const sjcs_index* idx, cudaStream_t s,
                        const Schedule* sc = nullptr);

// sjcs_abi.cu: query preparation on stream s (radius table, shell lookup,
// zeroed accumulators, Morton-sorted halos) and schedule resolution
int query_prepare(sjcs_ctx* ctx, const float* d_halo_xyz, size_t stride, uint64_t nhalos, const float* r2,
                  int nrads, int flags, sjcs_query* q, cudaStream_t s);
struct Schedule;
Schedule schedule_for(sjcs_ctx* ctx, const sjcs_query* q, const sjcs_index* idx);
Schedule resolve(const sjcs_schedule& in);

// decode.cu: compressed (Gadget-encoded) particles
struct GadgetDecode {
    float cell_interval;  // BoxSize / n1d (fp32, as the reference stores it)
    float disp_min;
    double unitsep;       // (disp_max - disp_min) / 2^pos_bits
    long long id_start;
    long long ng1d, ng2d, ng3d;  // lattice per axis, per plane, total
    int nt1d, nt2d;              // tiles (one)
};
int gadget_decode_params(const void* header, GadgetDecode* out);
int launch_decode(const uint16_t* d_uv, uint64_t n, const GadgetDecode& g, float* d_xyz, cudaStream_t s);

// query_prep.cu
int sort_halos(sjcs_ctx* ctx, const float* d_halo_xyz, size_t stride_bytes, uint64_t nhalos,
               float4* out, cudaStream_t s);

// shell_count.cu.  sc == nullptr or mode SJCS_SCHED_STATIC: static
// schedule; SJCS_SCHED_QUEUE: persistent work queue (allocates scratch).
struct Schedule {
    int mode;             // SJCS_SCHED_STATIC or SJCS_SCHED_QUEUE (resolved, never AUTO)
    uint32_t piece;       // candidates per piece of a heavy halo
    uint32_t max_pieces;  // most warps sharing one halo
    uint32_t single;      // estimate (power of two) from which a halo is an item of its own
};
int launch_shell_count(sjcs_ctx* ctx, const sjcs_query* q, const sjcs_index* idx, cudaStream_t s,
                       const Schedule* sc = nullptr);
// k (1..kMaxFusedIndexes) grid indexes of one geometry counted in one
// static-schedule pass: the counts of k launch_shell_count calls.
constexpr int kMaxFusedIndexes = 4;
int launch_shell_count_multi(sjcs_ctx* ctx, const sjcs_query* q, const sjcs_index* const* idx, int k,
                             cudaStream_t s);

// scan.cu: exclusive prefix sum of m u32 values, in place.  `partials`
// (scan_partials_needed(m) u32) may be given; otherwise it is allocated.
int exclusive_scan_u32(uint32_t* d_data, uint64_t m, cudaStream_t s, uint32_t* partials = nullptr);
uint64_t scan_partials_needed(uint64_t m);

// index_build.cu: the stable LSD grid build on caller-provided buffers (no
// allocation; the fixed-buffer entry point and cell keys of more than 30 bits).
struct GridBuildBuffers {
    float4* pts;          // n sorted particles (output)
    uint32_t* cell_start; // ncells + 1 (output)
    uint32_t* kfinal;     // n
    uint32_t* kx;         // n (needed for two or more passes)
    uint4* px;            // n
    uint32_t* ky;         // n (needed for three or more passes)
    uint4* py;            // n
    uint32_t* hist;       // 2^digit_bits * ceil(n / 4096)
    uint32_t* partials;   // scan_partials_needed(2^digit_bits * ceil(n / 4096)), or null
    void* gaps;           // kGridGaps gap records (12 bytes each)
    uint32_t* ngaps;      // 1
    int digit_bits;       // radix digit: 9, or 8 (also for 0)
};
constexpr uint32_t kGridGaps = 1u << 16;
int grid_key_bits(const GridGeom& g);
int grid_digit_bits(const GridGeom& g);  // LSD build: 9 for 25-27-bit cell keys, else 8
int build_grid_into(const float* d_xyz, uint64_t n, const GridGeom& g, const GridBuildBuffers& b, cudaStream_t s);
// cell_start[c] = first slot of cell c, from the cell ids of the sorted particles.
int fill_cell_table(const uint32_t* sorted_cells, uint64_t n, uint64_t ncells, uint32_t* cell_start, void* gaps,
                    uint32_t* ngaps, cudaStream_t s);
}  // namespace sjcs
