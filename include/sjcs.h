/*
 * sjcs.h -- C ABI of the B200 (sm_100a) spatial-join-count-over-shells hot path.
 *
 * The reference program (astr_rcount) builds one STR tree per particle file and
 * then, for every halo, counts the particles that fall into each of n radial
 * shells under a periodic [0,1000)^3 box.  Its index layer is a per-halo C API:
 *
 *   constructArraySTR / insertDataArraySTR / makeTreeWithSameThreadPoolArraySTR
 *       include/objects/ArraySTR/ArraySTR.h:52-56
 *   multiRangeCountWithPriodicBoundArraySTR / multiRangeCountArraySTR
 *       include/objects/ArraySTR/MultiRangeCount.h:10-11
 *   MultiRangeCountContext {nrads, central, radiuses (squared, ascending), counts}
 *       include/objects/RTree/MultiRangeCountContext.h:7-18
 *   destructArraySTR  include/objects/ArraySTR/ArraySTR.h:53
 *
 * and the driver calls it once per halo from a thread pool
 * (threadJoin, src/astr_rcount/main.c:795-826).  A per-halo call cannot feed a
 * GPU, so this ABI keeps the same seam -- build an index over one particle
 * file, count shells for a set of halos against it, accumulate counts across
 * files, destroy the index -- but batched over all halos at once.
 *
 * Conventions
 *  - Every entry point returns an int status (SJCS_OK == 0).  On failure,
 *    sjcs_last_error() returns a message for the calling thread.
 *  - Objects are opaque handles owned by the caller.  A context owns one GPU
 *    and its streams; indexes and queries belong to the context that made them.
 *  - Counts follow the reference: per halo, per shell, unsigned 64-bit on the
 *    host, INCREMENTED (never cleared) by each particle file's pass.  A particle
 *    lands in the first shell i with dist < r2[i] (dist = squared distance in
 *    fp32, (dx*dx + dy*dy) + dz*dz, no FMA) after passing the inclusive query
 *    box test; periodic images follow the reference's out-of-bound rule.
 *  - Pointers named d_* are device pointers; all others are host pointers.
 *  - No entry point falls back to a CPU implementation: without a usable GPU
 *    they fail with SJCS_ERR_CUDA.
 */
#ifndef SJCS_H
#define SJCS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define SJCS_OK            0
#define SJCS_ERR_INVALID   1  /* bad argument (null pointer, bad size, bad radius table) */
#define SJCS_ERR_CUDA      2  /* CUDA runtime error or no usable device */
#define SJCS_ERR_NOMEM     3  /* device or pinned-host allocation failed */
#define SJCS_ERR_STATE     4  /* object used with another context, or after destroy */

/* index kinds */
#define SJCS_INDEX_GRID     0 /* uniform cell grid: particles grouped by cell in cell order, cell-offset table */
#define SJCS_INDEX_LEARNED  1 /* particles sorted by 63-bit Morton key; cell ranks from a two-level
                                 piecewise-linear model (1 root + 4096 fp32 linear leaves, per-leaf
                                 max error) corrected by a bounded exact search; the Morton
                                 cell-offset table is kept as fallback and judge */
#define SJCS_INDEX_MORTON   2 /* particles sorted by 63-bit Morton key, plain Morton cell-offset table */

/* index option flags */
#define SJCS_INDEX_VERIFY   0x1 /* learned kind: after training, compare the corrected model rank of
                                   every cell boundary with the offset table; on any mismatch the
                                   index answers from the table */

/* count schedules: how the count kernel hands halos to warps */
#define SJCS_SCHED_AUTO    0 /* the context's autotuned choice for this workload shape, else STATIC */
#define SJCS_SCHED_STATIC  1 /* warps take halos strided over the Morton order, in batches of 32 */
#define SJCS_SCHED_QUEUE   2 /* persistent warps pull work from a queue ordered by estimated candidate
                                count (largest first); heavy halos are split into pieces that several
                                warps count together (every index kind) */

/* query flags */
#define SJCS_QUERY_PERIODIC     0x1 /* periodic images, as multiRangeCountWithPriodicBoundArraySTR */
#define SJCS_QUERY_NONPERIODIC  0x0 /* single image, as multiRangeCountArraySTR (MultiRangeCount.c:75-83) */

typedef struct sjcs_ctx   sjcs_ctx;   /* one GPU: streams, scratch, tuning cache */
typedef struct sjcs_index sjcs_index; /* device-resident index over one particle file */
typedef struct sjcs_query sjcs_query; /* device-resident halos + radius table + u32 count accumulators */
typedef struct sjcs_step  sjcs_step;  /* one particle file's step (copy, build, count) captured as a CUDA graph */
typedef struct sjcs_server sjcs_server; /* request loop over device-resident indexes */

/* Build options.  Zero-initialised options select an automatic grid for the
 * plain index (sized from n and radius_hint). */
typedef struct sjcs_index_opts {
    int      kind;         /* SJCS_INDEX_GRID, SJCS_INDEX_LEARNED or SJCS_INDEX_MORTON */
    float    radius_hint;  /* largest search radius expected (sqrt of r2[nrads-1]); 0 = unknown */
    uint32_t grid[3];      /* grid kind: cells per axis (x, y, z), 0 = automatic.  Morton kinds:
                              grid[0] = cell level L in [1,10] (cells of 1000/2^L per axis,
                              8^L + 1 table entries), 0 = automatic; grid[1], grid[2] zero */
    uint32_t flags;        /* SJCS_INDEX_VERIFY */
    uint32_t reserved[3];  /* must be zero */
} sjcs_index_opts;

/* Training record of a learned index (after sjcs_index_wait). */
typedef struct sjcs_learned_info {
    uint32_t level;       /* Morton cell level of the lookups */
    uint32_t leaves;      /* leaf models (4096) */
    uint32_t nonempty;    /* leaves holding at least one key */
    uint32_t max_err;     /* largest per-leaf error bound, in ranks */
    double   mean_err;    /* mean error bound over non-empty leaves */
    uint64_t checked;     /* cell boundaries judged against the table (0 without SJCS_INDEX_VERIFY) */
    uint64_t mismatches;  /* judged lookups that disagreed (> 0: the index answers from the table) */
    float    sort_ms;     /* key, sort and offset table kernels */
    float    train_ms;    /* training (and judge) kernels */
} sjcs_learned_info;

/* Timing from CUDA events on the stream that ran the work (milliseconds; 0
 * where not applicable).  For an index: its copy and build.  For a query: the
 * count kernels of every sjcs_query_count since creation or the last
 * sjcs_query_reset (count_ms is their sum, count_calls their number) and the
 * last read-back. */
typedef struct sjcs_timing {
    float h2d_ms;         /* host-to-device copy inside the call */
    float build_ms;       /* index build kernels (keys, sort or partition, offsets) */
    float count_ms;       /* shell-count kernel(s) */
    float d2h_ms;         /* device-to-host read-back (widening kernel + copy) */
    uint32_t count_calls; /* number of sjcs_query_count calls summed in count_ms */
} sjcs_timing;

/* A count schedule.  Zero fields take the defaults. */
typedef struct sjcs_schedule {
    int      mode;        /* SJCS_SCHED_* */
    uint32_t piece;       /* queue: candidates per piece of a heavy halo, i.e. the work one warp
                             takes at a time (rounded up to a power of two; 0 = 8192) */
    uint32_t max_pieces;  /* queue: most warps counting one halo together (0 = 64) */
    uint32_t single;      /* queue: estimated candidates from which a halo is a queue item of its
                             own; lighter halos share items, up to 32 halos and about `piece`
                             candidates per item (power of two; 0 = piece/8) */
} sjcs_schedule;

/* ---- errors / version ---------------------------------------------------- */

/* Message for the last failing call on this thread ("" if none).  Replaces the
 * reference's stderr prints before NULL returns (e.g. src/Gadget/BufHalo.c:85-98). */
const char *sjcs_last_error(void);
/* Library version string. */
const char *sjcs_version(void);

/* ---- context ------------------------------------------------------------- */

/* Open a context on CUDA device `device`.  The reference's analogue is the
 * SameThreadPool the driver builds before the file loop
 * (src/astr_rcount/main.c:245, constructSameThreadPool). */
int sjcs_ctx_create(int device, sjcs_ctx **out);
/* Wait for all work of the context and release it (main.c:263,
 * destructSameThreadPool). */
int sjcs_ctx_destroy(sjcs_ctx *ctx);
/* Block until every stream of the context is idle (the reference's
 * waitCompletionSameThreadPool, src/objects/SameThreadPool/SameThreadPool.c:62-68). */
int sjcs_ctx_sync(sjcs_ctx *ctx);
/* Number of streaming multiprocessors of the context's device. */
int sjcs_ctx_num_sms(const sjcs_ctx *ctx, int *out);
/* Device memory is taken from the device's stream-ordered pool, which keeps
 * freed blocks for reuse.  sjcs_ctx_reserve grows the pool to hold at least
 * `bytes` (so later builds and queries of that size take no new memory from
 * the driver); sjcs_ctx_trim returns every unused block to the driver.  Both
 * wait for the context's work.  *free_bytes / *pool_bytes report the device's
 * free memory and the pool's size (either may be NULL). */
int sjcs_ctx_reserve(sjcs_ctx *ctx, uint64_t bytes);
int sjcs_ctx_trim(sjcs_ctx *ctx);
int sjcs_ctx_memory(sjcs_ctx *ctx, uint64_t *free_bytes, uint64_t *pool_bytes);
/* The context's CUDA streams (cudaStream_t): which = 0 build stream (copies and
 * index builds), 1 count stream (halo preparation, counts, read-back).  Lets a
 * caller order its own work or timing events against the library's. */
int sjcs_ctx_stream(const sjcs_ctx *ctx, int which, void **stream);
/* Number of kernels this library has launched in this process so far. */
uint64_t sjcs_launch_counter(void);
/* Whether an index build's kernels may run beside the counts already queued
 * on the context (overlap != 0), or wait for them (overlap == 0, the
 * default).  Either way the build's host-to-device copy overlaps the counts.
 * On one GPU the two kinds of kernel compete for the same SMs and L2, so
 * running them back to back is faster than side by side; the reference's
 * backlog pipeline (src/astr_rcount/main.c:266-350) overlaps them because its
 * builds and searches use separate CPU threads. */
int sjcs_ctx_set_overlap(sjcs_ctx *ctx, int overlap);

/* ---- pinned host memory (for the driver's file reads) -------------------- */

/* Page-locked host buffer, so that file reads land in memory the copy engines
 * can read at full speed.  Replaces the malloc in reallocBufFloatVector3D
 * (src/Gadget/BufVector3D.c, used by readDecodedParticles :285-308). */
int sjcs_host_alloc(size_t bytes, void **out);
int sjcs_host_free(void *p);

/* ---- index (one particle file) ------------------------------------------- */

/* Build an index over n particles given as x,y,z float triplets in HOST
 * memory (the layout of a decoded particle file).  The copy to the device and
 * the build run asynchronously on the context's build stream; the call returns
 * once the work is queued and the host buffer may be reused only after
 * sjcs_index_wait (or any later call that waits on the index).
 * Replaces constructArraySTR + insertDataArraySTR x n +
 * makeTreeWithSameThreadPoolArraySTR (include/objects/ArraySTR/ArraySTR.h:52-56,
 * called from constructIndexWithSameThreadPool, src/astr_rcount/main.c:732-786).
 * n == 0 is allowed and yields an index that matches nothing (the reference
 * refuses to build it, src/objects/ArraySTR/Build.c:860-863). */
int sjcs_index_build(sjcs_ctx *ctx, const float *xyz, uint64_t n,
                     const sjcs_index_opts *opts, sjcs_index **out);
/* Same, with the particles already in device memory (d_xyz, n*3 floats).
 * The build runs on the context's build stream (sjcs_ctx_stream, which = 0):
 * work that writes d_xyz on another stream must be ordered before it by the
 * caller (e.g. cudaEventRecord on the producer's stream and
 * cudaStreamWaitEvent on the build stream), and d_xyz must stay untouched
 * until sjcs_index_wait.  The Python binding does both for CUDA tensors. */
int sjcs_index_build_device(sjcs_ctx *ctx, const float *d_xyz, uint64_t n,
                            const sjcs_index_opts *opts, sjcs_index **out);
/* Same, reading a decoded particle file (x,y,z float triplets, count =
 * file size / 12, as readDecodedParticles, src/Gadget/BufVector3D.c:285-308).
 * Several threads read the file in 8 MB chunks into a small page-locked
 * staging area owned by the context (allocated on first use) and each chunk is
 * copied to the device as soon as it is read, so no page-locked copy of the
 * whole file is made and reading overlaps the upload.  Returns once the file
 * is read and the copies and the build are queued.  A missing or unreadable
 * file fails with SJCS_ERR_INVALID. */
int sjcs_index_build_file(sjcs_ctx *ctx, const char *path, const sjcs_index_opts *opts, sjcs_index **out);
/* Get a context ready for particle files of up to max_particles: page-lock
 * the staging slots of sjcs_index_build_file and grow the device pool to hold
 * one file's upload, index and build scratch, so the first file pays for
 * neither.  It may run on a helper thread while the caller does host work
 * that does not use the context (the driver parses the halo file meanwhile).
 * No counterpart in the reference (its buffers are allocated per file). */
int sjcs_ctx_prepare_files(sjcs_ctx *ctx, uint64_t max_particles);
/* Same, from compressed (Gadget-encoded) particles: n uint16 triplets in HOST
 * memory (the displacement record of a compressed file) and the file's
 * 256-byte header (the layout of GadgetHeader, include/Gadget/GadgetHeader.h:4-27;
 * sjcs_gadget_header in sjcs_host.h).  The triplets are copied to the device
 * and decoded there.  Replaces the decode loop of
 * constructIndexWithSameThreadPool (src/astr_rcount/main.c:739-763:
 * decodeCompressedParticle per particle, src/Gadget/BufVector3D.c:169-201)
 * and the build. */
int sjcs_index_build_compressed(sjcs_ctx *ctx, const uint16_t *uv, uint64_t n, const void *gadget_header,
                                const sjcs_index_opts *opts, sjcs_index **out);
/* Decode only, on the device: n triplets (host) into n x,y,z floats (host),
 * exactly as decodeCompressedParticle computes them.  Blocks. */
int sjcs_decode_compressed(sjcs_ctx *ctx, const uint16_t *uv, uint64_t n, const void *gadget_header, float *xyz);
/* Block until the index is built. */
int sjcs_index_wait(sjcs_index *idx);
/* Number of particles in the index (getNumberOfDataArraySTR, ArraySTR.h:58). */
int sjcs_index_size(const sjcs_index *idx, uint64_t *out);
/* Cells per axis actually used by a grid index (2^L per axis for the Morton
 * kinds). */
int sjcs_index_grid(const sjcs_index *idx, uint32_t out[3]);
/* Training record of a learned index; waits for the build.  No counterpart in
 * the reference (its R-tree has no learned component). */
int sjcs_index_learned_info(sjcs_index *idx, sjcs_learned_info *out);
/* Timing of the build (valid after sjcs_index_wait). */
int sjcs_index_timing(const sjcs_index *idx, sjcs_timing *out);
/* Release the index after all queued work that reads it
 * (destructArraySTR, include/objects/ArraySTR/ArraySTR.h:53). */
int sjcs_index_destroy(sjcs_index *idx);

/* ---- query (halos + shells + count accumulators) ------------------------- */

/* Upload nhalos halo centres and the squared-radius table and prepare device
 * count accumulators (zeroed).  halo_xyz points at the first halo's x; halos
 * are `stride_bytes` apart with y,z following x (stride 24 and a pointer to
 * Halo.point reads the reference's BufHalo array directly,
 * include/Gadget/BufHalo.h:26-30; stride 12 reads packed triplets).
 * r2 holds nrads squared radii as built by the driver (Logspace then r*r,
 * src/astr_rcount/main.c:644-649); any table is accepted -- a non-decreasing,
 * finite one takes the fast binning path, anything else the reference's
 * first-match scan.  flags: SJCS_QUERY_PERIODIC or SJCS_QUERY_NONPERIODIC.
 * The halos go up on the context's upload stream (beside counts already
 * queued); halos in page-locked memory are read after the call returns and
 * must stay unchanged until the query's first count has finished
 * (sjcs_query_wait), pageable ones are copied before it returns.
 * Replaces constructMultiRangeCountContext + the per-row set-up in threadJoin
 * (src/objects/RTree/MultiRangeCountContext.c:8-25, src/astr_rcount/main.c:816-821). */
int sjcs_query_create(sjcs_ctx *ctx, const float *halo_xyz, size_t stride_bytes,
                      uint64_t nhalos, const float *r2, int nrads, int flags,
                      sjcs_query **out);
/* Same, halos already in device memory; the halo upload runs on the count
 * stream (sjcs_ctx_stream, which = 1), which the caller orders after the
 * halos' producer. */
int sjcs_query_create_device(sjcs_ctx *ctx, const float *d_halo_xyz, size_t stride_bytes,
                             uint64_t nhalos, const float *r2, int nrads, int flags,
                             sjcs_query **out);
/* Count every halo of the query against one index and add the counts to the
 * query's device accumulators (queued on the count stream after the index's
 * build).  Replaces one file's pass of threadJoin, i.e. nhalos calls of
 * multiRangeCountWithPriodicBoundArraySTR (include/objects/ArraySTR/MultiRangeCount.h:11)
 * or, without SJCS_QUERY_PERIODIC, of multiRangeCountArraySTR (:10). */
int sjcs_query_count(sjcs_ctx *ctx, sjcs_query *q, const sjcs_index *idx);
/* The counts of sjcs_query_count(ctx, q, idx[i]) for i = 0 .. k-1, added to
 * the query's accumulators.  Runs of up to 4 grid indexes with the same cell
 * grid (equal particle counts and radius hints give the same automatic grid),
 * under the static schedule, are counted in one pass: each halo's rows are
 * planned once and its counters flushed once for the whole run, and the
 * indexes' row loads overlap each other's tests.  Any other index is counted
 * on its own.  The reference's file loop (src/astr_rcount/main.c:676-826)
 * counts one file at a time; this is the same sum over files with every
 * file's index resident at once. */
int sjcs_query_count_many(sjcs_ctx *ctx, sjcs_query *q, const sjcs_index *const *idx, int k);
/* Block until the last sjcs_query_count queued on q has finished (builds
 * queued on the build stream keep running). */
int sjcs_query_wait(sjcs_query *q);
/* Copy the accumulated counts to host memory as uint64 [nhalos][nrads] in the
 * order the halos were given.  accumulate != 0 adds them to `counts` (the
 * reference's += on its calloc'd ulong_t array, src/astr_rcount/main.c:651),
 * accumulate == 0 overwrites.  Blocks until the copy is done. */
int sjcs_query_read_counts(sjcs_ctx *ctx, sjcs_query *q, uint64_t *counts, int accumulate);
/* Queue a read-back of the accumulated counts (uint64 [nhalos][nrads], caller's
 * halo order, overwriting) into page-locked host memory (cudaMallocHost,
 * cudaHostRegister or sjcs_host_alloc) and return at once.  The copy runs on
 * the context's read-back stream after every count queued on q so far, so it
 * overlaps uploads and builds queued afterwards (host-to-device and
 * device-to-host copies use separate copy engines).  The counts are in place
 * when sjcs_query_wait_read returns; until then `counts` must stay valid.
 * Later counts, resets and sjcs_query_destroy on q wait for the read on the
 * device.  Non-page-locked `counts` fail with SJCS_ERR_INVALID.  The
 * asynchronous form of sjcs_query_read_counts(..., accumulate = 0); the
 * reference reads its counts in place after the last file (main.c:651). */
int sjcs_query_read_counts_async(sjcs_ctx *ctx, sjcs_query *q, uint64_t *counts);
/* sjcs_query_read_counts_async with uint32 counts [nhalos][nrads]: a direct
 * copy of the query's 32-bit accumulators, half the bytes of the uint64 read.
 * Exact while the query has not folded (every count is then at most the
 * query's bound, which stays <= 2^32 - 1 until a fold); after a fold
 * (sjcs_query_folds > 0) it fails with SJCS_ERR_INVALID and the counts must be
 * read as uint64.  Completion is awaited with sjcs_query_wait_read. */
int sjcs_query_read_counts32_async(sjcs_ctx *ctx, sjcs_query *q, uint32_t *counts);
/* Block until the last read queued by sjcs_query_read_counts_async (or its
 * uint32 form) on q is in
 * host memory (returns at once when none is pending). */
int sjcs_query_wait_read(sjcs_query *q);
/* Device pointer to the query's uint32 accumulators [nhalos][nrads] in the
 * order the halos were given (valid until sjcs_query_destroy).  They hold the
 * counts since the query's last fold (sjcs_query_folds; with no fold, all of
 * them). */
int sjcs_query_device_counts(const sjcs_query *q, uint32_t **d_counts);
/* The reference accumulates unsigned 64-bit counts over any number of
 * particle files (ulong_t counts[], src/astr_rcount/main.c:651).  A query
 * accumulates on the device in uint32 and keeps an upper bound of what its
 * counts since the last fold can hold (each sjcs_query_count or step launch
 * adds n, or 8n for periodic queries with R >= 499, whose particles can lie in
 * several images' boxes); before a call could carry an accumulator past the
 * fold limit, the query adds the uint32 accumulators into 64-bit device
 * totals and clears them (a fold).  Read-backs return the 64-bit totals, so
 * counts never wrap.  A single call that could add more than the limit by
 * itself (more than 2^32 - 1 particles, or 2^29 with R >= 499) fails with
 * SJCS_ERR_INVALID.
 * sjcs_query_set_fold_limit lowers the limit (default and maximum 2^32 - 1;
 * at least 1): folds then happen sooner, with the same results -- a test
 * hook that exercises the fold on small inputs.  sjcs_query_folds gives the
 * number of folds since creation or the last reset.  Neither has a
 * counterpart in the reference. */
int sjcs_query_set_fold_limit(sjcs_ctx *ctx, sjcs_query *q, uint64_t limit);
int sjcs_query_folds(const sjcs_query *q, uint32_t *out);
/* Zero the accumulators and the timing history (start a new run over the
 * same halos). */
int sjcs_query_reset(sjcs_ctx *ctx, sjcs_query *q);
/* Count-kernel time summed over the sjcs_query_count calls since creation or
 * reset, and the last read-back time (blocks until those are done). */
int sjcs_query_timing(const sjcs_query *q, sjcs_timing *out);
int sjcs_query_destroy(sjcs_query *q);

/* ---- captured file steps (no counterpart in the reference: its per-file
 * step is constructIndexWithSameThreadPool + threadJoin + destructIndex,
 * src/astr_rcount/main.c:176-243) ---------------------------------------- */

/* Capture one whole file step as a CUDA graph: the copy of n particles from
 * the PINNED host buffer host_xyz (sjcs_host_alloc), the index build with
 * `opts`, the count of every halo of q against it (added to q's
 * accumulators, with q's schedule as resolved now) and the release of the
 * index.  Nothing runs at creation.  The graph's memory (particles, index,
 * scratch) is reserved once and reused by every launch. */
int sjcs_step_create(sjcs_ctx *ctx, sjcs_query *q, const float *host_xyz, uint64_t n,
                     const sjcs_index_opts *opts, sjcs_step **out);
/* Replay the step on the current contents of its host buffer (one graph
 * launch, ordered after all earlier work of the context; later counts and
 * read-backs of q are ordered after it).  The buffer may be refilled once
 * sjcs_step_wait has returned. */
int sjcs_step_launch(sjcs_ctx *ctx, sjcs_step *st);
int sjcs_step_wait(sjcs_step *st);
/* Device time of the last launch, in milliseconds (blocks until it is done). */
int sjcs_step_time(sjcs_step *st, float *ms);
/* Destroy after the last launch has finished; q must outlive its steps. */
int sjcs_step_destroy(sjcs_step *st);

/* ---- serving (no counterpart in the reference, which runs one batch job) ---- */

typedef struct sjcs_server_opts {
    uint32_t slots;       /* requests on the GPU at once, one CUDA stream each (0 = 4, at most 64) */
    uint32_t pad_;
    uint64_t mem_budget;  /* device bytes the admitted requests may hold together
                             (0 = 80% of the device memory free when the server starts) */
    uint32_t reserved[4]; /* must be zero */
} sjcs_server_opts;

typedef struct sjcs_request_info {
    double queue_ms;      /* submission to admission (waiting for a slot or memory) */
    double service_ms;    /* admission to detected completion */
    double latency_ms;    /* submission to detected completion */
    int    status;        /* SJCS_OK or the request's error */
} sjcs_request_info;

typedef struct sjcs_server_info {
    uint64_t submitted, completed, queued;
    uint32_t inflight, max_inflight, slots, pad_;
    uint64_t budget_bytes, in_use_bytes, peak_bytes;
} sjcs_server_info;

/* Start a request loop over the given indexes (built in ctx, kept resident by
 * the caller until the server is destroyed; each request's counts are summed
 * over all of them, as the driver sums particle files).  A dispatcher thread
 * admits requests first come first served whenever a slot is free and the
 * request's device memory fits in the budget left by the running ones; each
 * admitted request runs on its own stream, so requests overlap on the GPU. */
int sjcs_server_create(sjcs_ctx *ctx, sjcs_index *const *indexes, int nindexes,
                       const sjcs_server_opts *opts, sjcs_server **out);
/* Queue one request: nhalos halo centres (host memory, `stride_bytes` apart),
 * a squared-radius table and query flags as for sjcs_query_create.  When it
 * completes, out_counts (host, uint32 [nhalos][nrads], pinned or not) holds
 * its counts.  Both buffers must stay valid until sjcs_server_wait returns.
 * Returns at once with a ticket; SJCS_ERR_NOMEM if the request alone needs
 * more device memory than the budget.  The counts are uint32: a request whose
 * counts could exceed 2^32 - 1 (the server's indexes hold more than 2^32 - 1
 * particles together, or 2^29 for periodic radius tables with R >= 499; see
 * sjcs_query_set_fold_limit) fails with SJCS_ERR_INVALID. */
int sjcs_server_submit(sjcs_server *srv, const float *halo_xyz, size_t stride_bytes, uint64_t nhalos,
                       const float *r2, int nrads, int flags, uint32_t *out_counts, uint64_t *ticket);
/* Block until the ticket's request has completed; info (may be NULL) gets its
 * timing.  Returns the request's status.  A ticket can be waited for once. */
int sjcs_server_wait(sjcs_server *srv, uint64_t ticket, sjcs_request_info *info);
int sjcs_server_stats(sjcs_server *srv, sjcs_server_info *out);
/* Finish every submitted request, then stop (before its indexes and ctx go). */
int sjcs_server_destroy(sjcs_server *srv);

/* ---- schedules and autotuning (no counterpart in the reference, whose
 * threads take halos in chunks of 100 from a shared counter,
 * src/astr_rcount/main.c:802-823) ---------------------------------------- */

/* Schedule used by later sjcs_query_count calls on q (default SJCS_SCHED_AUTO).
 * The schedule changes only how work is spread over warps, never the counts. */
int sjcs_query_set_schedule(sjcs_ctx *ctx, sjcs_query *q, const sjcs_schedule *sched);
int sjcs_query_get_schedule(const sjcs_query *q, sjcs_schedule *out);
/* Time every candidate schedule (static; queue with pieces of 2048, 8192,
 * 32768 and 131072 candidates and up to 64 warps per halo; queue with pieces
 * of 32768 and up to 256 warps per halo) on the full query against
 * idx, keep the fastest on q and remember it in the context for queries of
 * the same shape (index kind, particles and halos to the nearest power of
 * two, largest radius, shells, periodicity), where SJCS_SCHED_AUTO finds it.
 * The query's counts are left as they were.  Blocks; trial_ms[i] (up to
 * max_trials entries, may be NULL) receives each trial's kernel time in the
 * order above and *ntrials their number. */
int sjcs_autotune(sjcs_ctx *ctx, sjcs_query *q, const sjcs_index *idx, sjcs_schedule *chosen,
                  float *trial_ms, int max_trials, int *ntrials);

/* ---- one-shot, reference semantics --------------------------------------- */

/* counts[h*nrads + i] += number of particles of idx in shell i of halo h, for
 * the nhalos halos at halo_xyz (host, stride as above).  Synchronous.  This is
 * threadJoin's whole loop for one file (src/astr_rcount/main.c:795-826) with
 * the same argument meaning as MultiRangeCountContext. */
int sjcs_multi_range_count(sjcs_ctx *ctx, const sjcs_index *idx,
                           const float *halo_xyz, size_t stride_bytes, uint64_t nhalos,
                           const float *r2, int nrads, int flags, uint64_t *counts);

/* ---- allocation-free count for small inputs ------------------------------ */

/* Limits of sjcs_count_noalloc and the size of the scratch array every GPU
 * that loads this library holds until the process exits. */
#define SJCS_NOALLOC_MAX_PARTICLES  131072u   /* 2^17 */
#define SJCS_NOALLOC_MAX_HALOS      32768u    /* 2^15 */
#define SJCS_NOALLOC_MAX_CELLS      131072u   /* grid cells used for the index */
#define SJCS_NOALLOC_MAX_SHELLS     256
#define SJCS_NOALLOC_SCRATCH_BYTES  9734656u  /* about 9.3 MB */

/* No counterpart in the reference: it exists for callers that must not have
 * a library allocate device memory -- e.g. a host program whose framework has
 * already reserved the GPU's memory for its own caching allocator, or a
 * latency-critical loop that cannot absorb the synchronisation cudaMalloc
 * and cudaFree may imply.  It builds the grid index over n particles
 * (d_xyz, device, n*3 floats), counts the shells of nhalos halos
 * (d_halo_xyz, device, stride as sjcs_query_create) and ADDS the counts to
 * d_counts (device, uint32 [nhalos][nrads], caller's halo order), queued on
 * `stream` (a cudaStream_t; NULL = default stream).  It calls no cudaMalloc,
 * cudaFree or allocating library routine: all scratch lives in one
 * file-scope device array of SJCS_NOALLOC_SCRATCH_BYTES.  Sizes beyond the
 * limits above are rejected with SJCS_ERR_INVALID.  The first call on a
 * device (that device current) looks up the array's address with
 * cudaGetSymbolAddress; make that first call before any stream capture.
 * Under lazy module loading (the CUDA default since 12.2) that first call is
 * also when the driver creates the array on the device, so make it before a
 * framework reserves the device's memory (or set CUDA_MODULE_LOADING=EAGER).
 * All calls share the array, so calls that overlap on the GPU race: keep
 * them on one stream.  Counts equal those of sjcs_query_count; each call
 * adds at most n (8n for periodic tables with R >= 499) to an accumulator,
 * and keeping d_counts below 2^32 across calls is the caller's part. */
int sjcs_count_noalloc(const float *d_xyz, uint64_t n,
                       const float *d_halo_xyz, size_t stride_bytes, uint64_t nhalos,
                       const float *r2, int nrads, int flags,
                       uint32_t *d_counts, void *stream);

/* ---- radius schedule ----------------------------------------------------- */

/* r2[i] = (float)pow(2, log2(min) + i*(log2(max)-log2(min))/(n-1)) squared in
 * fp32, last entry (float)pow(2, log2(max)) squared -- Logspace
 * (include/support_functions.h:18-34) followed by r[i] *= r[i]
 * (src/astr_rcount/main.c:646-649).  min > max is swapped as the driver does
 * (main.c:531-533).  Host-only; needs no GPU. */
int sjcs_radius_table(double minrad, double maxrad, int nrads, float *r2);

#ifdef __cplusplus
}
#endif

#endif /* SJCS_H */
