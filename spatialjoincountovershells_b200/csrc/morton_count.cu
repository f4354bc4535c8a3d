// Warp-cooperative periodic multi-shell count over a Morton index (plain
// Morton offset table or learned rank model).
//
// One warp owns one halo at a time.  For every periodic image the warp lists
// the level-L Morton cells of the query box (lane k takes cell k of the box),
// drops the cells that cannot hold a particle within R (conservative gap
// test on all three axes, the margins of the grid kernel), looks up each
// kept cell's slot range [rank(c), rank(c+1)) -- from the offset table, or
// from the learned model with its bounded exact correction -- and hands the
// non-empty ranges, 32 at a time, to the shared candidate loop (coalesced
// float4 loads, exact reference predicate, shell binning).  The arithmetic of
// the box test, the distance and the shell is the one of the grid kernel
// (count_common.cuh), so both index forms produce the reference's counts.
//
// Periodic images and their precedence follow MultiRangeCount.c:31-71; the
// non-periodic half-width quirk (MultiRangeCount.c:81) comes in through
// CountParams::half.
#include <cmath>

#include "count_common.cuh"
#include "morton.cuh"
#include "queue_common.cuh"
#include "sjcs_internal.cuh"

namespace sjcs {
namespace {

using namespace count;

constexpr int MC_WARPS = 4;
constexpr int MC_THREADS = MC_WARPS * 32;
constexpr int kMaxSmemTable = 8192;
constexpr int kMaxSmemRads = 1024;
constexpr int kPend = 64;  // pending slot ranges per warp

enum Lookup { LOOK_TABLE = 0, LOOK_MODEL = 1 };

struct MortonParams {
    const uint32_t* __restrict__ table;  // 8^L + 1 offsets
    const LearnedLeaf* __restrict__ leaves;
    const LearnedRoot* __restrict__ root;
    const uint32_t* __restrict__ wpref;  // &pts[0].w (stride 4 words)
    int sh;         // 21 - L: morton_q(v) >> sh is the level-L cell
    int key_shift;  // 63 - 3L: cell code -> first key of the cell
    float h;        // 1000 / 2^L
    int G;          // 2^L
};

struct RootRegs {
    unsigned long long kmin, kmax;
    uint32_t shift, n;
    bool table_only;  // the judge found a mismatch: the table answers
};

__device__ __forceinline__ int mcell_lo(const MortonParams& m, float v) { return (int)(morton_q(v) >> m.sh); }
__device__ __forceinline__ int mcell_hi(const MortonParams& m, float v) {
    // a NaN upper bound passes every particle on that side: open to the edge
    return (v != v) ? m.G - 1 : (int)(morton_q(v) >> m.sh);
}

// The candidates of up to 32 slot ranges: all of them, or piece `part` of
// `nparts` (heavy halos shared by several warps of the queue schedule).
template <int BIN, bool BIG>
__device__ __forceinline__ void run_ranges(const CountParams& p, const Image& im, uint32_t s0, uint32_t s1,
                                           uint32_t* __restrict__ sink, const float* __restrict__ tab,
                                           const uint32_t* __restrict__ lut, int lane, uint32_t part, uint32_t nparts) {
    if (nparts > 1) run_rows_part<BIN, BIG>(p, im, s0, s1, sink, tab, lut, lane, part, nparts);
    else run_rows<BIN, BIG>(p, im, s0, s1, sink, tab, lut, lane);
}

template <int LOOK, int BIN, bool BIG>
__device__ __forceinline__ void count_image_m(const CountParams& p, const MortonParams& m, const RootRegs& rr,
                                              float cx, float cy, float cz, uint32_t* __restrict__ sink,
                                              const float* __restrict__ tab, const uint32_t* __restrict__ lut,
                                              uint2* __restrict__ pend, int lane, uint32_t part = 0,
                                              uint32_t nparts = 1) {
    Image im;
    im.cx = cx;
    im.cy = cy;
    im.cz = cz;
    im.lox = __fsub_rn(cx, p.half);
    im.hix = __fadd_rn(cx, p.half);
    im.loy = __fsub_rn(cy, p.half);
    im.hiy = __fadd_rn(cy, p.half);
    im.loz = __fsub_rn(cz, p.half);
    im.hiz = __fadd_rn(cz, p.half);
    const int x0 = mcell_lo(m, im.lox), x1 = mcell_hi(m, im.hix);
    const int y0 = mcell_lo(m, im.loy), y1 = mcell_hi(m, im.hiy);
    const int z0 = mcell_lo(m, im.loz), z1 = mcell_hi(m, im.hiz);
    const uint32_t nx = (uint32_t)(x1 - x0 + 1), ny = (uint32_t)(y1 - y0 + 1), nz = (uint32_t)(z1 - z0 + 1);
    const uint32_t total = nx * ny * nz;  // <= 2^30 (L <= 10)
    const uint32_t lt = (1u << lane) - 1u;
    uint32_t npend = 0;
    // 64 box cells per round, two per lane: the four lookups of a lane (both
    // ends of both cells) go out together
    for (uint32_t cb = 0; cb < total; cb += 64u) {
        uint32_t code[2];
        bool keep[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const uint32_t k = cb + 32u * (uint32_t)u + (uint32_t)lane;
            keep[u] = k < total;
            const uint32_t t = k / nx;
            const int xx = x0 + (int)(k - t * nx), yy = y0 + (int)(t % ny), zz = z0 + (int)(t / ny);
            if (keep[u] && p.prune) {
                const float gx = cell_gap(cx, xx, m.h, m.G), gy = cell_gap(cy, yy, m.h, m.G),
                            gz = cell_gap(cz, zz, m.h, m.G);
                const float rem = __fadd_rn(__fsub_rn(__fsub_rn(__fsub_rn(p.r2p, __fmul_rn(gx, gx)), __fmul_rn(gy, gy)),
                                                      __fmul_rn(gz, gz)),
                                            p.r2slack);
                keep[u] = rem >= 0.0f;  // no particle of this cell can be within R otherwise
            }
            code[u] = keep[u] ? morton_cell((uint32_t)xx, (uint32_t)yy, (uint32_t)zz) : 0u;
        }
        uint32_t s[4];
        if (LOOK == LOOK_TABLE || rr.table_only) {
#pragma unroll
            for (int j = 0; j < 4; ++j) s[j] = keep[j >> 1] ? __ldg(m.table + code[j >> 1] + (j & 1)) : 0u;
        } else {
            LearnedRoot rt;
            rt.kmin = rr.kmin;
            rt.kmax = rr.kmax;
            rt.shift = rr.shift;
            rt.n = rr.n;
            const uint64_t qk[4] = {(uint64_t)code[0] << m.key_shift, (uint64_t)(code[0] + 1u) << m.key_shift,
                                    (uint64_t)code[1] << m.key_shift, (uint64_t)(code[1] + 1u) << m.key_shift};
            const bool act[4] = {keep[0], keep[0], keep[1], keep[1]};
            learned_rank_n<4>(rt, m.leaves, m.wpref, qk, act, s);
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const uint32_t s0 = s[2 * u], s1 = s[2 * u + 1];
            const bool ne = keep[u] && s1 > s0;
            const uint32_t bal = __ballot_sync(0xffffffffu, ne);
            if (ne) pend[npend + __popc(bal & lt)] = make_uint2(s0, s1);
            npend += __popc(bal);
            if (npend >= 32u) {
                __syncwarp();
                const uint2 r = pend[lane];
                __syncwarp();
                if ((uint32_t)lane < npend - 32u) pend[lane] = pend[32 + lane];
                __syncwarp();
                npend -= 32u;
                run_ranges<BIN, BIG>(p, im, r.x, r.y, sink, tab, lut, lane, part, nparts);
            }
        }
    }
    if (npend) {
        __syncwarp();
        const uint2 r = (uint32_t)lane < npend ? pend[lane] : make_uint2(0u, 0u);
        __syncwarp();
        run_ranges<BIN, BIG>(p, im, r.x, r.y, sink, tab, lut, lane, part, nparts);
    }
}

// One halo: every periodic image (MultiRangeCount.c:31-71), then the warp's
// counters flushed into the halo's row.
template <int LOOK, int BIN, bool BIG>
__device__ __forceinline__ void count_halo_m(const CountParams& p, const MortonParams& m, const RootRegs& rr,
                                             const float4 c, uint32_t* __restrict__ wcnt,
                                             const float* __restrict__ tab, const uint32_t* __restrict__ lut,
                                             uint2* __restrict__ pend, int lane, uint32_t part, uint32_t nparts) {
    uint32_t* row = p.counts + (uint64_t)__float_as_uint(c.w) * (uint64_t)p.nrads;
    uint32_t* sink = BIG ? row : wcnt;
    count_image_m<LOOK, BIN, BIG>(p, m, rr, c.x, c.y, c.z, sink, tab, lut, pend, lane, part, nparts);
    if (p.periodic) {
        const float lox = __fsub_rn(c.x, p.half), hix = __fadd_rn(c.x, p.half);
        const float loy = __fsub_rn(c.y, p.half), hiy = __fadd_rn(c.y, p.half);
        const float loz = __fsub_rn(c.z, p.half), hiz = __fadd_rn(c.z, p.half);
        const unsigned F = ((lox < kBoxLow) | (hix > kBoxUpp) ? 1u : 0u) |
                           ((loy < kBoxLow) | (hiy > kBoxUpp) ? 2u : 0u) |
                           ((loz < kBoxLow) | (hiz > kBoxUpp) ? 4u : 0u);
        if (F) {
            // min_oob takes precedence over max_oob on an axis (MultiRangeCount.c:38-43)
            const float sx = (lox < kBoxLow) ? __fadd_rn(c.x, kBoxUpp) : __fsub_rn(c.x, kBoxUpp);
            const float sy = (loy < kBoxLow) ? __fadd_rn(c.y, kBoxUpp) : __fsub_rn(c.y, kBoxUpp);
            const float sz = (loz < kBoxLow) ? __fadd_rn(c.z, kBoxUpp) : __fsub_rn(c.z, kBoxUpp);
            for (unsigned S = F; S != 0; S = (S - 1u) & F)
                count_image_m<LOOK, BIN, BIG>(p, m, rr, (S & 1u) ? sx : c.x, (S & 2u) ? sy : c.y,
                                              (S & 4u) ? sz : c.z, sink, tab, lut, pend, lane, part, nparts);
        }
    }
    if (!BIG) {
        __syncwarp();
        for (int sh = lane; sh < p.nrads; sh += 32) {
            const uint32_t v = wcnt[sh];
            if (v) {
                wcnt[sh] = 0u;
                atomicAdd(row + sh, v);  // result unused: compiles to a reduction
            }
        }
        __syncwarp();
    }
}

// Shared-memory set-up common to both schedules and the root model in registers.
struct MView {
    uint2* pend;
    const float* tab;
    const uint32_t* lut;
    uint32_t* wcnt;
    RootRegs rr;
};

template <int LOOK, bool BIG>
__device__ __forceinline__ MView setup_m(const CountParams& p, const MortonParams& m, uint32_t* smem, int tid,
                                         int warp) {
    MView v;
    v.pend = reinterpret_cast<uint2*>(smem) + warp * kPend;
    float* r2s = reinterpret_cast<float*>(reinterpret_cast<uint2*>(smem) + MC_WARPS * kPend);
    uint32_t* luts = reinterpret_cast<uint32_t*>(r2s + p.pad);
    v.wcnt = luts + p.nlut + warp * p.nrads;
    if (!BIG) {
        for (int i = tid; i < p.pad; i += MC_THREADS) r2s[i] = p.r2[i];
        for (int i = tid; i < p.nlut; i += MC_THREADS) luts[i] = p.lut[i];
        for (int i = tid; i < MC_WARPS * p.nrads; i += MC_THREADS) luts[p.nlut + i] = 0u;
    }
    v.rr = RootRegs{};
    if (LOOK == LOOK_MODEL) {
        v.rr.kmin = m.root->kmin;
        v.rr.kmax = m.root->kmax;
        v.rr.shift = m.root->shift;
        v.rr.n = m.root->n;
        v.rr.table_only = m.root->mismatches != 0ull;
    }
    v.tab = BIG ? p.r2 : r2s;
    v.lut = BIG ? p.lut : luts;
    return v;
}

// Static schedule: warp gw of W takes halos gw, gw + W, ... (the resident
// warps work on one window of the Morton order and share particle lines).
template <int LOOK, int BIN, bool BIG>
__global__ void __launch_bounds__(MC_THREADS, 8) k_morton_count(CountParams p, MortonParams m) {
    extern __shared__ uint32_t smem[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const MView v = setup_m<LOOK, BIG>(p, m, smem, tid, warp);
    __syncthreads();
    const uint64_t W = (uint64_t)gridDim.x * MC_WARPS;
    for (uint64_t hk = (uint64_t)blockIdx.x * MC_WARPS + warp; hk < p.nhalos; hk += W)
        count_halo_m<LOOK, BIN, BIG>(p, m, v.rr, p.halos[hk], v.wcnt, v.tab, v.lut, v.pend, lane, 0, 1);
}

// Rank of a cell boundary at any level <= 10 (queue estimates): the table
// covers the index's level L, so a coarser cell c' starts at table[c' * 8^(L-l)].
template <int LOOK>
__device__ __forceinline__ uint32_t rank_at(const MortonParams& m, const RootRegs& rr, uint32_t code, int up) {
    if (LOOK == LOOK_TABLE || rr.table_only) return __ldg(m.table + ((uint64_t)code << (3 * up)));
    LearnedRoot rt;
    rt.kmin = rr.kmin;
    rt.kmax = rr.kmax;
    rt.shift = rr.shift;
    rt.n = rr.n;
    return learned_rank(rt, m.leaves, m.wpref, (unsigned long long)code << (m.key_shift + 3 * up));
}

// Queue estimate (lane per halo): particles in the halo's box of cells one
// level coarser than the index's (x 2^k for k periodic axes), from the same
// ranks the count uses (offset table or learned model).
template <int LOOK>
__global__ void k_estimate_m(CountParams p, MortonParams m, uint32_t* __restrict__ key, uint32_t* __restrict__ hist) {
    __shared__ uint32_t sh[kBuckets];
    for (int i = threadIdx.x; i < kBuckets; i += blockDim.x) sh[i] = 0;
    RootRegs rr{};
    if (LOOK == LOOK_MODEL) {
        rr.kmin = m.root->kmin;
        rr.kmax = m.root->kmax;
        rr.shift = m.root->shift;
        rr.n = m.root->n;
        rr.table_only = m.root->mismatches != 0ull;
    }
    __syncthreads();
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < p.nhalos) {
        const float4 c = p.halos[i];
        const int up = m.G > 1 ? 1 : 0;  // one level coarser
        const int sh2 = m.sh + up, G2 = m.G >> up;
        const float lo[3] = {__fsub_rn(c.x, p.half), __fsub_rn(c.y, p.half), __fsub_rn(c.z, p.half)};
        const float hi[3] = {__fadd_rn(c.x, p.half), __fadd_rn(c.y, p.half), __fadd_rn(c.z, p.half)};
        int a0[3], a1[3];
        uint64_t ncell = 1;
        for (int a = 0; a < 3; ++a) {
            a0[a] = (int)(morton_q(lo[a]) >> sh2);
            a1[a] = (hi[a] != hi[a]) ? G2 - 1 : (int)(morton_q(hi[a]) >> sh2);
            ncell *= (uint64_t)(a1[a] - a0[a] + 1);
        }
        uint64_t e = 0;
        if (ncell > 64) {
            e = 0x40000000ull;  // huge box: certainly heavy
        } else {
            for (int z = a0[2]; z <= a1[2]; ++z)
                for (int y = a0[1]; y <= a1[1]; ++y)
                    for (int x = a0[0]; x <= a1[0]; ++x) {
                        const uint32_t code = morton_cell((uint32_t)x, (uint32_t)y, (uint32_t)z);
                        e += rank_at<LOOK>(m, rr, code + 1u, up) - rank_at<LOOK>(m, rr, code, up);
                    }
            if (p.periodic) {
                const int k = ((lo[0] < kBoxLow) | (hi[0] > kBoxUpp)) + ((lo[1] < kBoxLow) | (hi[1] > kBoxUpp)) +
                              ((lo[2] < kBoxLow) | (hi[2] > kBoxUpp));
                e <<= k;
            }
        }
        const uint32_t ev = e < 0x40000000ull ? (uint32_t)e : 0x40000000u;
        const uint32_t k = 255u - est_bucket(ev);
        key[i] = k;
        atomicAdd(&sh[k], 1u);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < kBuckets; k += blockDim.x)
        if (sh[k]) atomicAdd(hist + k, sh[k]);
}

// Queue schedule: persistent warps claim items (batches of light halos, or
// pieces of heavy ones) largest first.
template <int LOOK, int BIN, bool BIG>
__global__ void __launch_bounds__(MC_THREADS, 8) k_morton_count_queue(CountParams p, MortonParams m, QueueParams q) {
    extern __shared__ uint32_t smem[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const MView v = setup_m<LOOK, BIG>(p, m, smem, tid, warp);
    __syncthreads();
    const uint32_t nitems = q.ctl[1];
    int bk = 0;
    for (;;) {
        BucketPlan bp;
        uint32_t r;
        if (!claim_item(q, nitems, lane, &bk, &bp, &r)) break;
        if (bp.per == 0) {
            const uint32_t pos = bp.start + r / bp.pieces, part = r % bp.pieces;
            count_halo_m<LOOK, BIN, BIG>(p, m, v.rr, p.halos[q.ord[pos]], v.wcnt, v.tab, v.lut, v.pend, lane, part,
                                         bp.pieces);
        } else {
            const uint32_t first = r * bp.per;
            const uint32_t nb = min(bp.per, bp.count - first);
            for (uint32_t k = 0; k < nb; ++k)
                count_halo_m<LOOK, BIN, BIG>(p, m, v.rr, p.halos[q.ord[bp.start + first + k]], v.wcnt, v.tab, v.lut,
                                             v.pend, lane, 0, 1);
        }
    }
}

template <int LOOK, int BIN, bool BIG>
int launch_m(sjcs_ctx* ctx, const CountParams& p, const MortonParams& m, size_t smem, cudaStream_t s) {
    auto kern = k_morton_count<LOOK, BIN, BIG>;
    if (smem > 48 * 1024)
        SJCS_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    SJCS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, MC_THREADS, smem));
    if (per_sm < 1) per_sm = 1;
    const uint64_t want = (p.nhalos + MC_WARPS - 1) / MC_WARPS;
    const uint64_t cap = (uint64_t)ctx->num_sms * (uint64_t)per_sm;
    kern<<<(unsigned)(want < cap ? want : cap), MC_THREADS, smem, s>>>(p, m);
    SJCS_LAUNCH_CHECK();
    return SJCS_OK;
}

template <int LOOK, int BIN, bool BIG>
int launch_mq(sjcs_ctx* ctx, const CountParams& p, const MortonParams& m, const Schedule& sc, size_t smem,
              cudaStream_t s) {
    const uint64_t n = p.nhalos;
    if (n * (uint64_t)sc.max_pieces >= (1ull << 32))
        return fail(SJCS_ERR_INVALID, "queue schedule: nhalos * max_pieces must stay below 2^32");
    const uint32_t ntiles = (uint32_t)((n + RS_TILE - 1) / RS_TILE);
    StreamScratch scr(s);  // freed (stream-ordered) after the kernels below
    uint32_t *key, *ord, *ctl, *hist, *rhist;
    BucketPlan* plan;
    SJCS_CUDA_TRY(scr.alloc(&key, n * sizeof(uint32_t)));
    SJCS_CUDA_TRY(scr.alloc(&ord, n * sizeof(uint32_t)));
    SJCS_CUDA_TRY(scr.alloc(&ctl, 4 * sizeof(uint32_t)));
    SJCS_CUDA_TRY(scr.alloc(&hist, kBuckets * sizeof(uint32_t)));
    SJCS_CUDA_TRY(scr.alloc(&plan, kBuckets * sizeof(BucketPlan)));
    SJCS_CUDA_TRY(scr.alloc(&rhist, (uint64_t)RS_BINS * ntiles * sizeof(uint32_t)));
    SJCS_CUDA_TRY(cudaMemsetAsync(hist, 0, kBuckets * sizeof(uint32_t), s));
    k_estimate_m<LOOK><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(p, m, key, hist);
    SJCS_LAUNCH_CHECK();
    int rc = order_and_plan(n, key, hist, sc, ord, plan, ctl, rhist, s);
    if (rc) return rc;
    auto kern = k_morton_count_queue<LOOK, BIN, BIG>;
    if (smem > 48 * 1024)
        SJCS_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    SJCS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, MC_THREADS, smem));
    if (per_sm < 1) per_sm = 1;
    kern<<<(unsigned)(ctx->num_sms * per_sm), MC_THREADS, smem, s>>>(p, m, QueueParams{ord, plan, ctl});
    SJCS_LAUNCH_CHECK();
    return SJCS_OK;
}

template <int LOOK, int BIN, bool BIG>
int launch_sched(sjcs_ctx* ctx, const CountParams& p, const MortonParams& m, const Schedule* sc, size_t smem,
                 cudaStream_t s) {
    if (sc && sc->mode == SJCS_SCHED_QUEUE) return launch_mq<LOOK, BIN, BIG>(ctx, p, m, *sc, smem, s);
    return launch_m<LOOK, BIN, BIG>(ctx, p, m, smem, s);
}

template <int LOOK>
int dispatch_bin(sjcs_ctx* ctx, int bin, bool big, const CountParams& p, const MortonParams& m, size_t smem,
                 cudaStream_t s, const Schedule* sc) {
    switch (bin) {
        case BIN_LUT:
            return big ? launch_sched<LOOK, BIN_LUT, true>(ctx, p, m, sc, smem, s)
                       : launch_sched<LOOK, BIN_LUT, false>(ctx, p, m, sc, smem, s);
        case BIN_BSEARCH:
            return big ? launch_sched<LOOK, BIN_BSEARCH, true>(ctx, p, m, sc, smem, s)
                       : launch_sched<LOOK, BIN_BSEARCH, false>(ctx, p, m, sc, smem, s);
        default:
            return big ? launch_sched<LOOK, BIN_FIRST_MATCH, true>(ctx, p, m, sc, smem, s)
                       : launch_sched<LOOK, BIN_FIRST_MATCH, false>(ctx, p, m, sc, smem, s);
    }
}

}  // namespace

int launch_morton_count(sjcs_ctx* ctx, const sjcs_query* q, const sjcs_index* idx, cudaStream_t s,
                        const Schedule* sc) {
    if (q->nhalos == 0 || idx->n == 0) return SJCS_OK;
    CountParams p{};
    p.pts = idx->pts;
    p.halos = q->halos;
    p.nhalos = q->nhalos;
    p.r2 = q->d_r2;
    p.lut = q->d_lut;
    p.nrads = q->nrads;
    p.pad = q->pad;
    p.nlut = q->nlut;
    p.lut_k0 = q->lut_k0;
    p.lut_shift = q->lut_shift;
    p.half = q->half;
    p.r2max = q->r2max;
    p.r2p = q->r2max * (1.0f + 1e-5f);
    p.r2slack = q->r2max * 1e-5f;
    p.periodic = (q->flags & SJCS_QUERY_PERIODIC) ? 1 : 0;
    p.prune = q->monotone && std::isfinite(q->r2max) ? 1 : 0;
    p.counts = q->counts;
    MortonParams m{};
    m.table = idx->cell_start;
    m.leaves = idx->leaves;
    m.root = idx->root;
    m.wpref = reinterpret_cast<const uint32_t*>(idx->pts) + 3;
    m.sh = kMortonBits - idx->level;
    m.key_shift = 63 - 3 * idx->level;
    m.G = 1 << idx->level;
    m.h = 1000.0f / (float)m.G;
    const int bin = !q->monotone ? BIN_FIRST_MATCH : (q->nlut > 0 ? BIN_LUT : BIN_BSEARCH);
    const bool big = q->pad > kMaxSmemTable || q->nrads > kMaxSmemRads;
    const size_t smem = MC_WARPS * kPend * sizeof(uint2) +
                        (big ? 0 : (size_t)(q->pad + q->nlut + MC_WARPS * q->nrads) * sizeof(uint32_t));
    // Learned kind: model lookups, unless the judge recorded a mismatch (the
    // kernel reads the record and then answers from the table).
    return idx->kind == SJCS_INDEX_LEARNED ? dispatch_bin<LOOK_MODEL>(ctx, bin, big, p, m, smem, s, sc)
                                           : dispatch_bin<LOOK_TABLE>(ctx, bin, big, p, m, smem, s, sc);
}

}  // namespace sjcs
