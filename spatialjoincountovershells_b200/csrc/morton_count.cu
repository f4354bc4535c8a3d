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

template <int LOOK, int BIN, bool BIG>
__device__ __forceinline__ void count_image_m(const CountParams& p, const MortonParams& m, const RootRegs& rr,
                                              float cx, float cy, float cz, uint32_t* __restrict__ sink,
                                              const float* __restrict__ tab, const uint32_t* __restrict__ lut,
                                              uint2* __restrict__ pend, int lane) {
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
                run_rows<BIN, BIG>(p, im, r.x, r.y, sink, tab, lut, lane);
            }
        }
    }
    if (npend) {
        __syncwarp();
        const uint2 r = (uint32_t)lane < npend ? pend[lane] : make_uint2(0u, 0u);
        __syncwarp();
        run_rows<BIN, BIG>(p, im, r.x, r.y, sink, tab, lut, lane);
    }
}

template <int LOOK, int BIN, bool BIG>
__global__ void __launch_bounds__(MC_THREADS, 8) k_morton_count(CountParams p, MortonParams m) {
    extern __shared__ uint32_t smem[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    uint2* pend = reinterpret_cast<uint2*>(smem) + warp * kPend;
    float* r2s = reinterpret_cast<float*>(reinterpret_cast<uint2*>(smem) + MC_WARPS * kPend);
    uint32_t* luts = reinterpret_cast<uint32_t*>(r2s + p.pad);
    uint32_t* wcnt = luts + p.nlut + warp * p.nrads;
    if (!BIG) {
        for (int i = tid; i < p.pad; i += MC_THREADS) r2s[i] = p.r2[i];
        for (int i = tid; i < p.nlut; i += MC_THREADS) luts[i] = p.lut[i];
        for (int i = tid; i < MC_WARPS * p.nrads; i += MC_THREADS) luts[p.nlut + i] = 0u;
    }
    RootRegs rr{};
    if (LOOK == LOOK_MODEL) {
        rr.kmin = m.root->kmin;
        rr.kmax = m.root->kmax;
        rr.shift = m.root->shift;
        rr.n = m.root->n;
        rr.table_only = m.root->mismatches != 0ull;
    }
    __syncthreads();
    const float* tab = BIG ? p.r2 : r2s;
    const uint32_t* lut = BIG ? p.lut : luts;
    const uint64_t W = (uint64_t)gridDim.x * MC_WARPS;
    for (uint64_t hk = (uint64_t)blockIdx.x * MC_WARPS + warp; hk < p.nhalos; hk += W) {
        const float4 c = p.halos[hk];
        uint32_t* row = p.counts + (uint64_t)__float_as_uint(c.w) * (uint64_t)p.nrads;
        uint32_t* sink = BIG ? row : wcnt;
        count_image_m<LOOK, BIN, BIG>(p, m, rr, c.x, c.y, c.z, sink, tab, lut, pend, lane);
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
                                                  (S & 4u) ? sz : c.z, sink, tab, lut, pend, lane);
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

template <int LOOK>
int dispatch_bin(sjcs_ctx* ctx, int bin, bool big, const CountParams& p, const MortonParams& m, size_t smem,
                 cudaStream_t s) {
    switch (bin) {
        case BIN_LUT:
            return big ? launch_m<LOOK, BIN_LUT, true>(ctx, p, m, smem, s)
                       : launch_m<LOOK, BIN_LUT, false>(ctx, p, m, smem, s);
        case BIN_BSEARCH:
            return big ? launch_m<LOOK, BIN_BSEARCH, true>(ctx, p, m, smem, s)
                       : launch_m<LOOK, BIN_BSEARCH, false>(ctx, p, m, smem, s);
        default:
            return big ? launch_m<LOOK, BIN_FIRST_MATCH, true>(ctx, p, m, smem, s)
                       : launch_m<LOOK, BIN_FIRST_MATCH, false>(ctx, p, m, smem, s);
    }
}

}  // namespace

int launch_morton_count(sjcs_ctx* ctx, const sjcs_query* q, const sjcs_index* idx, cudaStream_t s) {
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
    return idx->kind == SJCS_INDEX_LEARNED ? dispatch_bin<LOOK_MODEL>(ctx, bin, big, p, m, smem, s)
                 : dispatch_bin<LOOK_TABLE>(ctx, bin, big, p, m, smem, s);
}

}  // namespace sjcs
