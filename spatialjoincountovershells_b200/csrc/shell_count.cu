// Warp-cooperative periodic multi-shell count (plain grid index).
//
// One warp owns one halo at a time.  For every periodic image of the halo the
// warp turns the query box into at most a few dozen rows of cells (one row =
// one contiguous slot range of the sorted particles), flattens the rows into
// a single candidate sequence and lets lane l test candidates l, l+32, ...
// so every particle load is coalesced.  Accepted candidates are binned with a
// branch-free search of the squared-radius table in shared memory and counted
// in per-warp shared-memory counters; the warp adds its counters to the
// halo's row once per halo.
//
// Arithmetic follows the reference exactly (fp32, round-to-nearest, no FMA,
// no flush-to-zero):
//   R     = (float)sqrt((double)r2[n-1])               MultiRangeCount.c:19 (host side)
//   box   lo = c - R, hi = c + R                        setQueryMbr, Mbr.c:207-239
//   test  !(p < lo) && !(hi < p) on x, y, z             checkOverlapMbr, Mbr.c:167-205
//   dist  (dx*dx + dy*dy) + dz*dz, d = p - c            CalcDistance, Distance.h:5-25 (_mm_dp_ps 0x77)
//   shell first i with dist < r2[i]                     MultiRangeCountRecursive, MultiRangeCount.c:103-113
//   images: flags from the un-shifted box, lo < 0 -> c += 1000, else hi > 1000
//           -> c -= 1000, every non-empty subset of the flagged axes
//                                                       MultiRangeCount.c:31-71, Mbr.c:284-313
// For a non-decreasing, NaN-free table "first i with dist < r2[i]" equals
// #{i : r2[i] <= dist} and a particle is counted iff dist < r2[n-1]; other
// tables use the literal first-match scan.
#include "sjcs_internal.cuh"

namespace sjcs {
namespace {

constexpr int CT_WARPS = 8;
constexpr int CT_THREADS = CT_WARPS * 32;
constexpr int kMaxSmemTable = 8192;  // r2 entries held in shared memory
constexpr int kMaxSmemRads = 1024;   // per-warp shared counters up to this many shells

struct CountParams {
    const float* __restrict__ xs;
    const float* __restrict__ ys;
    const float* __restrict__ zs;
    const uint32_t* __restrict__ cs;
    GridGeom g;
    const float4* __restrict__ halos;
    uint64_t nhalos;
    const float* __restrict__ r2;  // [pad], +inf past nrads
    int nrads;
    int pad;
    float half;
    float r2max;
    int periodic;
    uint32_t* __restrict__ counts;
};

// BIG: table too large for shared memory -> table read from global memory and
// counts added with global atomics straight into the halo's row.
template <bool MONO, bool BIG>
__device__ __forceinline__ void count_image(const CountParams& p, float cx, float cy, float cz,
                                            uint32_t* __restrict__ sink, const float* __restrict__ tab,
                                            int lane) {
    const float lox = __fsub_rn(cx, p.half), hix = __fadd_rn(cx, p.half);
    const float loy = __fsub_rn(cy, p.half), hiy = __fadd_rn(cy, p.half);
    const float loz = __fsub_rn(cz, p.half), hiz = __fadd_rn(cz, p.half);
    // A NaN bound passes every particle on that side of the box test, so it
    // must open the cell range to the grid edge (cell_of maps NaN to cell 0,
    // which is right for a lower bound only).
    const int x0 = cell_of(lox, p.g.inv_h[0], p.g.G[0]);
    const int x1 = (hix != hix) ? p.g.G[0] - 1 : cell_of(hix, p.g.inv_h[0], p.g.G[0]);
    const int y0 = cell_of(loy, p.g.inv_h[1], p.g.G[1]);
    const int y1 = (hiy != hiy) ? p.g.G[1] - 1 : cell_of(hiy, p.g.inv_h[1], p.g.G[1]);
    const int z0 = cell_of(loz, p.g.inv_h[2], p.g.G[2]);
    const int z1 = (hiz != hiz) ? p.g.G[2] - 1 : cell_of(hiz, p.g.inv_h[2], p.g.G[2]);
    const int ny = y1 - y0 + 1;
    const int nrows = ny * (z1 - z0 + 1);

    for (int rb = 0; rb < nrows; rb += 32) {
        const int r = rb + lane;
        uint32_t start = 0, len = 0;
        if (r < nrows) {
            const int q = r / ny;
            const uint64_t rowcell =
                ((uint64_t)(z0 + q) * (uint64_t)p.g.G[1] + (uint64_t)(y0 + r - q * ny)) * (uint64_t)p.g.G[0];
            start = __ldg(p.cs + rowcell + x0);
            len = __ldg(p.cs + rowcell + x1 + 1) - start;
        }
        uint32_t incl = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        const uint32_t off = start - (incl - len);  // slot = t + off for t inside this row (mod 2^32)

        for (uint32_t wb = 0; wb < total; wb += 32) {
            const uint32_t t = wb + (uint32_t)lane;
            // row of t = #{rows j : incl_j <= t} (empty rows are skipped naturally)
            int rr = 0;
#pragma unroll
            for (int b = 16; b >= 1; b >>= 1) {
                const uint32_t v = __shfl_sync(0xffffffffu, incl, rr + b - 1);
                rr += (v <= t) ? b : 0;
            }
            const uint32_t o = __shfl_sync(0xffffffffu, off, rr);
            if (t < total) {
                const uint32_t k = t + o;
                const float px = __ldg(p.xs + k), py = __ldg(p.ys + k), pz = __ldg(p.zs + k);
                const bool inb = !(px < lox) & !(hix < px) & !(py < loy) & !(hiy < py) & !(pz < loz) &
                                 !(hiz < pz);
                const float dx = __fsub_rn(px, cx), dy = __fsub_rn(py, cy), dz = __fsub_rn(pz, cz);
                const float dist =
                    __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
                if (MONO) {
                    if (inb && dist < p.r2max) {
                        int s = 0;
                        for (int step = p.pad >> 1; step > 0; step >>= 1)
                            s += (tab[s + step - 1] <= dist) ? step : 0;
                        atomicAdd(sink + s, 1u);
                    }
                } else if (inb) {
                    for (int i = 0; i < p.nrads; ++i) {
                        if (dist < tab[i]) {
                            atomicAdd(sink + i, 1u);
                            break;
                        }
                    }
                }
            }
        }
    }
}

template <bool MONO, bool BIG>
__global__ void __launch_bounds__(CT_THREADS) k_shell_count(CountParams p) {
    extern __shared__ uint32_t smem[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    float* r2s = reinterpret_cast<float*>(smem);
    uint32_t* wcnt = smem + p.pad + warp * p.nrads;
    if (!BIG) {
        for (int i = tid; i < p.pad; i += CT_THREADS) r2s[i] = p.r2[i];
        for (int i = tid; i < CT_WARPS * p.nrads; i += CT_THREADS) smem[p.pad + i] = 0u;
        __syncthreads();
    }
    const float* tab = BIG ? p.r2 : r2s;
    const uint64_t stride = (uint64_t)gridDim.x * CT_WARPS;
    for (uint64_t h = (uint64_t)blockIdx.x * CT_WARPS + warp; h < p.nhalos; h += stride) {
        const float4 c = p.halos[h];
        uint32_t* row = p.counts + (uint64_t)__float_as_uint(c.w) * (uint64_t)p.nrads;
        uint32_t* sink = BIG ? row : wcnt;
        if (p.periodic) {
            const float lox = __fsub_rn(c.x, p.half), hix = __fadd_rn(c.x, p.half);
            const float loy = __fsub_rn(c.y, p.half), hiy = __fadd_rn(c.y, p.half);
            const float loz = __fsub_rn(c.z, p.half), hiz = __fadd_rn(c.z, p.half);
            // min_oob takes precedence over max_oob on an axis (MultiRangeCount.c:38-43)
            const float sx = (lox < kBoxLow) ? __fadd_rn(c.x, kBoxUpp) : __fsub_rn(c.x, kBoxUpp);
            const float sy = (loy < kBoxLow) ? __fadd_rn(c.y, kBoxUpp) : __fsub_rn(c.y, kBoxUpp);
            const float sz = (loz < kBoxLow) ? __fadd_rn(c.z, kBoxUpp) : __fsub_rn(c.z, kBoxUpp);
            const unsigned F = ((lox < kBoxLow) | (hix > kBoxUpp) ? 1u : 0u) |
                               ((loy < kBoxLow) | (hiy > kBoxUpp) ? 2u : 0u) |
                               ((loz < kBoxLow) | (hiz > kBoxUpp) ? 4u : 0u);
            // every subset S of F, the empty set (the un-shifted search) included
            unsigned S = F;
            for (;;) {
                count_image<MONO, BIG>(p, (S & 1u) ? sx : c.x, (S & 2u) ? sy : c.y, (S & 4u) ? sz : c.z,
                                       sink, tab, lane);
                if (S == 0) break;
                S = (S - 1u) & F;
            }
        } else {
            count_image<MONO, BIG>(p, c.x, c.y, c.z, sink, tab, lane);
        }
        if (!BIG) {
            __syncwarp();
            for (int s = lane; s < p.nrads; s += 32) {
                const uint32_t v = wcnt[s];
                if (v) {
                    wcnt[s] = 0u;
                    row[s] += v;
                }
            }
            __syncwarp();
        }
    }
}

template <bool MONO, bool BIG>
int launch_variant(sjcs_ctx* ctx, const CountParams& p, size_t smem, cudaStream_t s) {
    auto kern = k_shell_count<MONO, BIG>;
    if (smem > 48 * 1024) SJCS_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    SJCS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, CT_THREADS, smem));
    if (per_sm < 1) per_sm = 1;
    const uint64_t want = (p.nhalos + CT_WARPS - 1) / CT_WARPS;
    const uint64_t cap = (uint64_t)ctx->num_sms * (uint64_t)per_sm;
    const unsigned grid = (unsigned)(want < cap ? want : cap);
    kern<<<grid, CT_THREADS, smem, s>>>(p);
    SJCS_LAUNCH_CHECK();
    return SJCS_OK;
}

}  // namespace

int launch_shell_count(sjcs_ctx* ctx, const sjcs_query* q, const sjcs_index* idx, cudaStream_t s) {
    if (q->nhalos == 0 || idx->n == 0) return SJCS_OK;
    CountParams p;
    p.xs = idx->xs;
    p.ys = idx->ys;
    p.zs = idx->zs;
    p.cs = idx->cell_start;
    p.g = idx->geom;
    p.halos = q->halos;
    p.nhalos = q->nhalos;
    p.r2 = q->d_r2;
    p.nrads = q->nrads;
    p.pad = q->pad;
    p.half = q->half;
    p.r2max = q->r2max;
    p.periodic = (q->flags & SJCS_QUERY_PERIODIC) ? 1 : 0;
    p.counts = q->counts;
    const bool big = q->pad > kMaxSmemTable || q->nrads > kMaxSmemRads;
    const size_t smem = big ? 0 : (size_t)(q->pad + CT_WARPS * q->nrads) * sizeof(uint32_t);
    if (q->monotone)
        return big ? launch_variant<true, true>(ctx, p, smem, s) : launch_variant<true, false>(ctx, p, smem, s);
    return big ? launch_variant<false, true>(ctx, p, smem, s) : launch_variant<false, false>(ctx, p, smem, s);
}

}  // namespace sjcs
