// Warp-cooperative periodic multi-shell count (plain grid index).
//
// One warp owns one halo at a time.  For every periodic image of the halo the
// warp turns the query box into rows of cells (one row = one contiguous slot
// range of the sorted particles), clips each row's x-extent to the sphere of
// radius R with conservative floating-point margins (a row whose cells cannot
// hold a particle within R is skipped), flattens the rows into one candidate
// sequence and lets lane l test candidates l, l+32, ... so every particle load
// is a coalesced 128-bit load.  Accepted candidates are binned through a
// lookup table on the float bit pattern of the squared distance (one compare
// refines the slot) and counted in per-warp shared-memory counters; the warp
// adds its counters to the halo's row once per halo with fire-and-forget
// reductions.
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
// tables use the literal first-match scan (and no sphere clipping).
//
// Why the sphere clipping never drops a counted particle: a counted particle
// has fp32 dist < r2max, and fp32 rounding of the 3 differences and 5
// products/sums lowers the exact squared distance by at most a factor
// (1 - 2^-24)^5, so its exact squared distance is < r2max * (1 + 1e-5) = r2p.
// Its y lies inside its cell's y-extent, so (py - cy)^2 >= gy^2 where gy is a
// lower bound of the halo's distance to that extent (cell edges widened by
// 1e-3 + 2e-6*|edge|, far above the rounding of k*h and of the cell function);
// likewise z.  Hence (px - cx)^2 < r2p - gy^2 - gz^2, and the fp32 evaluation
// of that bound is off by at most 4 ulps of r2p < 1e-5*r2p, which is added
// back before the square root; the x cell range then uses cx -+ (xr + 1e-3 +
// 1e-6*(|cx| + xr)).
#include "sjcs_internal.cuh"

namespace sjcs {
namespace {

constexpr int CT_WARPS = 8;
constexpr int CT_THREADS = CT_WARPS * 32;
constexpr int kMaxSmemTable = 8192;  // r2 entries held in shared memory
constexpr int kMaxSmemRads = 1024;   // per-warp shared counters up to this many shells

enum BinMode { BIN_LUT = 0, BIN_BSEARCH = 1, BIN_FIRST_MATCH = 2 };

struct CountParams {
    const float4* __restrict__ pts;  // sorted particles (x, y, z, unused)
    const uint32_t* __restrict__ cs;
    GridGeom g;
    float h[3];                      // cell edge per axis, 1000 / G
    const float4* __restrict__ halos;
    uint64_t nhalos;
    const float* __restrict__ r2;    // [pad], +inf past nrads
    const uint32_t* __restrict__ lut;
    int nrads;
    int pad;
    int nlut;
    uint32_t lut_k0;                 // bit pattern of r2[0]
    int lut_shift;
    float half;
    float r2max;
    float r2p;                       // r2max * (1 + 1e-5)
    float r2slack;                   // r2max * 1e-5
    int periodic;
    int prune;
    uint32_t* __restrict__ counts;
};

__device__ __forceinline__ float edge_margin(float v) { return 1e-3f + 2e-6f * fabsf(v); }

// Lower bound of |c - y| over every y whose cell index is k.
__device__ __forceinline__ float cell_gap(float c, int k, float h, int G) {
    const float lo_e = (float)k * h, hi_e = (float)(k + 1) * h;
    const float lo = (k == 0) ? -INFINITY : lo_e - edge_margin(lo_e);
    const float hi = (k == G - 1) ? INFINITY : hi_e + edge_margin(hi_e);
    return fmaxf(0.0f, fmaxf(lo - c, c - hi));
}

template <int BIN>
__device__ __forceinline__ int bin_of(const CountParams& p, const float* __restrict__ tab,
                                      const uint32_t* __restrict__ lut, float dist) {
    if (BIN == BIN_LUT) {
        const uint32_t key = __float_as_uint(dist);
        if (key < p.lut_k0) return 0;
        const int s = (int)lut[(key - p.lut_k0) >> p.lut_shift];
        return s + ((tab[s] <= dist) ? 1 : 0);
    } else {
        int s = 0;
        for (int step = p.pad >> 1; step > 0; step >>= 1) s += (tab[s + step - 1] <= dist) ? step : 0;
        return s;
    }
}

// BIG: table too large for shared memory -> table read from global memory and
// counts added with global atomics straight into the halo's row.
template <int BIN, bool BIG>
__device__ __forceinline__ void count_image(const CountParams& p, float cx, float cy, float cz,
                                            uint32_t* __restrict__ sink, const float* __restrict__ tab,
                                            const uint32_t* __restrict__ lut, int lane) {
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
    const int64_t ny = y1 - y0 + 1;
    const int64_t nrows = ny * (int64_t)(z1 - z0 + 1);

    for (int64_t rb = 0; rb < nrows; rb += 32) {
        const int64_t r = rb + lane;
        uint32_t start = 0, len = 0;
        if (r < nrows) {
            const int64_t q = r / ny;
            const int yy = (int)(y0 + r - q * ny), zz = (int)(z0 + q);
            int xa = x0, xb = x1;
            if (p.prune) {
                const float gy = cell_gap(cy, yy, p.h[1], p.g.G[1]);
                const float gz = cell_gap(cz, zz, p.h[2], p.g.G[2]);
                const float rem = __fadd_rn(__fsub_rn(__fsub_rn(p.r2p, __fmul_rn(gy, gy)), __fmul_rn(gz, gz)),
                                            p.r2slack);
                if (rem < 0.0f) {
                    xb = xa - 1;  // no particle of this row can be within R
                } else {
                    float xr = __fsqrt_rn(rem);
                    xr = __fadd_rn(xr, 1e-3f + 1e-6f * (fabsf(cx) + xr));
                    const float xl = __fsub_rn(cx, xr), xh = __fadd_rn(cx, xr);
                    xa = max(xa, cell_of(xl, p.g.inv_h[0], p.g.G[0]));
                    if (xh == xh) xb = min(xb, cell_of(xh, p.g.inv_h[0], p.g.G[0]));
                }
            }
            if (xa <= xb) {
                const uint64_t rowcell = ((uint64_t)zz * (uint64_t)p.g.G[1] + (uint64_t)yy) * (uint64_t)p.g.G[0];
                start = __ldg(p.cs + rowcell + xa);
                len = __ldg(p.cs + rowcell + xb + 1) - start;
            }
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
                const float4 pp = __ldg(p.pts + (t + o));
                const bool inb = !(pp.x < lox) & !(hix < pp.x) & !(pp.y < loy) & !(hiy < pp.y) &
                                 !(pp.z < loz) & !(hiz < pp.z);
                const float dx = __fsub_rn(pp.x, cx), dy = __fsub_rn(pp.y, cy), dz = __fsub_rn(pp.z, cz);
                const float dist =
                    __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
                if (BIN != BIN_FIRST_MATCH) {
                    if (inb && dist < p.r2max) atomicAdd(sink + bin_of<BIN>(p, tab, lut, dist), 1u);
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

template <int BIN, bool BIG>
__global__ void __launch_bounds__(CT_THREADS, 4) k_shell_count(CountParams p) {
    extern __shared__ uint32_t smem[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    float* r2s = reinterpret_cast<float*>(smem);
    uint32_t* luts = smem + p.pad;
    uint32_t* wcnt = luts + p.nlut + warp * p.nrads;
    if (!BIG) {
        for (int i = tid; i < p.pad; i += CT_THREADS) r2s[i] = p.r2[i];
        for (int i = tid; i < p.nlut; i += CT_THREADS) luts[i] = p.lut[i];
        for (int i = tid; i < CT_WARPS * p.nrads; i += CT_THREADS) luts[p.nlut + i] = 0u;
        __syncthreads();
    }
    const float* tab = BIG ? p.r2 : r2s;
    const uint32_t* lut = BIG ? p.lut : luts;
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
                count_image<BIN, BIG>(p, (S & 1u) ? sx : c.x, (S & 2u) ? sy : c.y, (S & 4u) ? sz : c.z, sink, tab,
                                      lut, lane);
                if (S == 0) break;
                S = (S - 1u) & F;
            }
        } else {
            count_image<BIN, BIG>(p, c.x, c.y, c.z, sink, tab, lut, lane);
        }
        if (!BIG) {
            __syncwarp();
            for (int s = lane; s < p.nrads; s += 32) {
                const uint32_t v = wcnt[s];
                if (v) {
                    wcnt[s] = 0u;
                    atomicAdd(row + s, v);  // result unused: compiles to a reduction
                }
            }
            __syncwarp();
        }
    }
}

template <int BIN, bool BIG>
int launch_variant(sjcs_ctx* ctx, const CountParams& p, size_t smem, cudaStream_t s) {
    auto kern = k_shell_count<BIN, BIG>;
    if (smem > 48 * 1024)
        SJCS_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
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
    p.pts = idx->pts;
    p.cs = idx->cell_start;
    p.g = idx->geom;
    for (int a = 0; a < 3; ++a) p.h[a] = 1000.0f / (float)idx->geom.G[a];
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
    const int bin = !q->monotone ? BIN_FIRST_MATCH : (q->nlut > 0 ? BIN_LUT : BIN_BSEARCH);
    const bool big = q->pad > kMaxSmemTable || q->nrads > kMaxSmemRads;
    if (big) p.nlut = q->nlut;  // table and LUT are read from global memory
    const size_t smem = big ? 0 : (size_t)(q->pad + q->nlut + CT_WARPS * q->nrads) * sizeof(uint32_t);
    switch (bin) {
        case BIN_LUT:
            return big ? launch_variant<BIN_LUT, true>(ctx, p, smem, s) : launch_variant<BIN_LUT, false>(ctx, p, smem, s);
        case BIN_BSEARCH:
            return big ? launch_variant<BIN_BSEARCH, true>(ctx, p, smem, s)
                       : launch_variant<BIN_BSEARCH, false>(ctx, p, smem, s);
        default:
            return big ? launch_variant<BIN_FIRST_MATCH, true>(ctx, p, smem, s)
                       : launch_variant<BIN_FIRST_MATCH, false>(ctx, p, smem, s);
    }
}

}  // namespace sjcs
